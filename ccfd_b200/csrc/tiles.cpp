// Hilbert ordering of cells and construction of the staged tiles of the
// fused stage kernel (see tiles.h).
#include "tiles.h"

#include <algorithm>
#include <cmath>
#include <functional>
#include <memory>
#include <mutex>
#include <stdint.h>
#include <thread>

// Hilbert index of (x, y) on a 2^16 x 2^16 grid (the classical iterative
// quadrant-rotation construction).
static uint64_t hilbert_index(uint32_t x, uint32_t y) {
    const uint32_t n = 1u << 16;
    uint64_t d = 0;
    for (uint32_t s = n / 2; s > 0; s /= 2) {
        uint32_t rx = (x & s) ? 1u : 0u;
        uint32_t ry = (y & s) ? 1u : 0u;
        d += (uint64_t)s * s * ((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = n - 1 - x;
                y = n - 1 - y;
            }
            std::swap(x, y);
        }
    }
    return d;
}

void ccfd_hilbert_order(const ccfd_mesh* m, std::vector<int>& cell_order) {
    const long N = m->n_cells;
    double x0 = m->cell_bary[0], x1 = x0, y0 = m->cell_bary[1], y1 = y0;
    for (long c = 0; c < N; ++c) {
        x0 = std::min(x0, m->cell_bary[2 * c]);
        x1 = std::max(x1, m->cell_bary[2 * c]);
        y0 = std::min(y0, m->cell_bary[2 * c + 1]);
        y1 = std::max(y1, m->cell_bary[2 * c + 1]);
    }
    // square bounding box so that tiles stay compact on elongated domains
    double span = std::max(x1 - x0, y1 - y0);
    if (span <= 0) span = 1.0;
    std::vector<uint64_t> key(N);
    auto keys = [&](long a, long b) {
        for (long c = a; c < b; ++c) {
            double fx = (m->cell_bary[2 * c] - x0) / span, fy = (m->cell_bary[2 * c + 1] - y0) / span;
            uint32_t ix = (uint32_t)std::min(65535.0, std::max(0.0, fx * 65535.0));
            uint32_t iy = (uint32_t)std::min(65535.0, std::max(0.0, fy * 65535.0));
            key[c] = hilbert_index(ix, iy);
        }
    };
    {
        unsigned hw = std::thread::hardware_concurrency();
        long nth = std::max(1L, std::min<long>(hw ? hw : 1, std::min(16L, N / 65536)));
        std::vector<std::thread> pool;
        for (long k = 0; k + 1 < nth; ++k) pool.emplace_back(keys, N * k / nth, N * (k + 1) / nth);
        keys(N * (nth - 1) / nth, N);
        for (std::thread& th : pool) th.join();
    }
    // stable sort of the cells by key (the key is below 2^32): LSD radix
    // sort, four passes of 8 bits
    std::vector<int> a(N), b(N);
    for (long c = 0; c < N; ++c) a[c] = (int)c;
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 8 * pass;
        size_t cnt[257] = {0};
        for (long i = 0; i < N; ++i) ++cnt[((key[a[i]] >> shift) & 255u) + 1];
        for (int k = 0; k < 256; ++k) cnt[k + 1] += cnt[k];
        for (long i = 0; i < N; ++i) b[cnt[(key[a[i]] >> shift) & 255u]++] = a[i];
        a.swap(b);
    }
    cell_order.swap(a);
}

// Reverse Cuthill-McKee ordering of the cell graph (face neighbours):
// breadth-first levels from a cell of least degree (per connected
// component), neighbours in order of increasing degree, the whole order
// reversed (Cuthill and McKee 1969, George 1971).
void ccfd_rcm_order(const ccfd_mesh* m, std::vector<int>& cell_order) {
    const long N = m->n_cells;
    std::vector<int> deg(N), order;
    order.reserve(N);
    for (long c = 0; c < N; ++c) {
        int d = 0;
        for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) d += m->hs_nb[h] >= 0;
        deg[c] = d;
    }
    std::vector<char> seen(N, 0);
    std::vector<int> by_deg(N), nb;
    for (long c = 0; c < N; ++c) by_deg[c] = (int)c;
    std::stable_sort(by_deg.begin(), by_deg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    for (int start : by_deg) {
        if (seen[start]) continue;
        seen[start] = 1;
        size_t head = order.size();
        order.push_back(start);
        while (head < order.size()) {
            const int c = order[head++];
            nb.clear();
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
                const long e = m->hs_nb[h];
                if (e >= 0 && !seen[e]) {
                    seen[e] = 1;
                    nb.push_back((int)e);
                }
            }
            std::stable_sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] < deg[b]; });
            order.insert(order.end(), nb.begin(), nb.end());
        }
    }
    cell_order.assign(order.rbegin(), order.rend());
}

namespace {

// tiles [ta, tb) built by one thread: their concatenated arrays and per-tile
// sizes; u_code entries go straight into the shared array (disjoint ranges)
struct TilePart {
    std::vector<int> counts, e_ref, f_id, f_lr, f_hs, n_e, n_hs, n_f;
    std::vector<int16_t> hs_nbl, hs_loc;
    int max_e = 0, max_g = 0, max_hs = 0, max_f = 0;
};

// per-thread work arrays, reused across calls (a pool shared by all calls):
// fresh cell- and face-sized arrays per thread and call cost more in page
// faults than the tile construction
struct TileScratch {
    std::vector<int> loc, gloc, fmark, E, R1, R2, G, faces, bfaces;
    TilePart part;
};
std::mutex g_scratch_mu;
std::vector<std::unique_ptr<TileScratch>> g_scratch;

std::unique_ptr<TileScratch> take_scratch() {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (g_scratch.empty()) return std::unique_ptr<TileScratch>(new TileScratch());
    std::unique_ptr<TileScratch> s = std::move(g_scratch.back());
    g_scratch.pop_back();
    return s;
}

void give_scratch(std::unique_ptr<TileScratch> s) {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    g_scratch.push_back(std::move(s));
}

void build_range(const ccfd_mesh* m, const std::vector<int>& cperm, const std::vector<int>& cinv,
                 const std::vector<int>& fdev, int T, int ta, int tb, const std::vector<long>& dh,
                 std::vector<int>& u_code, TileScratch& W) {
    const long N = m->n_cells, F = m->n_faces, B = m->n_bc;
    std::vector<int>&loc = W.loc, &gloc = W.gloc, &fmark = W.fmark;
    std::vector<int>&E = W.E, &R1 = W.R1, &R2 = W.R2, &G = W.G, &faces = W.faces, &bfaces = W.bfaces;
    loc.assign(N, -1);
    gloc.assign(B, -1);
    fmark.assign(F, -1);
    TilePart& P = W.part;
    P.counts.clear();
    P.e_ref.clear();
    P.f_id.clear();
    P.f_lr.clear();
    P.f_hs.clear();
    P.n_e.clear();
    P.n_hs.clear();
    P.n_f.clear();
    P.hs_nbl.clear();
    P.hs_loc.clear();
    P.max_e = P.max_g = P.max_hs = P.max_f = 0;
    for (int t = ta; t < tb; ++t) {
        long d0 = (long)t * T, d1 = std::min(N, d0 + T);
        E.clear();
        R1.clear();
        R2.clear();
        G.clear();
        faces.clear();
        bfaces.clear();
        for (long d = d0; d < d1; ++d) {
            loc[d] = (int)E.size();
            E.push_back((int)d);
        }
        auto add_nbrs = [&](long d, std::vector<int>& out) {
            long c = cperm[d];
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
                long nb = m->hs_nb[h];
                if (nb < 0) continue;
                int nd = cinv[nb];
                if (loc[nd] < 0) {
                    loc[nd] = -2;  // claimed
                    out.push_back(nd);
                }
            }
        };
        for (long d = d0; d < d1; ++d) add_nbrs(d, R1);
        for (int d : R1) {
            loc[d] = (int)E.size();
            E.push_back(d);
        }
        for (int d : R1) add_nbrs(d, R2);
        for (int d : R2) {
            loc[d] = (int)E.size();
            E.push_back(d);
        }
        const int nT = (int)(d1 - d0), nG = nT + (int)R1.size(), nEc = (int)E.size();
        // ghosts adjacent to gradient cells
        for (int i = 0; i < nG; ++i) {
            long c = cperm[E[i]];
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
                long nb = m->hs_nb[h];
                if (nb >= 0) continue;
                int g = (int)(-1 - nb);
                if (gloc[g] < 0) {
                    gloc[g] = (int)(E.size() + G.size());
                    G.push_back(g);
                }
            }
        }
        // gradient half-sides: local neighbour index per half-side
        const size_t hs_nbl0 = P.hs_nbl.size();
        const int blk = (int)P.hs_loc.size();
        int hs_local = 0;
        for (int i = 0; i < nG; ++i) {
            P.hs_loc.push_back((int16_t)hs_local);
            long c = cperm[E[i]];
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h, ++hs_local) {
                long nb = m->hs_nb[h];
                int l = nb >= 0 ? loc[cinv[nb]] : gloc[-1 - nb];
                P.hs_nbl.push_back((int16_t)l);
            }
        }
        P.hs_loc.push_back((int16_t)hs_local);
        // faces touching tile cells in first-encounter order: interior
        // faces first, then the tile's boundary faces
        for (long d = d0; d < d1; ++d) {
            long c = cperm[d];
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
                long f = m->hs_face[h];
                if (m->hs_nb[h] < 0) {
                    bfaces.push_back((int)f);
                    continue;
                }
                if (fmark[f] != t) {
                    fmark[f] = t;
                    faces.push_back((int)f);
                }
            }
        }
        const int nFi = (int)faces.size();
        faces.insert(faces.end(), bfaces.begin(), bfaces.end());
        for (size_t j = 0; j < faces.size(); ++j) {
            long f = faces[j];
            long o = m->face_cells[2 * f], nbr = m->face_cells[2 * f + 1];
            int il = loc[cinv[o]];
            int hl = P.hs_loc[blk + il] + (int)(m->face_hs[2 * f] - m->hs_offset[o]);
            if ((int)j < nFi) {
                int ir = loc[cinv[nbr]];
                int hr = P.hs_loc[blk + ir] + (int)(m->face_hs[2 * f + 1] - m->hs_offset[nbr]);
                P.f_id.push_back(fdev[f]);
                P.f_lr.push_back(il | (ir << 16));
                P.f_hs.push_back(hl | (hr << 16));
            } else {
                int g = (int)(-1 - nbr);
                P.f_id.push_back(-1 - g);
                P.f_lr.push_back(il | (gloc[g] << 16));
                P.f_hs.push_back(hl);
            }
            fmark[f] = -3 - (int)j;  // local index for the codes below
        }
        for (long d = d0; d < d1; ++d) {
            long c = cperm[d];
            long k = dh[d];
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h, ++k) {
                int j = -3 - fmark[m->hs_face[h]];
                u_code[k] = 2 * j + (m->hs_sign[h] > 0 ? 0 : 1);
            }
        }
        for (size_t j = 0; j < faces.size(); ++j) fmark[faces[j]] = t;
        P.counts.push_back(nT);
        P.counts.push_back(nG);
        P.counts.push_back(nEc);
        P.counts.push_back((int)(E.size() + G.size()));
        for (int d : E) P.e_ref.push_back(d);
        for (int g : G) P.e_ref.push_back(-1 - g);
        P.n_e.push_back((int)(E.size() + G.size()));
        P.n_hs.push_back((int)(P.hs_nbl.size() - hs_nbl0));
        P.n_f.push_back((int)faces.size());
        P.max_e = std::max(P.max_e, (int)(E.size() + G.size()));
        P.max_g = std::max(P.max_g, nG);
        P.max_hs = std::max(P.max_hs, hs_local);
        P.max_f = std::max(P.max_f, (int)faces.size());
        // reset the local maps
        for (int d : E) loc[d] = -1;
        for (int g : G) gloc[g] = -1;
    }
}

template <typename V>
void append(V& dst, const V& src) {
    dst.insert(dst.end(), src.begin(), src.end());
}

}  // namespace

// Tiles are independent: ranges of tiles are built on several host threads
// (each with its own scratch) and concatenated in tile order, so the result
// does not depend on the thread count.
void ccfd_build_tiles(const ccfd_mesh* m, const std::vector<int>& cperm, const std::vector<int>& cinv,
                      const std::vector<int>& fdev, int T, TileSet& ts) {
    const long N = m->n_cells;
    // (the vectors keep their capacity from an earlier call)
    ts.e_off.clear();
    ts.counts.clear();
    ts.e_ref.clear();
    ts.hs_off.clear();
    ts.hs_nbl.clear();
    ts.hs_loc.clear();
    ts.f_off.clear();
    ts.f_id.clear();
    ts.f_lr.clear();
    ts.f_hs.clear();
    ts.max_e = ts.max_g = ts.max_hs = ts.max_f = 0;
    ts.tile_cells = T;
    ts.n_tiles = (int)((N + T - 1) / T);
    // device half-side offsets (device cell order keeps each cell's
    // reference side order)
    std::vector<long> dh(N + 1);
    dh[0] = 0;
    for (long d = 0; d < N; ++d) {
        long c = cperm[d];
        dh[d + 1] = dh[d] + (m->hs_offset[c + 1] - m->hs_offset[c]);
    }
    ts.u_code.assign(dh[N], 0);
    unsigned hw = std::thread::hardware_concurrency();
    int nth = (int)std::max(1u, std::min(hw ? hw : 1u, 16u));
    nth = std::max(1, std::min(nth, ts.n_tiles / 64));
    std::vector<std::unique_ptr<TileScratch>> work(nth);
    for (int k = 0; k < nth; ++k) work[k] = take_scratch();
    std::vector<std::thread> pool;
    for (int k = 0; k < nth; ++k) {
        int ta = (int)((long)ts.n_tiles * k / nth), tb = (int)((long)ts.n_tiles * (k + 1) / nth);
        if (k + 1 == nth)
            build_range(m, cperm, cinv, fdev, T, ta, tb, dh, ts.u_code, *work[k]);
        else
            pool.emplace_back(build_range, m, std::cref(cperm), std::cref(cinv), std::cref(fdev), T, ta, tb,
                              std::cref(dh), std::ref(ts.u_code), std::ref(*work[k]));
    }
    for (std::thread& th : pool) th.join();
    ts.e_off.push_back(0);
    ts.hs_off.push_back(0);
    ts.f_off.push_back(0);
    for (int k = 0; k < nth; ++k) {
        const TilePart& P = work[k]->part;
        append(ts.counts, P.counts);
        append(ts.e_ref, P.e_ref);
        append(ts.hs_nbl, P.hs_nbl);
        append(ts.hs_loc, P.hs_loc);
        append(ts.f_id, P.f_id);
        append(ts.f_lr, P.f_lr);
        append(ts.f_hs, P.f_hs);
        for (size_t i = 0; i < P.n_e.size(); ++i) {
            ts.e_off.push_back(ts.e_off.back() + P.n_e[i]);
            ts.hs_off.push_back(ts.hs_off.back() + P.n_hs[i]);
            ts.f_off.push_back(ts.f_off.back() + P.n_f[i]);
        }
        ts.max_e = std::max(ts.max_e, P.max_e);
        ts.max_g = std::max(ts.max_g, P.max_g);
        ts.max_hs = std::max(ts.max_hs, P.max_hs);
        ts.max_f = std::max(ts.max_f, P.max_f);
    }
    for (int k = 0; k < nth; ++k) give_scratch(std::move(work[k]));
}
