// Hilbert ordering of cells and construction of the staged tiles of the
// fused stage kernel (see tiles.h).
#include "tiles.h"

#include <algorithm>
#include <cmath>
#include <stdint.h>

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
    for (long c = 0; c < N; ++c) {
        double fx = (m->cell_bary[2 * c] - x0) / span, fy = (m->cell_bary[2 * c + 1] - y0) / span;
        uint32_t ix = (uint32_t)std::min(65535.0, std::max(0.0, fx * 65535.0));
        uint32_t iy = (uint32_t)std::min(65535.0, std::max(0.0, fy * 65535.0));
        key[c] = hilbert_index(ix, iy);
    }
    cell_order.resize(N);
    for (long c = 0; c < N; ++c) cell_order[c] = (int)c;
    std::stable_sort(cell_order.begin(), cell_order.end(),
                     [&](int a, int b) { return key[a] < key[b]; });
}

void ccfd_build_tiles(const ccfd_mesh* m, const std::vector<int>& cperm, const std::vector<int>& cinv,
                      const std::vector<int>& fdev, int T, TileSet& ts) {
    const long N = m->n_cells, F = m->n_faces, B = m->n_bc;
    ts = TileSet();
    ts.tile_cells = T;
    ts.n_tiles = (int)((N + T - 1) / T);
    std::vector<int> loc(N, -1), gloc(B, -1), fmark(F, -1);
    std::vector<int> E, R1, R2, G, faces;
    ts.e_off.push_back(0);
    ts.hs_off.push_back(0);
    ts.f_off.push_back(0);
    // device half-side offsets (device cell order keeps each cell's
    // reference side order)
    std::vector<long> dh(N + 1);
    dh[0] = 0;
    for (long d = 0; d < N; ++d) {
        long c = cperm[d];
        dh[d + 1] = dh[d] + (m->hs_offset[c + 1] - m->hs_offset[c]);
    }
    ts.u_code.assign(dh[N], 0);
    for (int t = 0; t < ts.n_tiles; ++t) {
        long d0 = (long)t * T, d1 = std::min(N, d0 + T);
        E.clear();
        R1.clear();
        R2.clear();
        G.clear();
        faces.clear();
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
        int hs_local = 0;
        for (int i = 0; i < nG; ++i) {
            ts.hs_loc.push_back((int16_t)hs_local);
            long c = cperm[E[i]];
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h, ++hs_local) {
                long nb = m->hs_nb[h];
                int l = nb >= 0 ? loc[cinv[nb]] : gloc[-1 - nb];
                ts.hs_nbl.push_back((int16_t)l);
            }
        }
        ts.hs_loc.push_back((int16_t)hs_local);
        // faces touching tile cells in first-encounter order: interior
        // faces first, then the tile's boundary faces
        std::vector<int> bfaces;
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
        const int blk = (int)ts.hs_loc.size() - (nG + 1);
        for (size_t j = 0; j < faces.size(); ++j) {
            long f = faces[j];
            long o = m->face_cells[2 * f], nbr = m->face_cells[2 * f + 1];
            int il = loc[cinv[o]];
            int hl = ts.hs_loc[blk + il] + (int)(m->face_hs[2 * f] - m->hs_offset[o]);
            if ((int)j < nFi) {
                int ir = loc[cinv[nbr]];
                int hr = ts.hs_loc[blk + ir] + (int)(m->face_hs[2 * f + 1] - m->hs_offset[nbr]);
                ts.f_id.push_back(fdev[f]);
                ts.f_lr.push_back(il | (ir << 16));
                ts.f_hs.push_back(hl | (hr << 16));
            } else {
                int g = (int)(-1 - nbr);
                ts.f_id.push_back(-1 - g);
                ts.f_lr.push_back(il | (gloc[g] << 16));
                ts.f_hs.push_back(hl);
            }
            fmark[f] = -3 - (int)j;  // local index for the codes below
        }
        for (long d = d0; d < d1; ++d) {
            long c = cperm[d];
            long k = dh[d];
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h, ++k) {
                int j = -3 - fmark[m->hs_face[h]];
                ts.u_code[k] = 2 * j + (m->hs_sign[h] > 0 ? 0 : 1);
            }
        }
        for (size_t j = 0; j < faces.size(); ++j) fmark[faces[j]] = t;
        ts.counts.push_back(nT);
        ts.counts.push_back(nG);
        ts.counts.push_back(nEc);
        ts.counts.push_back((int)(E.size() + G.size()));
        for (int d : E) ts.e_ref.push_back(d);
        for (int g : G) ts.e_ref.push_back(-1 - g);
        ts.e_off.push_back((int)ts.e_ref.size());
        ts.hs_off.push_back((int)ts.hs_nbl.size());
        ts.f_off.push_back((int)ts.f_id.size());
        ts.max_e = std::max(ts.max_e, (int)(E.size() + G.size()));
        ts.max_g = std::max(ts.max_g, nG);
        ts.max_hs = std::max(ts.max_hs, hs_local);
        ts.max_f = std::max(ts.max_f, (int)faces.size());
        // reset the local maps
        for (int d : E) loc[d] = -1;
        for (int g : G) gloc[g] = -1;
    }
}
