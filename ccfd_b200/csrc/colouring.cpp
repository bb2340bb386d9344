// Distance-3 colouring for the coloured finite-difference Jacobian.
//
// Greedy colouring in a fixed visiting order leaves seams where the mesh's
// periodic directions do not match the greedy's colour period (an O-grid
// with an odd number of cells around the airfoil takes 12 colours where the
// interior pattern needs 8).  A tabu search on the k-colouring problem
// (Hertz and de Werra 1987, "Using tabu search techniques for graph
// coloring", Computing 39; the move rule and tenure of Galinier and Hao
// 1999, "Hybrid evolutionary algorithms for graph coloring", J. Comb. Optim.
// 3) then tries k = colours - 1, - 2, ... from the last valid colouring:
// the cells of the removed colour take random colours, and single-cell
// moves that reduce the number of conflicting pairs most (ties broken at
// random, recently left colours forbidden for a while unless a move beats
// the best count so far) run until no conflict is left or the attempt has
// examined its budget of candidate moves (each move scans every
// conflicting cell against every other colour, so the budget bounds the
// work, not the number of moves: an attempt at a colour count below the
// optimum keeps many conflicts and would otherwise take seconds).
#include "colouring.h"

#include <stdint.h>

#include <algorithm>

#include "ccfd_b200.h"

namespace {

struct Rng {
    uint64_t s;
    uint32_t next() {
        // splitmix64
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return (uint32_t)((z ^ (z >> 31)) >> 32);
    }
};

// cells within three face-neighbour steps of each cell (itself excluded)
void balls(long n, const int* hs_off, const int* hs_nb, std::vector<long>& boff, std::vector<int>& badj) {
    boff.assign(n + 1, 0);
    badj.clear();
    badj.reserve((size_t)n * 25);
    std::vector<int> mark(n, -1), frontier, next;
    for (long d = 0; d < n; ++d) {
        boff[d] = (long)badj.size();
        frontier.assign(1, (int)d);
        mark[d] = (int)d;
        for (int r = 0; r < 3; ++r) {
            next.clear();
            for (int c : frontier)
                for (int h = hs_off[c]; h < hs_off[c + 1]; ++h) {
                    const int e = hs_nb[h];
                    if (e >= 0 && mark[e] != (int)d) {
                        mark[e] = (int)d;
                        next.push_back(e);
                        badj.push_back(e);
                    }
                }
            frontier.swap(next);
        }
    }
    boff[n] = (long)badj.size();
}

int greedy(long n, const std::vector<long>& boff, const std::vector<int>& badj, const int* order,
           std::vector<int>& color) {
    color.assign(n, -1);
    std::vector<int> used;
    int ncol = 0;
    for (long k = 0; k < n; ++k) {
        const int d = order ? order[k] : (int)k;
        used.assign(ncol + 1, 0);
        for (long j = boff[d]; j < boff[d + 1]; ++j)
            if (color[badj[j]] >= 0) used[color[badj[j]]] = 1;
        int c = 0;
        while (c < ncol && used[c]) ++c;
        color[d] = c;
        if (c == ncol) ++ncol;
    }
    return ncol;
}

// one attempt at a k-colouring from `color` (colours >= k re-drawn) that
// examines at most `budget` candidate moves; true and the colouring in
// `color` on success
bool tabu_k(long n, const std::vector<long>& boff, const std::vector<int>& badj, int k, long budget, Rng& rng,
            std::vector<int>& color) {
    std::vector<int> c(color);
    for (long d = 0; d < n; ++d)
        if (c[d] >= k) c[d] = (int)(rng.next() % (uint32_t)k);
    // gamma[d][x]: neighbours of d (within three steps) of colour x
    std::vector<int> gamma((size_t)n * k, 0);
    for (long d = 0; d < n; ++d)
        for (long j = boff[d]; j < boff[d + 1]; ++j) gamma[(size_t)d * k + c[badj[j]]]++;
    long conf = 0;
    for (long d = 0; d < n; ++d) conf += gamma[(size_t)d * k + c[d]];
    conf /= 2;
    std::vector<int> tabu((size_t)n * k, 0);
    std::vector<int> confl, pos(n, -1);
    auto update = [&](int v) {
        const bool in = gamma[(size_t)v * k + c[v]] > 0;
        if (in && pos[v] < 0) {
            pos[v] = (int)confl.size();
            confl.push_back(v);
        } else if (!in && pos[v] >= 0) {
            const int last = confl.back();
            confl[pos[v]] = last;
            pos[last] = pos[v];
            confl.pop_back();
            pos[v] = -1;
        }
    };
    for (long d = 0; d < n; ++d) update((int)d);
    long best = conf, examined = 0;
    for (long it = 1; conf > 0 && examined <= budget; ++it) {
        examined += (long)confl.size() * (k - 1) + 1;
        int bv = -1, bc = -1, bd = 1 << 30, ties = 0;
        for (int v : confl) {
            const int* g = &gamma[(size_t)v * k];
            const int cur = g[c[v]];
            for (int x = 0; x < k; ++x) {
                if (x == c[v]) continue;
                const int delta = g[x] - cur;
                if (tabu[(size_t)v * k + x] > it && conf + delta >= best) continue;
                if (delta < bd) {
                    bd = delta;
                    bv = v;
                    bc = x;
                    ties = 1;
                } else if (delta == bd && rng.next() % (uint32_t)(++ties) == 0) {
                    bv = v;
                    bc = x;
                }
            }
        }
        if (bv < 0) continue;
        const int old = c[bv];
        c[bv] = bc;
        conf += bd;
        tabu[(size_t)bv * k + old] = (int)std::min<long>(it + (long)(rng.next() % 10u) + (long)(0.6 * confl.size()),
                                                         0x7fffffffL);
        for (long j = boff[bv]; j < boff[bv + 1]; ++j) {
            const int e = badj[j];
            gamma[(size_t)e * k + old]--;
            gamma[(size_t)e * k + bc]++;
            update(e);
        }
        update(bv);
        best = std::min(best, conf);
    }
    if (conf > 0) return false;
    color.swap(c);
    return true;
}

}  // namespace

long ccfd_colouring_budget(long n) { return 1000000 + 64 * n; }

int ccfd_distance3_colouring(long n, const int* hs_off, const int* hs_nb, const int* order2, long budget,
                             std::vector<int>& color) {
    if (n <= 0) {
        color.clear();
        return 0;
    }
    std::vector<long> boff;
    std::vector<int> badj;
    balls(n, hs_off, hs_nb, boff, badj);
    int ncol = greedy(n, boff, badj, nullptr, color);
    if (order2) {
        std::vector<int> trial;
        const int nc2 = greedy(n, boff, badj, order2, trial);
        if (nc2 < ncol) {
            ncol = nc2;
            color.swap(trial);
        }
    }
    Rng rng{0x5eed2026ull};
    while (ncol > 1 && budget > 0 && tabu_k(n, boff, badj, ncol - 1, budget, rng, color)) --ncol;
    return ncol;
}

extern "C" int ccfd_colour_cells(long n_cells, const long* hs_offset, const long* hs_nb, long budget,
                                 int* color_out, int* n_colors) {
    if (n_cells < 0 || (n_cells > 0 && (!hs_offset || !hs_nb || !color_out)) || !n_colors) return CCFD_ERR_ARG;
    if (n_cells > 0 && (hs_offset[0] != 0 || hs_offset[n_cells] > 0x7fffffffL)) return CCFD_ERR_ARG;
    for (long i = 0; i < n_cells; ++i)
        if (hs_offset[i + 1] < hs_offset[i]) return CCFD_ERR_ARG;
    std::vector<int> off(n_cells + 1), nb(n_cells > 0 ? hs_offset[n_cells] : 0);
    for (long i = 0; i <= n_cells; ++i) off[i] = (int)hs_offset[i];
    for (size_t h = 0; h < nb.size(); ++h) {
        if (hs_nb[h] >= n_cells) return CCFD_ERR_ARG;
        nb[h] = hs_nb[h] < 0 ? -1 : (int)hs_nb[h];
    }
    std::vector<int> color;
    *n_colors = ccfd_distance3_colouring(n_cells, off.data(), nb.data(), nullptr,
                                         budget < 0 ? ccfd_colouring_budget(n_cells) : budget, color);
    std::copy(color.begin(), color.end(), color_out);
    return CCFD_OK;
}
