// Reverse Cuthill-McKee ordering: breadth-first numbering from a minimum
// degree cell, neighbours visited by increasing degree, then reversed.  It
// gives the face gathers of the residual kernels a narrow index bandwidth, so
// consecutive threads touch nearby cell records.
#include <algorithm>
#include <vector>

#include "reorder.h"

void ccfd_rcm_order(const ccfd_mesh* m, std::vector<int>& cell_order, std::vector<int>& face_order) {
    const long N = m->n_cells, F = m->n_faces;
    std::vector<int> deg(N, 0);
    for (long c = 0; c < N; ++c)
        for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h)
            if (m->hs_nb[h] >= 0) deg[c]++;
    std::vector<char> seen(N, 0);
    std::vector<int> order;
    order.reserve(N);
    std::vector<int> nbs;
    for (long start_scan = 0; (long)order.size() < N;) {
        // next component: unvisited cell of minimum degree
        long best = -1;
        for (long c = start_scan; c < N; ++c)
            if (!seen[c] && (best < 0 || deg[c] < deg[best])) best = c;
        while (start_scan < N && seen[start_scan]) ++start_scan;
        seen[best] = 1;
        size_t head = order.size();
        order.push_back((int)best);
        while (head < order.size()) {
            int c = order[head++];
            nbs.clear();
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
                long nb = m->hs_nb[h];
                if (nb >= 0 && !seen[nb]) {
                    seen[nb] = 1;
                    nbs.push_back((int)nb);
                }
            }
            std::stable_sort(nbs.begin(), nbs.end(), [&](int a, int b) { return deg[a] < deg[b]; });
            order.insert(order.end(), nbs.begin(), nbs.end());
        }
    }
    std::reverse(order.begin(), order.end());
    cell_order = order;
    std::vector<int> inv(N);
    for (long i = 0; i < N; ++i) inv[order[i]] = (int)i;
    std::vector<long long> key(F);
    for (long f = 0; f < F; ++f) {
        long c0 = m->face_cells[2 * f], c1 = m->face_cells[2 * f + 1];
        long a = inv[c0], b = c1 >= 0 ? inv[c1] : a;
        key[f] = std::min(a, b) * 4LL * N + std::max(a, b);
    }
    face_order.resize(F);
    for (long f = 0; f < F; ++f) face_order[f] = (int)f;
    std::stable_sort(face_order.begin(), face_order.end(), [&](int a, int b) { return key[a] < key[b]; });
}
