// Error norms of the flow solution against an exact function (calcErrors,
// src/analyze.c:445-514): L1, L2 and Linf of the primitive variables over
// the element quadrature points, with the solution expanded linearly from
// the barycentre by the limited gradients of the current state.
//
// One thread per cell, grid-stride; each CTA writes its partial sums and
// maxima, which the host adds in CTA order (deterministic for a given
// launch shape).  The reference sums in its element order; only the
// rounding of the sums differs.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "physics.cuh"

namespace ccfd {

constexpr int kErrThreads = 256;

__global__ void __launch_bounds__(kErrThreads)
    k_errors(DevMesh m, const double4* __restrict__ xq, const double4* __restrict__ prim,
             const double4* __restrict__ grad, const Phys* __restrict__ Pg, int which, double time,
             double* __restrict__ partial, unsigned* flags) {
    const Phys& P = *Pg;
    double l1[4] = {0, 0, 0, 0}, l2[4] = {0, 0, 0, 0}, li[4] = {0, 0, 0, 0};
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < m.N; d += gridDim.x * blockDim.x) {
        const double4 c = xq[d];
        const double area = m.cell_geo[d].x;
        const int h0 = m.hs_off[d], h1 = m.hs_off[d + 1];
        const int ns = h1 - h0;
        const bool quad = ns == 4;
        const double w = quad ? area / 6.0 : area / 3.0;
        const double4 pv = prim[d];
        const double p[4] = {pv.x, pv.y, pv.z, pv.w};
        double gx[4] = {0, 0, 0, 0}, gy[4] = {0, 0, 0, 0};
        if (grad) {
            const double4 a = grad[2 * d], b = grad[2 * d + 1];
            gx[0] = a.x; gx[1] = a.y; gx[2] = a.z; gx[3] = a.w;
            gy[0] = b.x; gy[1] = b.y; gy[2] = b.z; gy[3] = b.w;
        }
        for (int k = 0; k < ns + (quad ? 1 : 0); ++k) {
            double x[2], wk;
            if (k < ns) {
                const double4 gw = m.hs_gw[h0 + k];
                x[0] = c.x + gw.x;
                x[1] = c.y + gw.y;
                wk = w;
            } else {
                x[0] = c.z;
                x[1] = c.w;
                wk = area / 3.0;
            }
            double ex[4];
            exact_func(P, which, x, time, ex, flags);
            const double dx = x[0] - c.x, dy = x[1] - c.y;
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const double q = p[v] + dx * gx[v] + dy * gy[v];
                const double err = fabs(ex[v] - q);
                li[v] = fmax(li[v], err);
                l1[v] += err * wk;
                l2[v] += err * err * wk;
            }
        }
    }
    // CTA reduction: warp shuffles, then the warps' values in shared memory
    __shared__ double sh[kErrThreads / 32][12];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        for (int o = 16; o > 0; o >>= 1) {
            l1[v] += __shfl_down_sync(0xffffffffu, l1[v], o);
            l2[v] += __shfl_down_sync(0xffffffffu, l2[v], o);
            li[v] = fmax(li[v], __shfl_down_sync(0xffffffffu, li[v], o));
        }
    }
    if (lane == 0)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            sh[warp][v] = l1[v];
            sh[warp][4 + v] = l2[v];
            sh[warp][8 + v] = li[v];
        }
    __syncthreads();
    if (threadIdx.x < 12) {
        const int k = threadIdx.x;
        double r = sh[0][k];
        for (int w = 1; w < kErrThreads / 32; ++w) r = k < 8 ? r + sh[w][k] : fmax(r, sh[w][k]);
        partial[12 * blockIdx.x + k] = r;
    }
}

// exactFunc at the cell barycentres (the exact-solution output of
// csvOutput / curveOutput, src/output.c:59-71)
__global__ void __launch_bounds__(kErrThreads)
    k_exact_state(int n, const double4* __restrict__ xq, const Phys* __restrict__ Pg, int which, double time,
                  double4* __restrict__ out, unsigned* flags) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const double4 c = xq[d];
    const double x[2] = {c.x, c.y};
    double pv[4];
    exact_func(*Pg, which, x, time, pv, flags);
    out[d] = make_double4(pv[0], pv[1], pv[2], pv[3]);
}

void launch_exact_state(int n, const double4* xq, const Phys* phys_g, int which, double time, double4* out,
                        unsigned* flags, cudaStream_t st) {
    k_exact_state<<<(n + kErrThreads - 1) / kErrThreads, kErrThreads, 0, st>>>(n, xq, phys_g, which, time, out,
                                                                              flags);
}

int error_blocks(int n_cells) {
    int b = (n_cells + kErrThreads - 1) / kErrThreads;
    return b < 1 ? 1 : (b > 1184 ? 1184 : b);
}

void launch_errors(const DevMesh& m, const double4* xq, const double4* prim, const double4* grad,
                   const Phys* phys_g, int which, double time, double* partial, unsigned* flags,
                   cudaStream_t st) {
    k_errors<<<error_blocks(m.N), kErrThreads, 0, st>>>(m, xq, prim, grad, phys_g, which, time, partial,
                                                         flags);
}

}  // namespace ccfd
