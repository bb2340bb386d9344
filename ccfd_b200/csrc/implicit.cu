// Implicit backward-Euler path: Newton iteration with matrix-free GMRES and
// the LU-SGS preconditioner.
//
//   implicitTimeStep  src/timeDiscretization.c:412-552
//   GMRES_M           src/linearSolver.c:385-510 (right-preconditioned, one
//                     cycle of nKdim, modified Gram-Schmidt, Givens rotations)
//   matrixVector      src/linearSolver.c:343-373 (finite-difference Jacobian
//                     product (v - alpha dt (R(X + eps v) - R(X)) / eps),
//                     eps = sqrt(DBL_EPSILON) / |v|)
//   buildMatrix       src/linearSolver.c:186-252 (finite-difference Jacobian
//                     with respect to the primitive variables, diagonal and
//                     face-neighbour 4x4 blocks only, I - dt J)
//   calcDinv          src/linearSolver.c:136-179 (4x4 inverse, singular when
//                     |det| <= DBL_EPSILON)
//   LUSGS             src/linearSolver.c:261-333 (forward / backward sweeps in
//                     the reference's cell numbering)
//
// The reference stores the Jacobian densely, (4N)^2 doubles, and builds it
// with 4N residual evaluations.  Here the same entries live in block-sparse
// storage (one 4x4 block per cell and one per half-side) and the columns are
// obtained with 4 residual evaluations per colour of a distance-3 colouring:
// cells of one colour are far enough apart that their perturbations reach
// disjoint sets of recorded residuals.  The sweeps are level-scheduled: a
// cell's level is one more than the highest level among its neighbours of
// lower (forward) / higher (backward) reference number, so every level is a
// set of independent cells and the sweep result is exactly the sequential
// one.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "ccfd_ctx.cuh"
#include "host/ccfd_host.h"
#include "kernels.cuh"

using namespace ccfd;

namespace {

constexpr int kB = 256;  // threads per block of the vector kernels

// device scalars of one implicit step (offsets into ImpState::sc)
enum Sc {
    SC_NORMB = 0, SC_ABORT, SC_EPSFD, SC_NORM_X0, SC_NORM_XK, SC_EPS2LOC, SC_TMP,
    SC_H = 16
};

struct ImpState {
    int K = 0;            // nKdim
    long N = 0;
    double4 *XK = nullptr, *Q = nullptr, *RXK = nullptr, *F = nullptr, *dX = nullptr;
    double4 *W = nullptr, *V = nullptr, *Z = nullptr, *ptmp = nullptr, *ut = nullptr;
    double4 *dxs = nullptr;
    double *D = nullptr, *Dinv = nullptr, *O = nullptr;  // [N][16], [N][16], [H][16]
    double* sc = nullptr;        // device scalars
    int* flag = nullptr;         // [0] gmres done, [1] m_final, [2] singular
    double* partial = nullptr;   // per-block partial sums
    int nb = 0;
    // colouring (device cell lists per colour) and neighbour twins
    std::vector<int> color_off;  // host copy of the colour offsets
    int* color_cells = nullptr;
    int* twin = nullptr;         // [H] half-side of the neighbour that points back
    // LU-SGS level schedules
    int n_lev_f = 0, n_lev_b = 0;
    int *lev_f_off = nullptr, *lev_f_cells = nullptr, *lev_b_off = nullptr, *lev_b_cells = nullptr;
    int *lo_off = nullptr, *lo_nb = nullptr, *lo_h = nullptr;
    int *up_off = nullptr, *up_nb = nullptr, *up_h = nullptr;
    bool ready = false;
};

__device__ __forceinline__ void ld(const double4& v, double q[4]) {
    q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
}
__device__ __forceinline__ double4 mk(const double q[4]) { return make_double4(q[0], q[1], q[2], q[3]); }

// per-cell a.b with the reference's term order (src/linearSolver.c:121-124)
__device__ __forceinline__ double cell_dot(const double4& a, const double4& b) {
    double r = 0.0;
    r += a.x * b.x;
    r += a.y * b.y;
    r += a.z * b.z;
    r += a.w * b.w;
    return r;
}

__device__ __forceinline__ void block_partial(double v, double* partial) {
    __shared__ double sh[32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double x = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) partial[blockIdx.x] = x;
    }
}

__global__ void k_dot(const double4* __restrict__ a, const double4* __restrict__ b, long n,
                      double* __restrict__ partial, const int* __restrict__ skip) {
    if (skip && skip[0]) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = i < n ? cell_dot(a[i], b[i]) : 0.0;
    block_partial(v, partial);
}

// fixed-order final reduction; mode 0: sum, 1: sqrt(sum),
// 2: sqrt(DBL_EPSILON) / sqrt(sum) (the finite-difference step)
__global__ void k_final(const double* __restrict__ partial, int nb, double* out, int mode,
                        const int* __restrict__ skip) {
    if (skip && skip[0]) return;
    __shared__ double sh[kB];
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v += partial[i];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double r = sh[0];
        if (mode == 1) r = sqrt(r);
        else if (mode == 2) r = sqrt(DBL_EPSILON) / sqrt(r);
        *out = r;
    }
}

__global__ void k_copy(double4* __restrict__ dst, const double4* __restrict__ src, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

__global__ void k_cons2prim(const double4* __restrict__ cons, double4* __restrict__ prim, long n,
                            double gam1) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double c[4], p[4];
    ld(cons[i], c);
    cons_prim(gam1, c, p);
    prim[i] = mk(p);
}

// F = (cVar - Q) - alpha dt u_t and its dot partial
// (src/timeDiscretization.c:439-449, 533-536)
__global__ void k_newton_F(const double4* __restrict__ cons, const double4* __restrict__ Q,
                           const double4* __restrict__ ut, double adt, double4* __restrict__ F,
                           long n, double* __restrict__ partial) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        double c[4], q[4], u[4], f[4];
        ld(cons[i], c);
        ld(Q[i], q);
        ld(ut[i], u);
#pragma unroll
        for (int k = 0; k < 4; ++k) f[k] = c[k] - q[k] - adt * u[k];
        double4 fv = mk(f);
        F[i] = fv;
        v = cell_dot(fv, fv);
    }
    block_partial(v, partial);
}

// R0 = -B, delX = 0, V0 = R0 / normR0 (src/linearSolver.c:392-408)
__global__ void k_gmres_init(const double4* __restrict__ B, const double* __restrict__ sc,
                             double4* __restrict__ V0, double4* __restrict__ dX, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double b[4], v[4];
    ld(B[i], b);
    double nr = sc[SC_NORMB];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = -b[k] / nr;
    V0[i] = mk(v);
    dX[i] = make_double4(0.0, 0.0, 0.0, 0.0);
}

// U = XK + eps v, pVar = consPrim(U) (src/linearSolver.c:350-360)
__global__ void k_mv_prep(const double4* __restrict__ XK, const double4* __restrict__ v,
                          const double* __restrict__ sc, double4* __restrict__ prim, long n,
                          double gam1, const int* __restrict__ skip) {
    if (skip[0]) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x[4], z[4], c[4], p[4];
    ld(XK[i], x);
    ld(v[i], z);
    double e = sc[SC_EPSFD];
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = x[k] + e * z[k];
    cons_prim(gam1, c, p);
    prim[i] = mk(p);
}

// W = v - alpha dt (u_t - R_XK) / eps (src/linearSolver.c:364-372), and the
// partial of the first Gram-Schmidt product V0 . W
__global__ void k_mv_finish(const double4* __restrict__ v, const double4* __restrict__ ut,
                            const double4* __restrict__ rxk, const double* __restrict__ sc,
                            double adt, double4* __restrict__ W, const double4* __restrict__ V0,
                            long n, double* __restrict__ partial, const int* __restrict__ skip) {
    if (skip[0]) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double d = 0.0;
    if (i < n) {
        double z[4], u[4], r[4], w[4];
        ld(v[i], z);
        ld(ut[i], u);
        ld(rxk[i], r);
        double e = sc[SC_EPSFD];
#pragma unroll
        for (int k = 0; k < 4; ++k) w[k] = z[k] - adt * (u[k] - r[k]) / e;
        double4 wv = mk(w);
        W[i] = wv;
        d = cell_dot(V0[i], wv);
    }
    block_partial(d, partial);
}

// W -= h V_prev (modified Gram-Schmidt step, src/linearSolver.c:440-450),
// then the partial of V_next . W (or W . W when V_next is null)
__global__ void k_mgs(double4* __restrict__ W, const double4* __restrict__ Vp,
                      const double* __restrict__ h, const double4* __restrict__ Vn, long n,
                      double* __restrict__ partial, const int* __restrict__ skip) {
    if (skip[0]) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double d = 0.0;
    if (i < n) {
        double w[4], p[4];
        ld(W[i], w);
        ld(Vp[i], p);
        double hh = *h;
#pragma unroll
        for (int k = 0; k < 4; ++k) w[k] -= hh * p[k];
        double4 wv = mk(w);
        W[i] = wv;
        d = Vn ? cell_dot(Vn[i], wv) : cell_dot(wv, wv);
    }
    block_partial(d, partial);
}

// Givens rotations, residual estimate and stop test of iteration m, and the
// back substitution when the cycle ends (src/linearSolver.c:454-481)
__global__ void k_givens(double* sc, int* flag, int m, int K) {
    if (flag[0]) return;
    double* H = sc + SC_H;  // H[r * (K + 1) + c]
    double* gam = H + (K + 1) * (K + 1);
    double* C = gam + (K + 1);
    double* S = C + K;
    double* alp = S + K;
    const int ld = K + 1;
    for (int nn = 0; nn <= m - 1; ++nn) {
        double tmp = C[nn] * H[nn * ld + m] + S[nn] * H[(nn + 1) * ld + m];
        H[(nn + 1) * ld + m] = -S[nn] * H[nn * ld + m] + C[nn] * H[(nn + 1) * ld + m];
        H[nn * ld + m] = tmp;
    }
    double bet = sqrt(H[m * ld + m] * H[m * ld + m] + H[(m + 1) * ld + m] * H[(m + 1) * ld + m]);
    S[m] = H[(m + 1) * ld + m] / bet;
    C[m] = H[m * ld + m] / bet;
    H[m * ld + m] = bet;
    gam[m + 1] = -S[m] * gam[m];
    gam[m] = C[m] * gam[m];
    if ((fabs(gam[m + 1]) <= sc[SC_ABORT]) || (m == K - 1)) {
        for (int nn = m; nn >= 0; --nn) {
            alp[nn] = gam[nn];
            for (int o = nn + 1; o <= m; ++o) alp[nn] -= H[nn * ld + o] * alp[o];
            alp[nn] /= H[nn * ld + nn];
        }
        flag[0] = 1;
        flag[1] = m;
        if (!isfinite(alp[0])) flag[3] = 1;
    }
}

// V[m+1] = W / H[m+1][m] (src/linearSolver.c:496-502)
__global__ void k_vnext(const double4* __restrict__ W, const double* __restrict__ h,
                        double4* __restrict__ Vn, long n, const int* __restrict__ flag) {
    if (flag[0]) return;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double w[4];
    ld(W[i], w);
    double hh = *h;
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k] = w[k] / hh;
    Vn[i] = mk(w);
}

// delX += alp[nn] Z[nn], nn = 0..m in order (src/linearSolver.c:482-490)
__global__ void k_delx(double4* __restrict__ dX, const double4* __restrict__ Z,
                       const double* __restrict__ alp, const int* __restrict__ flag, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int m = flag[1];
    double x[4];
    ld(dX[i], x);
    for (int nn = 0; nn <= m; ++nn) {
        double z[4];
        ld(Z[(long)nn * n + i], z);
        double a = alp[nn];
#pragma unroll
        for (int k = 0; k < 4; ++k) x[k] += a * z[k];
    }
    dX[i] = mk(x);
}

// XK += delX, cVar = XK, pVar = consPrim(cVar) (src/timeDiscretization.c:505-520)
__global__ void k_newton_update(double4* __restrict__ XK, const double4* __restrict__ dX,
                                double4* __restrict__ cons, double4* __restrict__ prim, long n,
                                double gam1) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x[4], d[4], p[4];
    ld(XK[i], x);
    ld(dX[i], d);
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] += d[k];
    double4 xv = mk(x);
    XK[i] = xv;
    cons[i] = xv;
    cons_prim(gam1, x, p);
    prim[i] = mk(p);
}

// ---------------------------------------------------------------- Jacobian
// perturb (sign +1) or restore (sign 0) variable v of the cells of a colour
__global__ void k_jac_perturb(double4* __restrict__ prim, const double4* __restrict__ base,
                              const int* __restrict__ cells, int n, int v, double eps, int add) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int d = cells[k];
    double q[4];
    ld(base[d], q);
    if (add) q[v] += eps;
    prim[d] = mk(q);
}

// record column v of the diagonal block of each perturbed cell and of the
// off-diagonal blocks of its face neighbours (src/linearSolver.c:203-222)
__global__ void k_jac_collect(const int* __restrict__ cells, int n, int v,
                              const double4* __restrict__ ut, const double4* __restrict__ rxk,
                              const int* __restrict__ hs_off, const int* __restrict__ hs_nb,
                              const int* __restrict__ twin, double* __restrict__ D,
                              double* __restrict__ O, double sreps) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int d = cells[k];
    double u[4], r[4];
    ld(ut[d], u);
    ld(rxk[d], r);
#pragma unroll
    for (int j = 0; j < 4; ++j) D[16 * (long)d + 4 * j + v] = 0.0 + (u[j] - r[j]) * sreps;
    for (int h = hs_off[d]; h < hs_off[d + 1]; ++h) {
        int e = hs_nb[h];
        if (e < 0) continue;
        ld(ut[e], u);
        ld(rxk[e], r);
        long t = twin[h];
#pragma unroll
        for (int j = 0; j < 4; ++j) O[16 * t + 4 * j + v] = 0.0 + (u[j] - r[j]) * sreps;
    }
}

// own 4x4 inverse by expansion in complementary 2x2 minors; singular when
// |det| <= DBL_EPSILON as in calcDinv
__device__ bool inv4(const double a[16], double r[16]) {
    double s0 = a[0] * a[5] - a[4] * a[1];
    double s1 = a[0] * a[6] - a[4] * a[2];
    double s2 = a[0] * a[7] - a[4] * a[3];
    double s3 = a[1] * a[6] - a[5] * a[2];
    double s4 = a[1] * a[7] - a[5] * a[3];
    double s5 = a[2] * a[7] - a[6] * a[3];
    double c5 = a[10] * a[15] - a[14] * a[11];
    double c4 = a[9] * a[15] - a[13] * a[11];
    double c3 = a[9] * a[14] - a[13] * a[10];
    double c2 = a[8] * a[15] - a[12] * a[11];
    double c1 = a[8] * a[14] - a[12] * a[10];
    double c0 = a[8] * a[13] - a[12] * a[9];
    double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    if (fabs(det) <= DBL_EPSILON) return false;
    double id = 1.0 / det;
    r[0] = (a[5] * c5 - a[6] * c4 + a[7] * c3) * id;
    r[1] = (-a[1] * c5 + a[2] * c4 - a[3] * c3) * id;
    r[2] = (a[13] * s5 - a[14] * s4 + a[15] * s3) * id;
    r[3] = (-a[9] * s5 + a[10] * s4 - a[11] * s3) * id;
    r[4] = (-a[4] * c5 + a[6] * c2 - a[7] * c1) * id;
    r[5] = (a[0] * c5 - a[2] * c2 + a[3] * c1) * id;
    r[6] = (-a[12] * s5 + a[14] * s2 - a[15] * s1) * id;
    r[7] = (a[8] * s5 - a[10] * s2 + a[11] * s1) * id;
    r[8] = (a[4] * c4 - a[5] * c2 + a[7] * c0) * id;
    r[9] = (-a[0] * c4 + a[1] * c2 - a[3] * c0) * id;
    r[10] = (a[12] * s4 - a[13] * s2 + a[15] * s0) * id;
    r[11] = (-a[8] * s4 + a[9] * s2 - a[11] * s0) * id;
    r[12] = (-a[4] * c3 + a[5] * c1 - a[6] * c0) * id;
    r[13] = (a[0] * c3 - a[1] * c1 + a[2] * c0) * id;
    r[14] = (-a[12] * s3 + a[13] * s1 - a[14] * s0) * id;
    r[15] = (a[8] * s3 - a[9] * s1 + a[10] * s0) * id;
    return true;
}

// I - dt J on the stored blocks and the inverses of the diagonal blocks
// (src/linearSolver.c:226-251)
__global__ void k_jac_finish(double* __restrict__ D, double* __restrict__ Dinv,
                             double* __restrict__ O, const int* __restrict__ hs_off, long n,
                             double dt, int* __restrict__ flag) {
    long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    double a[16], r[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = D[16 * d + k] * -dt;
#pragma unroll
    for (int k = 0; k < 4; ++k) a[5 * k] += 1.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) D[16 * d + k] = a[k];
    if (!inv4(a, r)) {
        atomicOr(&flag[2], 1);
#pragma unroll
        for (int k = 0; k < 16; ++k) r[k] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) Dinv[16 * d + k] = r[k];
    for (long h = hs_off[d]; h < hs_off[d + 1]; ++h)
#pragma unroll
        for (int k = 0; k < 16; ++k) O[16 * h + k] = O[16 * h + k] * -dt;
}

// ---------------------------------------------------------------- LU-SGS
// One CTA walks the levels of the forward sweep (lower neighbours), then
// the backward sweep (upper neighbours) (src/linearSolver.c:261-333).
__global__ void __launch_bounds__(1024) k_lusgs(
    const double4* __restrict__ B, double4* __restrict__ dxs, double4* __restrict__ dx,
    const double* __restrict__ Dinv, const double* __restrict__ O, int nlf,
    const int* __restrict__ lf_off, const int* __restrict__ lf_cells, int nlb,
    const int* __restrict__ lb_off, const int* __restrict__ lb_cells,
    const int* __restrict__ lo_off, const int* __restrict__ lo_nb, const int* __restrict__ lo_h,
    const int* __restrict__ up_off, const int* __restrict__ up_nb, const int* __restrict__ up_h,
    const int* __restrict__ skip) {
    if (skip[0]) return;
    for (int L = 0; L < nlf; ++L) {
        for (int k = lf_off[L] + threadIdx.x; k < lf_off[L + 1]; k += blockDim.x) {
            int i = lf_cells[k];
            double t1[4] = {0.0, 0.0, 0.0, 0.0};
            for (int q = lo_off[i]; q < lo_off[i + 1]; ++q) {
                const double* blk = O + 16 * (long)lo_h[q];
                double x[4];
                ld(dxs[lo_nb[q]], x);
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) t1[a] += blk[4 * a + b] * x[b];
            }
            const double* di = Dinv + 16 * (long)i;
            double b[4], t2[4];
            ld(B[i], b);
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                t2[a] = 0.0;
#pragma unroll
                for (int c = 0; c < 4; ++c) t2[a] += di[4 * a + c] * (b[c] - t1[c]);
            }
            dxs[i] = mk(t2);
        }
        __syncthreads();
    }
    for (int L = 0; L < nlb; ++L) {
        for (int k = lb_off[L] + threadIdx.x; k < lb_off[L + 1]; k += blockDim.x) {
            int i = lb_cells[k];
            double t1[4] = {0.0, 0.0, 0.0, 0.0};
            for (int q = up_off[i]; q < up_off[i + 1]; ++q) {
                const double* blk = O + 16 * (long)up_h[q];
                double x[4];
                ld(dx[up_nb[q]], x);
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) t1[a] += blk[4 * a + b] * x[b];
            }
            const double* di = Dinv + 16 * (long)i;
            double s[4], t2[4];
            ld(dxs[i], s);
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                t2[a] = 0.0;
#pragma unroll
                for (int c = 0; c < 4; ++c) t2[a] += di[4 * a + c] * t1[c];
                s[a] = s[a] - t2[a];
            }
            dx[i] = mk(s);
        }
        __syncthreads();
    }
}

}  // namespace

namespace ccfd {
void imp_step_end_launch(Ctrl* ctrl, const StepParams& sp, const double* res_partial, int nres,
                         const double2* dt_partial, const int* dt_bad, int ndt, const int* wall_ghost,
                         const double* wall_nl, const double* ghost_pface, cudaStream_t st);
}

// ------------------------------------------------------------------- host
#define CK(x)                               \
    do {                                    \
        cudaError_t e_ = (x);               \
        if (e_ != cudaSuccess) {            \
            ctx->last_cuda_error = (int)e_; \
            return CCFD_ERR_CUDA;           \
        }                                   \
    } while (0)

template <typename T>
static int ialloc(ccfd_ctx* ctx, T** p, size_t n) {
    void* q = nullptr;
    if (n == 0) n = 1;
    if (cudaMalloc(&q, n * sizeof(T)) != cudaSuccess) return CCFD_ERR_NOMEM;
    ctx->allocs.push_back(q);
    ctx->device_bytes += n * sizeof(T);
    *p = (T*)q;
    return CCFD_OK;
}

template <typename T>
static int iupload(ccfd_ctx* ctx, T** p, const std::vector<T>& h) {
    int st = ialloc(ctx, p, h.size());
    if (st) return st;
    if (!h.empty())
        CK(cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return CCFD_OK;
}

// Host set-up: colouring, twins, level schedules (device cell numbering,
// reference cell order for the sweeps).  Needs the device CSR on the host.
void ccfd_implicit_free(ccfd_ctx* ctx) {
    delete (ImpState*)ctx->implicit_state;
    ctx->implicit_state = nullptr;
}

int ccfd_implicit_setup(ccfd_ctx* ctx, const std::vector<int>& hs_off, const std::vector<int>& hs_nb) {
    ImpState* S = new ImpState();
    ctx->implicit_state = S;
    const long N = ctx->N;
    const int K = std::max(1, ctx->params.n_kdim);
    S->K = K;
    S->N = N;
    S->nb = (int)((N + kB - 1) / kB);
    const long H = hs_off[N];
    int st;
    if ((st = ialloc(ctx, &S->XK, N)) || (st = ialloc(ctx, &S->Q, N)) || (st = ialloc(ctx, &S->RXK, N)) ||
        (st = ialloc(ctx, &S->F, N)) || (st = ialloc(ctx, &S->dX, N)) || (st = ialloc(ctx, &S->W, N)) ||
        (st = ialloc(ctx, &S->V, (size_t)(K + 1) * N)) || (st = ialloc(ctx, &S->Z, (size_t)K * N)) ||
        (st = ialloc(ctx, &S->ptmp, N)) || (st = ialloc(ctx, &S->ut, N)) ||
        (st = ialloc(ctx, &S->sc, SC_H + (K + 1) * (K + 1) + 4 * (K + 1) + 8)) ||
        (st = ialloc(ctx, &S->flag, 8)) || (st = ialloc(ctx, &S->partial, S->nb + 1)))
        return st;
    if (ctx->params.precond) {
        if ((st = ialloc(ctx, &S->D, 16 * (size_t)N)) || (st = ialloc(ctx, &S->Dinv, 16 * (size_t)N)) ||
            (st = ialloc(ctx, &S->O, 16 * (size_t)H)) || (st = ialloc(ctx, &S->dxs, N)))
            return st;
        // twins
        std::vector<int> twin(H, -1);
        for (long d = 0; d < N; ++d)
            for (int h = hs_off[d]; h < hs_off[d + 1]; ++h) {
                int e = hs_nb[h];
                if (e < 0) continue;
                for (int g = hs_off[e]; g < hs_off[e + 1]; ++g)
                    if (hs_nb[g] == (int)d) {
                        twin[h] = g;
                        break;
                    }
            }
        // distance-3 greedy colouring: a cell's colour differs from every
        // cell within three face-neighbour steps
        std::vector<int> color(N, -1), mark(N, -1), frontier, next, seen;
        int ncol = 0;
        std::vector<int> used;
        for (long d = 0; d < N; ++d) {
            seen.clear();
            frontier.assign(1, (int)d);
            mark[d] = (int)d;
            seen.push_back((int)d);
            for (int r = 0; r < 3; ++r) {
                next.clear();
                for (int c : frontier)
                    for (int h = hs_off[c]; h < hs_off[c + 1]; ++h) {
                        int e = hs_nb[h];
                        if (e >= 0 && mark[e] != (int)d) {
                            mark[e] = (int)d;
                            next.push_back(e);
                            seen.push_back(e);
                        }
                    }
                frontier.swap(next);
            }
            used.assign(ncol + 1, 0);
            for (int e : seen)
                if (color[e] >= 0) used[color[e]] = 1;
            int c = 0;
            while (c < ncol && used[c]) ++c;
            color[d] = c;
            if (c == ncol) ++ncol;
        }
        std::vector<int> coff(ncol + 1, 0), ccells(N);
        for (long d = 0; d < N; ++d) coff[color[d] + 1]++;
        for (int c = 0; c < ncol; ++c) coff[c + 1] += coff[c];
        std::vector<int> fill(coff.begin(), coff.end() - 1);
        for (long d = 0; d < N; ++d) ccells[fill[color[d]]++] = (int)d;
        S->color_off = coff;
        // lower / upper neighbour lists in side order, by reference number
        const std::vector<int>& ref = ctx->cell_of_dev;
        std::vector<int> lo_off(N + 1, 0), up_off(N + 1, 0), lo_nb, lo_h, up_nb, up_h;
        for (long d = 0; d < N; ++d) {
            lo_off[d] = (int)lo_nb.size();
            up_off[d] = (int)up_nb.size();
            for (int h = hs_off[d]; h < hs_off[d + 1]; ++h) {
                int e = hs_nb[h];
                if (e < 0) continue;
                if (ref[e] < ref[d]) {
                    lo_nb.push_back(e);
                    lo_h.push_back(h);
                } else {
                    up_nb.push_back(e);
                    up_h.push_back(h);
                }
            }
        }
        lo_off[N] = (int)lo_nb.size();
        up_off[N] = (int)up_nb.size();
        // levels, walking the reference numbering
        std::vector<int> lf(N, 0), lb(N, 0);
        const std::vector<int>& dev = ctx->dev_of_cell;
        int nlf = 0, nlb = 0;
        for (long i = 0; i < N; ++i) {
            int d = dev[i], l = 0;
            for (int q = lo_off[d]; q < lo_off[d + 1]; ++q) l = std::max(l, lf[lo_nb[q]] + 1);
            lf[d] = l;
            nlf = std::max(nlf, l + 1);
        }
        for (long i = N - 1; i >= 0; --i) {
            int d = dev[i], l = 0;
            for (int q = up_off[d]; q < up_off[d + 1]; ++q) l = std::max(l, lb[up_nb[q]] + 1);
            lb[d] = l;
            nlb = std::max(nlb, l + 1);
        }
        auto bucket = [&](const std::vector<int>& lev, int nl, std::vector<int>& off, std::vector<int>& cells) {
            off.assign(nl + 1, 0);
            cells.resize(N);
            for (long d = 0; d < N; ++d) off[lev[d] + 1]++;
            for (int l = 0; l < nl; ++l) off[l + 1] += off[l];
            std::vector<int> f(off.begin(), off.end() - 1);
            for (long d = 0; d < N; ++d) cells[f[lev[d]]++] = (int)d;
        };
        std::vector<int> lfo, lfc, lbo, lbc;
        bucket(lf, nlf, lfo, lfc);
        bucket(lb, nlb, lbo, lbc);
        S->n_lev_f = nlf;
        S->n_lev_b = nlb;
        if ((st = iupload(ctx, &S->twin, twin)) || (st = iupload(ctx, &S->color_cells, ccells)) ||
            (st = iupload(ctx, &S->lo_off, lo_off)) || (st = iupload(ctx, &S->lo_nb, lo_nb)) ||
            (st = iupload(ctx, &S->lo_h, lo_h)) || (st = iupload(ctx, &S->up_off, up_off)) ||
            (st = iupload(ctx, &S->up_nb, up_nb)) || (st = iupload(ctx, &S->up_h, up_h)) ||
            (st = iupload(ctx, &S->lev_f_off, lfo)) || (st = iupload(ctx, &S->lev_f_cells, lfc)) ||
            (st = iupload(ctx, &S->lev_b_off, lbo)) || (st = iupload(ctx, &S->lev_b_cells, lbc)))
            return st;
    }
    CK(cudaMemsetAsync(S->sc, 0, sizeof(double) * (SC_H + (K + 1) * (K + 1) + 4 * (K + 1) + 8), ctx->stream));
    CK(cudaMemsetAsync(S->flag, 0, sizeof(int) * 8, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    S->ready = true;
    return CCFD_OK;
}

// residual of the primitive state `prim` at time `time` into `ut` (fused
// stage kernel in residual mode)
int ccfd_residual_of(ccfd_ctx* ctx, const double4* prim, double time, double4* ut);

static double host_scalar(ccfd_ctx* ctx, const double* p) {
    double v = 0.0;
    cudaMemcpyAsync(&v, p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return v;
}

// buildMatrix (src/linearSolver.c:186-252) at the current primitive state
static int build_matrix(ccfd_ctx* ctx, ImpState* S, double t, double dt) {
    const long N = S->N;
    double4* base = ctx->prim_buf[ctx->cur];
    double4* pert = ctx->prim_buf[ctx->cur ^ 1];
    CK(cudaMemcpyAsync(pert, base, sizeof(double4) * N, cudaMemcpyDeviceToDevice, ctx->stream));
    const double reps = sqrt(DBL_EPSILON), sreps = 1.0 / reps;
    const int ncol = (int)S->color_off.size() - 1;
    for (int c = 0; c < ncol; ++c) {
        int off = S->color_off[c], n = S->color_off[c + 1] - off;
        int nb = (n + kB - 1) / kB;
        for (int v = 0; v < 4; ++v) {
            k_jac_perturb<<<nb, kB, 0, ctx->stream>>>(pert, base, S->color_cells + off, n, v, reps, 1);
            int st = ccfd_residual_of(ctx, pert, t, S->ut);
            if (st) return st;
            k_jac_collect<<<nb, kB, 0, ctx->stream>>>(S->color_cells + off, n, v, S->ut, S->RXK,
                                                      ctx->mesh.hs_off, ctx->mesh.hs_nb, S->twin, S->D, S->O,
                                                      sreps);
            k_jac_perturb<<<nb, kB, 0, ctx->stream>>>(pert, base, S->color_cells + off, n, v, reps, 0);
        }
    }
    k_jac_finish<<<S->nb, kB, 0, ctx->stream>>>(S->D, S->Dinv, S->O, ctx->mesh.hs_off, N, dt, S->flag);
    CK(cudaGetLastError());
    return CCFD_OK;
}

// GMRES_M (src/linearSolver.c:385-510): B = F_XK, result in S->dX
static int gmres(ccfd_ctx* ctx, ImpState* S, double time, double t, double dt, double alpha, int* iters) {
    const long N = S->N;
    const int K = S->K, nb = S->nb;
    const double gam1 = ctx->phys.gam1;
    double* H = S->sc + SC_H;
    double* gam = H + (K + 1) * (K + 1);
    double* alp = gam + (K + 1) + 2 * K;
    int* flag = S->flag;
    cudaStream_t st = ctx->stream;
    // abortCrit = epsGMRES * normB; normR0 = normB; gam[0] = normR0
    double normB = host_scalar(ctx, S->sc + SC_NORMB);
    double hv[2] = {ctx->params.eps_gmres * normB, normB};
    CK(cudaMemcpyAsync(S->sc + SC_ABORT, &hv[0], sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(gam, &hv[1], sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(flag, 0, sizeof(int) * 4, st));
    k_gmres_init<<<nb, kB, 0, st>>>(S->F, S->sc, S->V, S->dX, N);
    if (ctx->params.precond) {
        int s = build_matrix(ctx, S, t, dt);
        if (s) return s;
    }
    const double adt = alpha * dt;
    int m = 0;
    for (m = 0; m < K; ++m) {
        double4* Vm = S->V + (long)m * N;
        double4* Zm = S->Z + (long)m * N;
        if (ctx->params.precond) {
            k_lusgs<<<1, 1024, 0, st>>>(Vm, S->dxs, Zm, S->Dinv, S->O, S->n_lev_f, S->lev_f_off, S->lev_f_cells,
                                        S->n_lev_b, S->lev_b_off, S->lev_b_cells, S->lo_off, S->lo_nb, S->lo_h,
                                        S->up_off, S->up_nb, S->up_h, flag);
        } else {
            k_copy<<<nb, kB, 0, st>>>(Zm, Vm, N);
        }
        // matrixVector: epsFD = sqrt(eps) / |Z|
        k_dot<<<nb, kB, 0, st>>>(Zm, Zm, N, S->partial, flag);
        k_final<<<1, kB, 0, st>>>(S->partial, nb, S->sc + SC_EPSFD, 2, flag);
        k_mv_prep<<<nb, kB, 0, st>>>(S->XK, Zm, S->sc, S->ptmp, N, gam1, flag);
        int s = ccfd_residual_of(ctx, S->ptmp, time, S->ut);
        if (s) return s;
        k_mv_finish<<<nb, kB, 0, st>>>(Zm, S->ut, S->RXK, S->sc, adt, S->W, S->V, N, S->partial, flag);
        // modified Gram-Schmidt
        for (int nn = 0; nn <= m; ++nn) {
            double* hnm = H + nn * (K + 1) + m;
            k_final<<<1, kB, 0, st>>>(S->partial, nb, hnm, 0, flag);
            const double4* Vnext = nn < m ? S->V + (long)(nn + 1) * N : nullptr;
            k_mgs<<<nb, kB, 0, st>>>(S->W, S->V + (long)nn * N, hnm, Vnext, N, S->partial, flag);
        }
        double* hm1 = H + (m + 1) * (K + 1) + m;
        k_final<<<1, kB, 0, st>>>(S->partial, nb, hm1, 1, flag);
        k_givens<<<1, 1, 0, st>>>(S->sc, flag, m, K);
        k_vnext<<<nb, kB, 0, st>>>(S->W, hm1, S->V + (long)(m + 1) * N, N, flag);
        CK(cudaGetLastError());
        int hf[4];
        CK(cudaMemcpyAsync(hf, flag, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (hf[2]) return CCFD_ERR_SINGULAR;
        if (hf[0]) {
            if (hf[3]) return CCFD_ERR_GMRES;
            break;
        }
    }
    k_delx<<<nb, kB, 0, st>>>(S->dX, S->Z, alp, flag, N);
    CK(cudaGetLastError());
    *iters = std::min(m, K - 1) + 1;
    return CCFD_OK;
}

static int finish_partial(ccfd_ctx* ctx, ImpState* S, double* out, int mode) {
    k_final<<<1, kB, 0, ctx->stream>>>(S->partial, S->nb, out, mode, nullptr);
    CK(cudaGetLastError());
    return CCFD_OK;
}

// one implicitTimeStep (src/timeDiscretization.c:412-552) at ctrl->t, ctrl->dt
static int implicit_step(ccfd_ctx* ctx, ImpState* S) {
    const long N = S->N;
    const int nb = S->nb;
    cudaStream_t st = ctx->stream;
    const double gam1 = ctx->phys.gam1;
    const ccfd_params& p = ctx->params;
    Ctrl& c = *ctx->h_ctrl;
    const double t = c.t, dt = c.dt, alpha = 1.0, beta = 1.0;
    double4* prim = ctx->prim_buf[ctx->cur];
    // Q = cVar; pVar = consPrim(cVar)
    k_copy<<<nb, kB, 0, st>>>(S->Q, ctx->cons0, N);
    k_cons2prim<<<nb, kB, 0, st>>>(ctx->cons0, prim, N, gam1);
    const double time = t + beta * dt;
    int s = ccfd_residual_of(ctx, prim, time, S->RXK);
    if (s) return s;
    k_newton_F<<<nb, kB, 0, st>>>(ctx->cons0, S->Q, S->RXK, alpha * dt, S->F, N, S->partial);
    k_copy<<<nb, kB, 0, st>>>(S->XK, ctx->cons0, N);
    if ((s = finish_partial(ctx, S, S->sc + SC_NORM_X0, 0))) return s;
    const double eps2newton = p.eps_newton * p.eps_newton;
    double n0 = host_scalar(ctx, S->sc + SC_NORM_X0);
    double eps2loc = fmax(1e-8 * 1e-8 * N * eps2newton / n0, eps2newton);
    double nk = n0;
    int inner = 0;
    while ((nk > eps2loc * n0) && (inner < p.n_newton_iter)) {
        inner++;
        double nb_ = sqrt(nk);
        CK(cudaMemcpyAsync(S->sc + SC_NORMB, &nb_, sizeof(double), cudaMemcpyHostToDevice, st));
        int it = 0;
        if ((s = gmres(ctx, S, time, t, dt, alpha, &it))) return s;
        ctx->gmres_total += it;
        k_newton_update<<<nb, kB, 0, st>>>(S->XK, S->dX, ctx->cons0, prim, N, gam1);
        if ((s = ccfd_residual_of(ctx, prim, time, S->RXK))) return s;
        k_newton_F<<<nb, kB, 0, st>>>(ctx->cons0, S->Q, S->RXK, alpha * dt, S->F, N, S->partial);
        if ((s = finish_partial(ctx, S, S->sc + SC_NORM_XK, 0))) return s;
        nk = host_scalar(ctx, S->sc + SC_NORM_XK);
        if (!isfinite(nk)) return CCFD_ERR_STATE;
    }
    ctx->newton_total += inner;
    if (inner == p.n_newton_iter) return CCFD_ERR_NEWTON;
    return CCFD_OK;
}

static int run_implicit(ccfd_ctx* ctx, long nsteps, ccfd_report* report) {
    CK(cudaSetDevice(ctx->device));
    ImpState* S = (ImpState*)ctx->implicit_state;
    if (!S || !S->ready) return CCFD_ERR_ARG;
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    Ctrl& c = *ctx->h_ctrl;
    const long long big = (1LL << 62);
    long long stop_at = nsteps > 0 ? c.iter + nsteps : big;
    c.stop_at = stop_at;
    CK(cudaMemcpyAsync(&ctx->ctrl->stop_at, &c.stop_at, sizeof(long long), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(ctx->ev_run0, st));
    int status = CCFD_OK;
    double4* prim = ctx->prim_buf[ctx->cur];
    launch_dt(ctx->mesh, ctx->phys, ctx->ctrl, ctx->sp, prim, ctx->dt_partial, ctx->dt_bad, st);
    launch_step_begin(ctx->ctrl, ctx->sp, ctx->dt_partial, ctx->dt_bad, ctx->nb_cells, st);
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    while (!c.done && c.active && c.iter < stop_at) {
        status = implicit_step(ctx, S);
        if (status) break;
        // global residual of the final residual evaluation, stop tests and
        // the next dt (calcTimeStep of the new state)
        launch_dt(ctx->mesh, ctx->phys, nullptr, ctx->sp, prim, ctx->dt_partial, ctx->dt_bad, st);
        imp_step_end_launch(ctx->ctrl, ctx->sp, ctx->res_partial, ctx->tiles.n_tiles, ctx->dt_partial,
                            ctx->dt_bad, ctx->nb_cells, ctx->wall_ghost, ctx->wall_nl, ctx->ghost_pface, st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    CK(cudaEventRecord(ctx->ev_run1, st));
    CK(cudaEventSynchronize(ctx->ev_run1));
    float run_ms = 0.0f;
    CK(cudaEventElapsedTime(&run_ms, ctx->ev_run0, ctx->ev_run1));
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (report) {
        memset(report, 0, sizeof(*report));
        report->t = c.t;
        report->dt = c.dt;
        report->iterations = c.iter;
        for (int v = 0; v < 6; ++v) report->residual[v] = c.res[v];
        for (int v = 0; v < 4; ++v) report->first_residual[v] = c.res_first[v];
        report->cl = c.cl;
        report->cd = c.cd;
        report->converged = c.converged;
        report->finished = c.finished;
        report->newton_iterations = ctx->newton_total;
        report->gmres_iterations = ctx->gmres_total;
        report->device_ms = run_ms;
    }
    if (status) return status;
    if (c.flags & FLAG_DT) return CCFD_ERR_DT;
    if (c.flags & FLAG_STATE) return CCFD_ERR_STATE;
    return CCFD_OK;
}

extern "C" int ccfd_run_implicit(ccfd_ctx* ctx, long nsteps, ccfd_report* report) {
    if (!ctx || !ctx->uploaded) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    return run_implicit(ctx, nsteps, report);
}

// ---------------------------------------------------------------- batching
// Implicit batch members are stepped one after another by the
// single-instance driver, each within its own step budget; the batch stream
// is idle meanwhile (the member's own stream carries the work).
int ccfd_implicit_batch_join(ccfd_batch*, ccfd_ctx* ctx) {
    ImpState* S = (ImpState*)ctx->implicit_state;
    return (S && S->ready) ? CCFD_OK : CCFD_ERR_ARG;
}

int ccfd_implicit_batch_leave(ccfd_batch*, ccfd_ctx*) { return CCFD_OK; }

int ccfd_implicit_batch_steps(ccfd_batch*, const std::vector<ccfd_ctx*>& members, int steps) {
    for (ccfd_ctx* ctx : members) {
        Ctrl& c = *ctx->h_ctrl;
        CK(cudaMemcpy(&c, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
        if (c.done || c.iter >= c.stop_at) continue;
        long long budget = c.stop_at;
        long n = (long)std::min<long long>(steps, budget - c.iter);
        int st = run_implicit(ctx, n, nullptr);
        // restore the member's own budget (the driver set stop_at for this call)
        CK(cudaMemcpy(&ctx->ctrl->stop_at, &budget, sizeof(long long), cudaMemcpyHostToDevice));
        if (st && st != CCFD_ERR_NEWTON && st != CCFD_ERR_SINGULAR && st != CCFD_ERR_GMRES &&
            st != CCFD_ERR_STATE && st != CCFD_ERR_DT)
            return st;
        if (st) {
            // a failed member stops; its status stays readable in its report
            unsigned f = st == CCFD_ERR_NEWTON ? FLAG_NEWTON : st == CCFD_ERR_SINGULAR ? FLAG_SINGULAR
                       : st == CCFD_ERR_GMRES ? FLAG_GMRES : st == CCFD_ERR_DT ? FLAG_DT : FLAG_STATE;
            CK(cudaMemcpy(&c, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
            c.flags |= f;
            c.done = 1;
            c.active = 0;
            CK(cudaMemcpy(ctx->ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice));
        }
    }
    return CCFD_OK;
}
