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
//
// Every kernel works on a set of members (independent cases) at once:
// blockIdx.y selects the member's descriptor, blockIdx.x the block of its
// cells.  All members advance in lockstep through the same sequence of
// Newton and Krylov iterations; a member whose GMRES cycle or Newton loop has
// ended (or failed) is switched off by flags in device memory and its blocks
// return at once, so the result of every member is exactly that of the
// member running alone.  A single case is a set of one.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <thread>
#include <tuple>
#include <vector>

#include "ccfd_ctx.cuh"
#include "colouring.h"
#include "host/ccfd_host.h"
#include "kernels.cuh"

using namespace ccfd;

namespace {

constexpr int kB = 256;  // threads per block of the vector kernels
constexpr int kSweepThreads = 512;  // threads of the LU-SGS CTA (one per member), 4 per cell

// device scalars of one implicit step (offsets into ImpState::sc)
enum Sc {
    SC_NORMB = 0, SC_ABORT, SC_EPSFD, SC_NORM_X0, SC_NORM_XK, SC_EPS2LOC, SC_TMP,
    SC_H = 16
};

// per-member control words (ImpDev::ctl)
enum Ctl {
    CTL_NEWTON = 0,    // Newton loop of the current time step running
    CTL_INNER,         // Newton iterations of the current time step
    CTL_GMRES_TOTAL,   // GMRES iterations so far (report)
    CTL_NEWTON_TOTAL,  // Newton iterations so far (report)
    CTL_SKIP_JAC,      // residual evaluations of the Jacobian colour loop skipped
    CTL_STATUS,        // failure status (ccfd_status) of the current step
    CTL_SKIP_NEWTON,   // == !CTL_NEWTON (skip word of the Newton residuals)
    CTL_SKIP_GMRES,    // GMRES iteration skipped (cycle ended or Newton off)
    CTL_WORDS = 8
};

// Device descriptor of one member (pointers into its context and state).
struct ImpDev {
    long N;
    int K, nb, precond, n_newton;
    double gam1, eps_gmres, eps2newton;
    double4 *XK, *Q, *RXK, *F, *dX, *W, *V, *Z, *ptmp, *ut, *dxs, *cons, *prim, *pert;
    double *D, *Dinv, *O, *sc, *partial;
    // mixed precision (fp32 = 1): Krylov basis V, Z, the sweep vector and the
    // LU-SGS blocks D^-1, O in FP32 (Vf, Zf, dxsf, Dinvf, Of instead of the
    // FP64 arrays); residuals, W, the Newton update and GMRES scalars FP64
    int fp32;
    float4 *Vf, *Zf, *dxsf;
    float *Dinvf, *Of;
    double4* rjb;  // mixed precision: R(U, t) of the FP32-flux evaluation, base of the Jacobian columns
    int* flag;  // [0] GMRES cycle done, [1] final m, [2] singular, [3] non-finite
    int* ctl;   // Ctl words
    Ctrl* ctrl;
    const int *hs_off, *hs_nb, *twin;
    int ncol;
    const int *color_off, *color_cells;
    int n_lev_f, n_lev_b;
    // sweeps in level order: level offsets; per position the cell, its
    // lower (forward) / upper (backward) neighbours and the half-sides of
    // their off-diagonal blocks in side order, -1 padded to four
    const int *lev_f_off, *fw_cell, *lev_b_off, *bw_cell;
    const int4 *fw_nb, *fw_h, *bw_nb, *bw_h;
};

struct ImpState {
    int K = 0;            // nKdim
    long N = 0;
    double4 *XK = nullptr, *Q = nullptr, *RXK = nullptr, *F = nullptr, *dX = nullptr;
    double4 *W = nullptr, *V = nullptr, *Z = nullptr, *ptmp = nullptr, *ut = nullptr;
    double4 *dxs = nullptr;
    double *D = nullptr, *Dinv = nullptr, *O = nullptr;  // [N][16], [N][16], [H][16]
    bool fp32 = false;           // mixed precision: the FP32 arrays below instead
    float4 *Vf = nullptr, *Zf = nullptr, *dxsf = nullptr;
    float *Dinvf = nullptr, *Of = nullptr;
    double4* RJB = nullptr;      // mixed precision: base residual of the Jacobian columns
    double* sc = nullptr;        // device scalars
    int* flag = nullptr;         // [0] gmres done, [1] m_final, [2] singular, [3] non-finite
    int* ctl = nullptr;          // Ctl words
    double* partial = nullptr;   // per-block partial sums
    int nb = 0;
    // colouring (device cell lists per colour) and neighbour twins
    std::vector<int> color_off;  // host copy of the colour offsets
    int* color_off_d = nullptr;
    int* color_cells = nullptr;
    int* twin = nullptr;         // [H] half-side of the neighbour that points back
    // LU-SGS level schedules
    int n_lev_f = 0, n_lev_b = 0, max_level = 0;
    int *lev_f_off = nullptr, *fw_cell = nullptr, *lev_b_off = nullptr, *bw_cell = nullptr;
    int4 *fw_nb = nullptr, *fw_h = nullptr, *bw_nb = nullptr, *bw_h = nullptr;
    bool ready = false;
    void* solo = nullptr;        // the member set of this context running alone
    std::vector<int> hs_off_h;   // device CSR offsets of the half-sides (host copy)
    bool jac_built = false;      // ccfd_build_matrix has filled the blocks
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

// Krylov basis access in the member's precision (FP64 arithmetic outside)
__device__ __forceinline__ double4 getV(const ImpDev& d, long k) {
    if (d.fp32) {
        float4 v = d.Vf[k];
        return make_double4(v.x, v.y, v.z, v.w);
    }
    return d.V[k];
}
__device__ __forceinline__ double4 getZ(const ImpDev& d, long k) {
    if (d.fp32) {
        float4 v = d.Zf[k];
        return make_double4(v.x, v.y, v.z, v.w);
    }
    return d.Z[k];
}
__device__ __forceinline__ void putV(const ImpDev& d, long k, double4 v) {
    if (d.fp32) d.Vf[k] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
    else d.V[k] = v;
}
__device__ __forceinline__ void putZ(const ImpDev& d, long k, double4 v) {
    if (d.fp32) d.Zf[k] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
    else d.Z[k] = v;
}

__device__ __forceinline__ bool newton_on(const ImpDev& d) { return d.ctl[CTL_NEWTON] != 0; }
__device__ __forceinline__ bool gmres_on(const ImpDev& d) { return d.ctl[CTL_SKIP_GMRES] == 0; }

// a member's step fails: its Newton loop and GMRES cycle stop, the control
// block records the error and the member does not step again
__device__ void fail_member(const ImpDev& d, int status, unsigned devflag) {
    d.ctl[CTL_STATUS] = status;
    d.ctl[CTL_NEWTON_TOTAL] += d.ctl[CTL_INNER];
    d.ctl[CTL_NEWTON] = 0;
    d.ctl[CTL_SKIP_NEWTON] = 1;
    d.ctl[CTL_SKIP_GMRES] = 1;
    d.flag[0] = 1;
    d.ctrl->flags |= devflag;
    d.ctrl->done = 1;
    d.ctrl->active = 0;
}

#define MEMBER const ImpDev& d = I[blockIdx.y]
#define CELL_INDEX                                           \
    if ((int)blockIdx.x >= d.nb) return;                     \
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x

// start of a time step: members whose control block lets them step run
// their Newton loop
__global__ void kb_step_prepare(const ImpDev* __restrict__ I) {
    MEMBER;
    if (threadIdx.x) return;
    int on = d.ctrl->active != 0;
    d.ctl[CTL_NEWTON] = on;
    d.ctl[CTL_SKIP_NEWTON] = !on;
    d.ctl[CTL_SKIP_GMRES] = 1;
    d.ctl[CTL_INNER] = 0;
    d.ctl[CTL_STATUS] = 0;
}

// Q = cVar; pVar = consPrim(cVar) (src/timeDiscretization.c:420-433)
__global__ void kb_step_begin(const ImpDev* __restrict__ I) {
    MEMBER;
    if (!newton_on(d)) return;
    CELL_INDEX;
    if (i >= d.N) return;
    double c[4], p[4];
    double4 cv = d.cons[i];
    d.Q[i] = cv;
    ld(cv, c);
    cons_prim(d.gam1, c, p);
    d.prim[i] = mk(p);
}

// F = (cVar - Q) - alpha dt u_t and its dot partial; at the step start also
// XK = cVar (src/timeDiscretization.c:439-449, 533-536)
__global__ void kb_newton_F(const ImpDev* __restrict__ I, int copy_xk) {
    MEMBER;
    if (!newton_on(d)) return;
    CELL_INDEX;
    double v = 0.0;
    if (i < d.N) {
        const double adt = 1.0 * d.ctrl->dt;
        double c[4], q[4], u[4], f[4];
        double4 cv = d.cons[i];
        ld(cv, c);
        ld(d.Q[i], q);
        ld(d.RXK[i], u);
#pragma unroll
        for (int k = 0; k < 4; ++k) f[k] = c[k] - q[k] - adt * u[k];
        double4 fv = mk(f);
        d.F[i] = fv;
        if (copy_xk) d.XK[i] = cv;
        v = cell_dot(fv, fv);
    }
    block_partial(v, d.partial);
}

enum FinalTarget { FT_NORM_X0 = 0, FT_NORM_XK, FT_EPSFD, FT_H };

// fixed-order final reduction of a member's partials; mode 0: sum,
// 1: sqrt(sum), 2: sqrt(DBL_EPSILON) / sqrt(sum) (the finite-difference step)
__global__ void kb_final(const ImpDev* __restrict__ I, int target, int row, int col, int mode,
                         int gmres_gate) {
    MEMBER;
    if (gmres_gate ? !gmres_on(d) : !newton_on(d)) return;
    __shared__ double sh[kB];
    double v = 0.0;
    for (int k = threadIdx.x; k < d.nb; k += blockDim.x) v += d.partial[k];
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
        double* out = target == FT_NORM_X0 ? d.sc + SC_NORM_X0
                    : target == FT_NORM_XK ? d.sc + SC_NORM_XK
                    : target == FT_EPSFD   ? d.sc + SC_EPSFD
                                           : d.sc + SC_H + row * (d.K + 1) + col;
        *out = r;
    }
}

// eps2newtonLoc and the first test of the Newton loop
// (src/timeDiscretization.c:469-478)
__global__ void kb_newton_start(const ImpDev* __restrict__ I) {
    MEMBER;
    if (threadIdx.x || !newton_on(d)) return;
    double n0 = d.sc[SC_NORM_X0];
    double eps2loc = fmax(1e-8 * 1e-8 * d.N * d.eps2newton / n0, d.eps2newton);
    d.sc[SC_EPS2LOC] = eps2loc;
    d.sc[SC_NORM_XK] = n0;
    if (!((n0 > eps2loc * n0) && (0 < d.n_newton))) {
        d.ctl[CTL_NEWTON] = 0;
        d.ctl[CTL_SKIP_NEWTON] = 1;
        if (d.n_newton == 0) {
            d.ctl[CTL_STATUS] = CCFD_ERR_NEWTON;
            d.ctrl->flags |= FLAG_NEWTON;
            d.ctrl->done = 1;
            d.ctrl->active = 0;
        }
    }
}

// GMRES set-up: normB = sqrt(|F|^2), abortCrit, gam[0]; R0 = -B, delX = 0,
// V0 = R0 / normR0 (src/linearSolver.c:385-408)
__global__ void kb_gmres_init(const ImpDev* __restrict__ I) {
    MEMBER;
    if (!newton_on(d)) return;
    CELL_INDEX;
    const double nr = sqrt(d.sc[SC_NORM_XK]);
    if (i == 0) {
        double* H = d.sc + SC_H;
        double* gam = H + (d.K + 1) * (d.K + 1);
        d.sc[SC_NORMB] = nr;
        d.sc[SC_ABORT] = d.eps_gmres * nr;
        gam[0] = nr;
    }
    if (i >= d.N) return;
    double b[4], v[4];
    ld(d.F[i], b);
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = -b[k] / nr;
    putV(d, i, mk(v));
    d.dX[i] = make_double4(0.0, 0.0, 0.0, 0.0);
}

// flags of a new GMRES cycle (after kb_gmres_init has run on every block)
__global__ void kb_gmres_flags(const ImpDev* __restrict__ I) {
    MEMBER;
    if (threadIdx.x) return;
    int on = newton_on(d);
    d.flag[0] = on ? 0 : 1;
    d.flag[1] = d.flag[2] = d.flag[3] = 0;
    d.ctl[CTL_SKIP_GMRES] = !on;
}

// Z_m = V_m when the preconditioner is off
__global__ void kb_copy_vz(const ImpDev* __restrict__ I, int m) {
    MEMBER;
    if (d.precond || !gmres_on(d)) return;
    CELL_INDEX;
    if (i < d.N) putZ(d, (long)m * d.N + i, getV(d, (long)m * d.N + i));
}

__global__ void kb_dot_zz(const ImpDev* __restrict__ I, int m) {
    MEMBER;
    if (!gmres_on(d)) return;
    CELL_INDEX;
    double v = 0.0;
    if (i < d.N) {
        double4 z = getZ(d, (long)m * d.N + i);
        v = cell_dot(z, z);
    }
    block_partial(v, d.partial);
}

// U = XK + eps v, pVar = consPrim(U) (src/linearSolver.c:350-360)
__global__ void kb_mv_prep(const ImpDev* __restrict__ I, int m) {
    MEMBER;
    if (!gmres_on(d)) return;
    CELL_INDEX;
    if (i >= d.N) return;
    double x[4], z[4], c[4], p[4];
    ld(d.XK[i], x);
    ld(getZ(d, (long)m * d.N + i), z);
    double e = d.sc[SC_EPSFD];
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = x[k] + e * z[k];
    cons_prim(d.gam1, c, p);
    d.ptmp[i] = mk(p);
}

// W = v - alpha dt (u_t - R_XK) / eps (src/linearSolver.c:364-372), and the
// partial of the first Gram-Schmidt product V0 . W
__global__ void kb_mv_finish(const ImpDev* __restrict__ I, int m) {
    MEMBER;
    if (!gmres_on(d)) return;
    CELL_INDEX;
    double dd = 0.0;
    if (i < d.N) {
        const double adt = 1.0 * d.ctrl->dt;
        double z[4], u[4], r[4], w[4];
        ld(getZ(d, (long)m * d.N + i), z);
        ld(d.ut[i], u);
        ld(d.RXK[i], r);
        double e = d.sc[SC_EPSFD];
#pragma unroll
        for (int k = 0; k < 4; ++k) w[k] = z[k] - adt * (u[k] - r[k]) / e;
        double4 wv = mk(w);
        d.W[i] = wv;
        dd = cell_dot(getV(d, i), wv);
    }
    block_partial(dd, d.partial);
}

// W -= H[nn][m] V_nn (modified Gram-Schmidt step, src/linearSolver.c:
// 440-450), then the partial of V_{nn+1} . W (or W . W after the last one)
__global__ void kb_mgs(const ImpDev* __restrict__ I, int nn, int m) {
    MEMBER;
    if (!gmres_on(d)) return;
    CELL_INDEX;
    double dd = 0.0;
    if (i < d.N) {
        double w[4], p[4];
        ld(d.W[i], w);
        ld(getV(d, (long)nn * d.N + i), p);
        double hh = d.sc[SC_H + nn * (d.K + 1) + m];
#pragma unroll
        for (int k = 0; k < 4; ++k) w[k] -= hh * p[k];
        double4 wv = mk(w);
        d.W[i] = wv;
        dd = nn < m ? cell_dot(getV(d, (long)(nn + 1) * d.N + i), wv) : cell_dot(wv, wv);
    }
    block_partial(dd, d.partial);
}

// Givens rotations, residual estimate and stop test of iteration m, and the
// back substitution when the cycle ends (src/linearSolver.c:454-481)
__global__ void kb_givens(const ImpDev* __restrict__ I, int m) {
    MEMBER;
    if (threadIdx.x || !gmres_on(d)) return;
    const int K = d.K;
    double* sc = d.sc;
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
        d.flag[0] = 1;
        d.flag[1] = m;
        if (!isfinite(alp[0])) d.flag[3] = 1;
        d.ctl[CTL_SKIP_GMRES] = 1;
    }
}

// V[m+1] = W / H[m+1][m] (src/linearSolver.c:496-502)
__global__ void kb_vnext(const ImpDev* __restrict__ I, int m) {
    MEMBER;
    if (!gmres_on(d)) return;
    CELL_INDEX;
    if (i >= d.N) return;
    double w[4];
    ld(d.W[i], w);
    double hh = d.sc[SC_H + (m + 1) * (d.K + 1) + m];
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k] = w[k] / hh;
    putV(d, (long)(m + 1) * d.N + i, mk(w));
}

// end of a GMRES cycle: iteration count, breakdown test
__global__ void kb_gmres_end(const ImpDev* __restrict__ I) {
    MEMBER;
    if (threadIdx.x || !newton_on(d)) return;
    d.ctl[CTL_GMRES_TOTAL] += min(d.flag[1], d.K - 1) + 1;
    if (d.flag[3]) fail_member(d, CCFD_ERR_GMRES, FLAG_GMRES);
}

// delX += alp[nn] Z[nn], nn = 0..m in order (src/linearSolver.c:482-490);
// XK += delX, cVar = XK, pVar = consPrim(cVar) (src/timeDiscretization.c:
// 505-520)
__global__ void kb_newton_update(const ImpDev* __restrict__ I) {
    MEMBER;
    if (!newton_on(d)) return;
    CELL_INDEX;
    if (i >= d.N) return;
    const double* alp = d.sc + SC_H + (d.K + 1) * (d.K + 1) + (d.K + 1) + 2 * d.K;
    int m = d.flag[1];
    double x[4];
    ld(d.dX[i], x);
    for (int nn = 0; nn <= m; ++nn) {
        double z[4];
        ld(getZ(d, (long)nn * d.N + i), z);
        double a = alp[nn];
#pragma unroll
        for (int k = 0; k < 4; ++k) x[k] += a * z[k];
    }
    d.dX[i] = mk(x);
    double xk[4], p[4];
    ld(d.XK[i], xk);
#pragma unroll
    for (int k = 0; k < 4; ++k) xk[k] += x[k];
    double4 xv = mk(xk);
    d.XK[i] = xv;
    d.cons[i] = xv;
    cons_prim(d.gam1, xk, p);
    d.prim[i] = mk(p);
}

// Newton loop test after an update (src/timeDiscretization.c:478-549)
__global__ void kb_newton_check(const ImpDev* __restrict__ I) {
    MEMBER;
    if (threadIdx.x || !newton_on(d)) return;
    int inner = ++d.ctl[CTL_INNER];
    double nk = d.sc[SC_NORM_XK], n0 = d.sc[SC_NORM_X0], eps2loc = d.sc[SC_EPS2LOC];
    if (!isfinite(nk)) {
        fail_member(d, CCFD_ERR_STATE, FLAG_STATE);
        return;
    }
    if ((nk > eps2loc * n0) && (inner < d.n_newton)) return;
    if (inner == d.n_newton) {
        fail_member(d, CCFD_ERR_NEWTON, FLAG_NEWTON);
        return;
    }
    d.ctl[CTL_NEWTON_TOTAL] += inner;
    d.ctl[CTL_NEWTON] = 0;
    d.ctl[CTL_SKIP_NEWTON] = 1;
}

// ---------------------------------------------------------------- Jacobian
// Perturbation of the finite-difference columns.  FP64: sqrt(DBL_EPSILON), as
// buildMatrix (src/linearSolver.c:199).  Mixed precision evaluates the
// columns with FP32 reconstruction and fluxes (the preconditioner only sets
// how fast GMRES converges, not the converged state), where a step below the
// FP32 resolution of the state would vanish: sqrt(FLT_EPSILON), the step that
// balances truncation and rounding error, with an FP32-flux R(U) as base.
__device__ __forceinline__ double jac_eps(const ImpDev& d) {
    return d.fp32 ? sqrt((double)FLT_EPSILON) : sqrt(DBL_EPSILON);
}

// gate of colour c: members that build a preconditioner and have colour c
__global__ void kb_jac_gate(const ImpDev* __restrict__ I, int c) {
    MEMBER;
    if (threadIdx.x) return;
    d.ctl[CTL_SKIP_JAC] = !(newton_on(d) && d.precond && c < d.ncol);
}

// perturbed copy of the state (buildMatrix works on a copy of pVar)
__global__ void kb_jac_copy(const ImpDev* __restrict__ I) {
    MEMBER;
    if (!newton_on(d) || !d.precond) return;
    CELL_INDEX;
    if (i < d.N) d.pert[i] = d.prim[i];
}

// perturb (add) or restore variable v of the cells of colour c
__global__ void kb_jac_perturb(const ImpDev* __restrict__ I, int c, int v, int add) {
    MEMBER;
    if (d.ctl[CTL_SKIP_JAC]) return;
    const int off = d.color_off[c], n = d.color_off[c + 1] - off;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double reps = jac_eps(d);
    int cell = d.color_cells[off + k];
    double q[4];
    ld(d.prim[cell], q);
    if (add) q[v] += reps;
    d.pert[cell] = mk(q);
}

// record column v of the diagonal block of each perturbed cell and of the
// off-diagonal blocks of its face neighbours (src/linearSolver.c:203-222)
__global__ void kb_jac_collect(const ImpDev* __restrict__ I, int c, int v) {
    MEMBER;
    if (d.ctl[CTL_SKIP_JAC]) return;
    const int off = d.color_off[c], n = d.color_off[c + 1] - off;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double sreps = 1.0 / jac_eps(d);
    const double4* base = d.fp32 ? d.rjb : d.RXK;
    int cell = d.color_cells[off + k];
    double u[4], r[4];
    ld(d.ut[cell], u);
    ld(base[cell], r);
#pragma unroll
    for (int j = 0; j < 4; ++j) d.D[16 * (long)cell + 4 * j + v] = 0.0 + (u[j] - r[j]) * sreps;
    for (int h = d.hs_off[cell]; h < d.hs_off[cell + 1]; ++h) {
        int e = d.hs_nb[h];
        if (e < 0) continue;
        ld(d.ut[e], u);
        ld(base[e], r);
        long t = d.twin[h];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double o = 0.0 + (u[j] - r[j]) * sreps;
            if (d.fp32) d.Of[16 * t + 4 * j + v] = (float)o;
            else d.O[16 * t + 4 * j + v] = o;
        }
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
__global__ void kb_jac_finish(const ImpDev* __restrict__ I) {
    MEMBER;
    if (!newton_on(d) || !d.precond) return;
    CELL_INDEX;
    if (i >= d.N) return;
    const double dt = d.ctrl->dt;
    double a[16], r[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = d.D[16 * i + k] * -dt;
#pragma unroll
    for (int k = 0; k < 4; ++k) a[5 * k] += 1.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) d.D[16 * i + k] = a[k];
    if (!inv4(a, r)) {
        atomicOr(&d.flag[2], 1);
#pragma unroll
        for (int k = 0; k < 16; ++k) r[k] = 0.0;
    }
    if (d.fp32) {
#pragma unroll
        for (int k = 0; k < 16; ++k) d.Dinvf[16 * i + k] = (float)r[k];
        for (long h = d.hs_off[i]; h < d.hs_off[i + 1]; ++h)
#pragma unroll
            for (int k = 0; k < 16; ++k) d.Of[16 * h + k] = (float)((double)d.Of[16 * h + k] * -dt);
    } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) d.Dinv[16 * i + k] = r[k];
        for (long h = d.hs_off[i]; h < d.hs_off[i + 1]; ++h)
#pragma unroll
            for (int k = 0; k < 16; ++k) d.O[16 * h + k] = d.O[16 * h + k] * -dt;
    }
}

// a singular diagonal block ends the member's step
// (src/linearSolver.c:245-249)
__global__ void kb_jac_check(const ImpDev* __restrict__ I) {
    MEMBER;
    if (threadIdx.x || !newton_on(d) || !d.precond) return;
    if (d.flag[2]) fail_member(d, CCFD_ERR_SINGULAR, FLAG_SINGULAR);
}

// ---------------------------------------------------------------- LU-SGS
// Four consecutive threads treat one cell of a level, thread a its row a:
// forward  dxs_i = Dinv_i (b_i - sum_lower O_ij dxs_j)
// backward dx_i  = dxs_i - Dinv_i (sum_upper O_ij dx_j)
// Row a of the neighbour sum accumulates the neighbours in side order and
// the columns in order, exactly as the reference's loops do; the four rows
// are exchanged by shuffles for the product with Dinv_i.  All loads of a
// cell depend only on its indices (prefetched one level ahead) and on
// results of earlier levels, so they are issued together.
template <typename T> struct Vec4;
template <> struct Vec4<double> { using t = double4; };
template <> struct Vec4<float> { using t = float4; };

template <bool FWD, typename T>
__device__ __forceinline__ void sweep_row(int i, int4 nb, int4 hh, int a, unsigned mask, int lane0,
                                          const T* __restrict__ B, const T* src, T* dst, const T* dxs,
                                          const T* __restrict__ Dinv, const T* __restrict__ O) {
    using V4 = typename Vec4<T>::t;
    const int nbv[4] = {nb.x, nb.y, nb.z, nb.w};
    const int hv[4] = {hh.x, hh.y, hh.z, hh.w};
    // component a of each neighbour state and row a of each block
    T xa[4];
    V4 orow[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (nbv[q] >= 0) {
            xa[q] = src[4 * (long)nbv[q] + a];
            orow[q] = reinterpret_cast<const V4*>(O + 16 * (long)hv[q])[a];
        }
    const V4 drow = reinterpret_cast<const V4*>(Dinv + 16 * (long)i)[a];
    const T own_a = FWD ? B[4 * (long)i + a] : dxs[4 * (long)i + a];
    T t1a = T(0.0);
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (nbv[q] >= 0) {
            const T o[4] = {orow[q].x, orow[q].y, orow[q].z, orow[q].w};
#pragma unroll
            for (int b = 0; b < 4; ++b) t1a += o[b] * __shfl_sync(mask, xa[q], lane0 + b);
        }
    const T di[4] = {drow.x, drow.y, drow.z, drow.w};
    T t2 = T(0.0);
    if (FWD) {
#pragma unroll
        for (int c = 0; c < 4; ++c)
            t2 += di[c] * (__shfl_sync(mask, own_a, lane0 + c) - __shfl_sync(mask, t1a, lane0 + c));
        dst[4 * (long)i + a] = t2;
    } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) t2 += di[c] * __shfl_sync(mask, t1a, lane0 + c);
        dst[4 * (long)i + a] = own_a - t2;
    }
}

template <bool FWD, typename T>
__device__ __forceinline__ void sweep(int nl, const int* __restrict__ off, const int* __restrict__ cell,
                                      const int4* __restrict__ nbs, const int4* __restrict__ hs,
                                      const T* __restrict__ B, const T* src, T* dst, const T* dxs,
                                      const T* __restrict__ Dinv, const T* __restrict__ O) {
    // the cell count per pass is a multiple of 8, so the four threads of a
    // cell always sit in one aligned quarter of a warp
    const int g = threadIdx.x >> 2, a = threadIdx.x & 3, ng = blockDim.x >> 2;
    const int lane0 = (threadIdx.x & 31) & ~3;
    const unsigned mask = 0xfu << lane0;
    int p = nl > 0 ? off[0] + g : 0;
    int end = nl > 0 ? off[1] : 0;
    bool have = p < end;
    int ci = 0;
    int4 nb = make_int4(-1, -1, -1, -1), hh = nb;
    if (have) {
        ci = cell[p];
        nb = nbs[p];
        hh = hs[p];
    }
    for (int L = 0; L < nl; ++L) {
        // prefetch the first position of the next level
        const int nend = L + 1 < nl ? off[L + 2] : end;
        const int np = end + g;
        const bool nhave = L + 1 < nl && np < nend;
        int nci = 0;
        int4 nnb = make_int4(-1, -1, -1, -1), nhh = nnb;
        if (nhave) {
            nci = cell[np];
            nnb = nbs[np];
            nhh = hs[np];
        }
        if (have) {
            int q = p;
            while (true) {
                sweep_row<FWD, T>(ci, nb, hh, a, mask, lane0, B, src, dst, dxs, Dinv, O);
                q += ng;
                if (q >= end) break;
                ci = cell[q];
                nb = nbs[q];
                hh = hs[q];
            }
        }
        __syncthreads();
        p = np;
        end = nend;
        have = nhave;
        ci = nci;
        nb = nnb;
        hh = nhh;
    }
}

// One CTA per member: the forward sweep, then the backward sweep
// (src/linearSolver.c:261-333): Z_m = LU-SGS(V_m), in the member's precision
// (members of the other precision are left to the other instantiation);
// THREADS / 4 cells of a level per pass.  512 threads: 1024 would take wide
// levels in one pass, but the register cap they impose spills and is slower
// (measured).
template <int THREADS, typename T>
__global__ void __launch_bounds__(THREADS) kb_lusgs(const ImpDev* __restrict__ I, int m) {
    const ImpDev& d = I[blockIdx.x];
    if (!d.precond || !gmres_on(d) || d.fp32 != (sizeof(T) == 4)) return;
    const T *B, *Dinv, *O;
    T *dxs, *dx;
    if constexpr (sizeof(T) == 8) {
        B = reinterpret_cast<const T*>(d.V + (long)m * d.N);
        dxs = reinterpret_cast<T*>(d.dxs);
        dx = reinterpret_cast<T*>(d.Z + (long)m * d.N);
        Dinv = reinterpret_cast<const T*>(d.Dinv);
        O = reinterpret_cast<const T*>(d.O);
    } else {
        B = reinterpret_cast<const T*>(d.Vf + (long)m * d.N);
        dxs = reinterpret_cast<T*>(d.dxsf);
        dx = reinterpret_cast<T*>(d.Zf + (long)m * d.N);
        Dinv = reinterpret_cast<const T*>(d.Dinvf);
        O = reinterpret_cast<const T*>(d.Of);
    }
    sweep<true, T>(d.n_lev_f, d.lev_f_off, d.fw_cell, d.fw_nb, d.fw_h, B, dxs, dxs, dxs, Dinv, O);
    sweep<false, T>(d.n_lev_b, d.lev_b_off, d.bw_cell, d.bw_nb, d.bw_h, B, dx, dx, dxs, Dinv, O);
}

// number of members whose Newton loop (what = 0) / GMRES cycle (what = 1)
// is still running
__global__ void kb_count(const ImpDev* __restrict__ I, int n, int what, int* out) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const ImpDev& d = I[k];
        int on = what ? gmres_on(d) : newton_on(d);
        if (on) atomicAdd(&cnt, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) *out = cnt;
}

}  // namespace

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
    if (ccfd_malloc_async(&q, n * sizeof(T), ctx->stream) != cudaSuccess) return CCFD_ERR_NOMEM;
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
struct ImpSet;
static void set_free(ImpSet* M);

void ccfd_implicit_free(ccfd_ctx* ctx) {
    ImpState* S = (ImpState*)ctx->implicit_state;
    if (S && S->solo) set_free((ImpSet*)S->solo);
    delete S;
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
    S->hs_off_h = hs_off;
    const long H = hs_off[N];
    int st;
    S->fp32 = ctx->params.precision == CCFD_MIXED;
    if (S->fp32) {
        if ((st = ialloc(ctx, &S->Vf, (size_t)(K + 1) * N)) || (st = ialloc(ctx, &S->Zf, (size_t)K * N)))
            return st;
    } else if ((st = ialloc(ctx, &S->V, (size_t)(K + 1) * N)) || (st = ialloc(ctx, &S->Z, (size_t)K * N))) {
        return st;
    }
    if ((st = ialloc(ctx, &S->XK, N)) || (st = ialloc(ctx, &S->Q, N)) || (st = ialloc(ctx, &S->RXK, N)) ||
        (st = ialloc(ctx, &S->F, N)) || (st = ialloc(ctx, &S->dX, N)) || (st = ialloc(ctx, &S->W, N)) ||
        (st = ialloc(ctx, &S->ptmp, N)) || (st = ialloc(ctx, &S->ut, N)) ||
        (st = ialloc(ctx, &S->sc, SC_H + (K + 1) * (K + 1) + 4 * (K + 1) + 8)) ||
        (st = ialloc(ctx, &S->flag, 8)) || (st = ialloc(ctx, &S->ctl, CTL_WORDS)) ||
        (st = ialloc(ctx, &S->partial, S->nb + 1)))
        return st;
    if (ctx->params.precond) {
        if ((st = ialloc(ctx, &S->D, 16 * (size_t)N))) return st;
        if (S->fp32) {
            if ((st = ialloc(ctx, &S->Dinvf, 16 * (size_t)N)) || (st = ialloc(ctx, &S->Of, 16 * (size_t)H)) ||
                (st = ialloc(ctx, &S->RJB, N)) ||
                (st = ialloc(ctx, &S->dxsf, N)))
                return st;
        } else if ((st = ialloc(ctx, &S->Dinv, 16 * (size_t)N)) || (st = ialloc(ctx, &S->O, 16 * (size_t)H)) ||
                   (st = ialloc(ctx, &S->dxs, N))) {
            return st;
        }
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
        // distance-3 colouring: a cell's colour differs from every cell
        // within three face-neighbour steps (greedy in device and in
        // reference order, then colours removed by a bounded tabu search);
        // any valid colouring gives the same entries
        std::vector<int> color;
        const int ncol = ccfd_distance3_colouring(N, hs_off.data(), hs_nb.data(), ctx->dev_of_cell.data(),
                                                  ccfd_colouring_budget(N), color);
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
        auto pack = [&](const std::vector<int>& cells, const std::vector<int>& off, const std::vector<int>& nb,
                        const std::vector<int>& hh, std::vector<int4>& pn, std::vector<int4>& ph) {
            pn.assign(N, make_int4(-1, -1, -1, -1));
            ph.assign(N, make_int4(-1, -1, -1, -1));
            for (long k = 0; k < N; ++k) {
                int d = cells[k], c = 0;
                int* n4 = &pn[k].x;
                int* h4 = &ph[k].x;
                for (int q = off[d]; q < off[d + 1]; ++q, ++c) {
                    n4[c] = nb[q];
                    h4[c] = hh[q];
                }
            }
        };
        std::vector<int4> fwn, fwh, bwn, bwh;
        pack(lfc, lo_off, lo_nb, lo_h, fwn, fwh);
        pack(lbc, up_off, up_nb, up_h, bwn, bwh);
        S->n_lev_f = nlf;
        S->n_lev_b = nlb;
        for (int l = 0; l < nlf; ++l) S->max_level = std::max(S->max_level, lfo[l + 1] - lfo[l]);
        for (int l = 0; l < nlb; ++l) S->max_level = std::max(S->max_level, lbo[l + 1] - lbo[l]);
        if ((st = iupload(ctx, &S->twin, twin)) || (st = iupload(ctx, &S->color_cells, ccells)) ||
            (st = iupload(ctx, &S->color_off_d, coff)) ||
            (st = iupload(ctx, &S->lev_f_off, lfo)) || (st = iupload(ctx, &S->fw_cell, lfc)) ||
            (st = iupload(ctx, &S->fw_nb, fwn)) || (st = iupload(ctx, &S->fw_h, fwh)) ||
            (st = iupload(ctx, &S->lev_b_off, lbo)) || (st = iupload(ctx, &S->bw_cell, lbc)) ||
            (st = iupload(ctx, &S->bw_nb, bwn)) || (st = iupload(ctx, &S->bw_h, bwh)))
            return st;
    }
    CK(cudaMemsetAsync(S->sc, 0, sizeof(double) * (SC_H + (K + 1) * (K + 1) + 4 * (K + 1) + 8), ctx->stream));
    CK(cudaMemsetAsync(S->flag, 0, sizeof(int) * 8, ctx->stream));
    CK(cudaMemsetAsync(S->ctl, 0, sizeof(int) * CTL_WORDS, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    S->ready = true;
    return CCFD_OK;
}

// ---------------------------------------------------------------- driver
// A set of implicit members stepped in lockstep on one stream: their device
// descriptors, and per kernel variant the residual-evaluation launch records
// (matrix-vector products at t + dt, Newton residuals at t + dt, Jacobian
// columns at t) over the concatenated tiles of the members.
struct ImpGroup {
    int flux, order, ns, fp32;
    int jac32 = 0;       // Jacobian columns (and their base) with FP32 fluxes (mixed-precision members)
    int n_tiles = 0, smem = 0, smem_jac = 0;
    StageLaunch *rec_mv = nullptr, *rec_nt = nullptr, *rec_jac = nullptr, *rec_jb = nullptr;
    int2* tmap = nullptr;
    int* ctr = nullptr;  // tile claim counters of the group's launches
};

struct ImpSet {
    std::vector<ccfd_ctx*> members;
    ImpDev* dev = nullptr;
    std::vector<ImpGroup> groups;
    int n = 0, max_nb = 0, max_col = 0, max_colsize = 0, max_K = 0, max_newton = 0;
    int max_level = 0;  // widest LU-SGS level (cells) over the members
    bool any_precond = false;
    bool pc64 = false, pc32 = false;  // preconditioned members in FP64 / FP32
    int* d_count = nullptr;
    int* h_count = nullptr;
    int h_count_v = 0;  // ordinary memory: freeing pinned memory would wait for the device
    cudaStream_t stream = nullptr;
    int last_cuda_error = 0;
};

static void set_free(ImpSet* M) {
    if (!M) return;
    for (auto& g : M->groups) {
        cudaFreeAsync(g.rec_mv, M->stream);
        cudaFreeAsync(g.rec_nt, M->stream);
        cudaFreeAsync(g.rec_jac, M->stream);
        cudaFreeAsync(g.rec_jb, M->stream);
        cudaFreeAsync(g.tmap, M->stream);
        cudaFreeAsync(g.ctr, M->stream);
    }
    if (M->dev) cudaFreeAsync(M->dev, M->stream);
    if (M->d_count) cudaFreeAsync(M->d_count, M->stream);
    delete M;
}

#define CKM(x)                              \
    do {                                    \
        cudaError_t e_ = (x);               \
        if (e_ != cudaSuccess) {            \
            M->last_cuda_error = (int)e_;   \
            return CCFD_ERR_CUDA;           \
        }                                   \
    } while (0)

static ImpDev make_dev(ccfd_ctx* ctx) {
    ImpState* S = (ImpState*)ctx->implicit_state;
    ImpDev d;
    memset(&d, 0, sizeof(d));
    d.N = S->N;
    d.K = S->K;
    d.nb = S->nb;
    d.precond = ctx->params.precond;
    d.n_newton = ctx->params.n_newton_iter;
    d.gam1 = ctx->phys.gam1;
    d.eps_gmres = ctx->params.eps_gmres;
    d.eps2newton = ctx->params.eps_newton * ctx->params.eps_newton;
    d.XK = S->XK; d.Q = S->Q; d.RXK = S->RXK; d.F = S->F; d.dX = S->dX; d.W = S->W;
    d.V = S->V; d.Z = S->Z; d.ptmp = S->ptmp; d.ut = S->ut; d.dxs = S->dxs;
    d.cons = ctx->cons0;
    d.prim = ctx->prim_buf[ctx->cur];
    d.pert = ctx->prim_buf[ctx->cur ^ 1];
    d.D = S->D; d.Dinv = S->Dinv; d.O = S->O; d.sc = S->sc; d.partial = S->partial;
    d.fp32 = S->fp32;
    d.Vf = S->Vf; d.Zf = S->Zf; d.dxsf = S->dxsf; d.Dinvf = S->Dinvf; d.Of = S->Of;
    d.rjb = S->RJB;
    d.flag = S->flag;
    d.ctl = S->ctl;
    d.ctrl = ctx->ctrl;
    d.hs_off = ctx->mesh.hs_off;
    d.hs_nb = ctx->mesh.hs_nb;
    d.twin = S->twin;
    d.ncol = ctx->params.precond ? (int)S->color_off.size() - 1 : 0;
    d.color_off = S->color_off_d;
    d.color_cells = S->color_cells;
    d.n_lev_f = S->n_lev_f; d.n_lev_b = S->n_lev_b;
    d.lev_f_off = S->lev_f_off; d.fw_cell = S->fw_cell; d.fw_nb = S->fw_nb; d.fw_h = S->fw_h;
    d.lev_b_off = S->lev_b_off; d.bw_cell = S->bw_cell; d.bw_nb = S->bw_nb; d.bw_h = S->bw_h;
    return d;
}

static int set_build(const std::vector<ccfd_ctx*>& members, cudaStream_t stream, ImpSet** out) {
    ImpSet* M = new ImpSet();
    *out = M;
    M->members = members;
    M->n = (int)members.size();
    M->stream = stream;
    std::vector<ImpDev> hd;
    std::map<std::tuple<int, int, int, int, int>, std::vector<int>> by_variant;
    for (int k = 0; k < M->n; ++k) {
        ccfd_ctx* ctx = members[k];
        ImpState* S = (ImpState*)ctx->implicit_state;
        hd.push_back(make_dev(ctx));
        M->max_nb = std::max(M->max_nb, S->nb);
        M->max_K = std::max(M->max_K, S->K);
        M->max_newton = std::max(M->max_newton, ctx->params.n_newton_iter);
        if (ctx->params.precond) {
            M->any_precond = true;
            if (S->fp32) M->pc32 = true;
            else M->pc64 = true;
            int ncol = (int)S->color_off.size() - 1;
            M->max_col = std::max(M->max_col, ncol);
            for (int c = 0; c < ncol; ++c)
                M->max_colsize = std::max(M->max_colsize, S->color_off[c + 1] - S->color_off[c]);
            M->max_level = std::max(M->max_level, S->max_level);
        }
        StageLaunch probe;
        ccfd_fill_stage(ctx, probe);
        by_variant[std::make_tuple(probe.flux_id, probe.order, probe.ns, probe.fp32, (int)S->fp32)].push_back(k);
    }
    CKM(ccfd_malloc_async((void**)&M->dev, sizeof(ImpDev) * M->n, stream));
    CKM(cudaMemcpyAsync(M->dev, hd.data(), sizeof(ImpDev) * M->n, cudaMemcpyHostToDevice, stream));
    CKM(ccfd_malloc_async((void**)&M->d_count, sizeof(int), stream));
    M->h_count = &M->h_count_v;
    for (auto& kv : by_variant) {
        ImpGroup g;
        std::tie(g.flux, g.order, g.ns, g.fp32, g.jac32) = kv.first;
        const std::vector<int>& idx = kv.second;
        std::vector<StageLaunch> mv(idx.size()), nt(idx.size()), jac(idx.size()), jb(idx.size());
        std::vector<int2> tmap;
        TileDev big;
        memset(&big, 0, sizeof(big));
        for (size_t j = 0; j < idx.size(); ++j) {
            ccfd_ctx* ctx = members[idx[j]];
            ImpState* S = (ImpState*)ctx->implicit_state;
            StageLaunch L;
            ccfd_fill_stage(ctx, L);
            L.ctrl = ctx->ctrl;
            L.mode = 0;
            L.res_partial = ctx->res_partial;
            // matrix-vector product: R(XK + eps Z_m) at t + dt
            L.a_time = 1.0;
            L.prim_in = S->ptmp;
            L.u_t = S->ut;
            L.skip = S->ctl + CTL_SKIP_GMRES;
            mv[j] = L;
            // Newton residual R(XK) at t + dt
            L.prim_in = ctx->prim_buf[ctx->cur];
            L.u_t = S->RXK;
            L.skip = S->ctl + CTL_SKIP_NEWTON;
            nt[j] = L;
            // Jacobian columns at t
            L.a_time = 0.0;
            L.prim_in = ctx->prim_buf[ctx->cur ^ 1];
            L.u_t = S->ut;
            L.skip = S->ctl + CTL_SKIP_JAC;
            L.fp32 = g.jac32;
            jac[j] = L;
            // their base in mixed precision: R(U, t) with FP32 fluxes
            L.u_t = S->RJB;
            jb[j] = L;
            for (int t = 0; t < ctx->tiles.n_tiles; ++t) tmap.push_back(make_int2((int)j, t));
            big.max_e = std::max(big.max_e, ctx->tiles.max_e);
            big.max_g = std::max(big.max_g, ctx->tiles.max_g);
            big.max_hs = std::max(big.max_hs, ctx->tiles.max_hs);
            big.max_f = std::max(big.max_f, ctx->tiles.max_f);
        }
        g.n_tiles = (int)tmap.size();
        g.smem = stage_smem_bytes(big, g.fp32);
        g.smem_jac = stage_smem_bytes(big, g.jac32);
        size_t rb = sizeof(StageLaunch) * idx.size();
        CKM(ccfd_malloc_async((void**)&g.rec_mv, rb, stream));
        CKM(ccfd_malloc_async((void**)&g.rec_nt, rb, stream));
        CKM(ccfd_malloc_async((void**)&g.rec_jac, rb, stream));
        if (g.jac32) {
            CKM(ccfd_malloc_async((void**)&g.rec_jb, rb, stream));
            CKM(cudaMemcpyAsync(g.rec_jb, jb.data(), rb, cudaMemcpyHostToDevice, stream));
        }
        CKM(ccfd_malloc_async((void**)&g.tmap, sizeof(int2) * tmap.size(), stream));
        CKM(ccfd_malloc_async((void**)&g.ctr, sizeof(int) * 2, stream));
        CKM(cudaMemsetAsync(g.ctr, 0, sizeof(int) * 2, stream));
        CKM(cudaMemcpyAsync(g.rec_mv, mv.data(), rb, cudaMemcpyHostToDevice, stream));
        CKM(cudaMemcpyAsync(g.rec_nt, nt.data(), rb, cudaMemcpyHostToDevice, stream));
        CKM(cudaMemcpyAsync(g.rec_jac, jac.data(), rb, cudaMemcpyHostToDevice, stream));
        CKM(cudaMemcpyAsync(g.tmap, tmap.data(), sizeof(int2) * tmap.size(), cudaMemcpyHostToDevice, stream));
        M->groups.push_back(g);
    }
    CKM(cudaStreamSynchronize(stream));
    return CCFD_OK;
}

// residual evaluations of a set: matrix-vector products, Newton residuals,
// Jacobian columns, and the FP32-flux base of the columns of mixed-precision
// members (their groups only)
enum RecKind { REC_MV, REC_NT, REC_JAC, REC_JB };

static void residuals(ImpSet* M, RecKind kind) {
    for (auto& g : M->groups) {
        if (kind == REC_JB && !g.jac32) continue;
        const bool jac = kind == REC_JAC || kind == REC_JB;
        BatchLaunch B;
        B.recs = kind == REC_MV ? g.rec_mv : kind == REC_NT ? g.rec_nt : kind == REC_JAC ? g.rec_jac : g.rec_jb;
        B.tmap = g.tmap;
        B.ctr = g.ctr;
        B.n_tiles = g.n_tiles;
        B.smem_bytes = jac ? g.smem_jac : g.smem;
        B.rk_mode = 0;
        B.stage = 0;
        B.flux_id = g.flux;
        B.order = g.order;
        B.ns = g.ns;
        B.fp32 = jac ? g.jac32 : g.fp32;
        launch_stage_batch(B, M->stream);
    }
}

// buildMatrix + calcDinv (src/linearSolver.c:186-252, :136-179) of the
// members that build a preconditioner: a perturbed copy of the state, the
// base of the mixed-precision columns, every colour and variable, blocks
// and inverses
static void build_jacobian(ImpSet* M, cudaStream_t st) {
    const dim3 gv(M->max_nb, M->n), g1(1, M->n);
    kb_jac_copy<<<gv, kB, 0, st>>>(M->dev);
    if (M->pc32) {
        kb_jac_gate<<<g1, 32, 0, st>>>(M->dev, 0);
        residuals(M, REC_JB);
    }
    const dim3 gc((M->max_colsize + kB - 1) / kB, M->n);
    for (int c = 0; c < M->max_col; ++c) {
        kb_jac_gate<<<g1, 32, 0, st>>>(M->dev, c);
        for (int v = 0; v < 4; ++v) {
            kb_jac_perturb<<<gc, kB, 0, st>>>(M->dev, c, v, 1);
            residuals(M, REC_JAC);
            kb_jac_collect<<<gc, kB, 0, st>>>(M->dev, c, v);
            kb_jac_perturb<<<gc, kB, 0, st>>>(M->dev, c, v, 0);
        }
    }
    kb_jac_finish<<<gv, kB, 0, st>>>(M->dev);
}

static int count_on(ImpSet* M, int what, int* out) {
    kb_count<<<1, 256, 0, M->stream>>>(M->dev, M->n, what, M->d_count);
    CKM(cudaMemcpyAsync(M->h_count, M->d_count, sizeof(int), cudaMemcpyDeviceToHost, M->stream));
    CKM(cudaStreamSynchronize(M->stream));
    *out = *M->h_count;
    return CCFD_OK;
}

// One implicitTimeStep (src/timeDiscretization.c:412-552) of every member
// whose control block lets it step, in lockstep.
static int set_step(ImpSet* M) {
    cudaStream_t st = M->stream;
    const dim3 gv(M->max_nb, M->n), g1(1, M->n);
    kb_step_prepare<<<g1, 32, 0, st>>>(M->dev);
    kb_step_begin<<<gv, kB, 0, st>>>(M->dev);
    residuals(M, REC_NT);
    kb_newton_F<<<gv, kB, 0, st>>>(M->dev, 1);
    kb_final<<<g1, kB, 0, st>>>(M->dev, FT_NORM_X0, 0, 0, 0, 0);
    kb_newton_start<<<g1, 32, 0, st>>>(M->dev);
    CKM(cudaGetLastError());
    for (int it = 0; it < M->max_newton; ++it) {
        int on = 0, s;
        if ((s = count_on(M, 0, &on))) return s;
        if (!on) break;
        // GMRES_M (src/linearSolver.c:385-510)
        kb_gmres_init<<<gv, kB, 0, st>>>(M->dev);
        kb_gmres_flags<<<g1, 32, 0, st>>>(M->dev);
        if (M->any_precond) {
            build_jacobian(M, st);
            kb_jac_check<<<g1, 32, 0, st>>>(M->dev);
        }
        for (int m = 0; m < M->max_K; ++m) {
            if (M->pc64) kb_lusgs<kSweepThreads, double><<<M->n, kSweepThreads, 0, st>>>(M->dev, m);
            if (M->pc32) kb_lusgs<kSweepThreads, float><<<M->n, kSweepThreads, 0, st>>>(M->dev, m);
            kb_copy_vz<<<gv, kB, 0, st>>>(M->dev, m);
            // matrixVector: epsFD = sqrt(eps) / |Z|
            kb_dot_zz<<<gv, kB, 0, st>>>(M->dev, m);
            kb_final<<<g1, kB, 0, st>>>(M->dev, FT_EPSFD, 0, 0, 2, 1);
            kb_mv_prep<<<gv, kB, 0, st>>>(M->dev, m);
            residuals(M, REC_MV);
            kb_mv_finish<<<gv, kB, 0, st>>>(M->dev, m);
            // modified Gram-Schmidt
            for (int nn = 0; nn <= m; ++nn) {
                kb_final<<<g1, kB, 0, st>>>(M->dev, FT_H, nn, m, 0, 1);
                kb_mgs<<<gv, kB, 0, st>>>(M->dev, nn, m);
            }
            kb_final<<<g1, kB, 0, st>>>(M->dev, FT_H, m + 1, m, 1, 1);
            kb_givens<<<g1, 32, 0, st>>>(M->dev, m);
            kb_vnext<<<gv, kB, 0, st>>>(M->dev, m);
            CKM(cudaGetLastError());
            if ((s = count_on(M, 1, &on))) return s;
            if (!on) break;
        }
        kb_gmres_end<<<g1, 32, 0, st>>>(M->dev);
        kb_newton_update<<<gv, kB, 0, st>>>(M->dev);
        residuals(M, REC_NT);
        kb_newton_F<<<gv, kB, 0, st>>>(M->dev, 0);
        kb_final<<<g1, kB, 0, st>>>(M->dev, FT_NORM_XK, 0, 0, 0, 0);
        kb_newton_check<<<g1, 32, 0, st>>>(M->dev);
        CKM(cudaGetLastError());
    }
    // global residual of the final residual evaluation, stop tests and the
    // next dt (calcTimeStep of the new state) of the members that stepped
    for (ccfd_ctx* ctx : M->members)
        imp_step_end_launch(ctx->ctrl, ctx->mesh, ctx->phys, ctx->sp, ctx->res_partial, ctx->tiles.n_tiles,
                            ctx->dt_partial, ctx->dt_bad, ctx->nb_cells, ctx->wall_ghost, ctx->wall_nl,
                            ctx->ghost_pface, ctx->prim_buf[ctx->cur], st);
    CKM(cudaGetLastError());
    return CCFD_OK;
}

// iteration counters of the members into their contexts (reports)
static int set_pull_counts(ImpSet* M) {
    for (ccfd_ctx* ctx : M->members) {
        ImpState* S = (ImpState*)ctx->implicit_state;
        int ctl[CTL_WORDS];
        CKM(cudaMemcpyAsync(ctl, S->ctl, sizeof(ctl), cudaMemcpyDeviceToHost, M->stream));
        CKM(cudaStreamSynchronize(M->stream));
        ctx->newton_total = ctl[CTL_NEWTON_TOTAL];
        ctx->gmres_total = ctl[CTL_GMRES_TOTAL];
    }
    return CCFD_OK;
}

static int run_implicit(ccfd_ctx* ctx, long nsteps, ccfd_report* report) {
    CK(cudaSetDevice(ctx->device));
    ImpState* S = (ImpState*)ctx->implicit_state;
    if (!S || !S->ready) return CCFD_ERR_ARG;
    cudaStream_t st = ctx->stream;
    int s;
    if (!S->solo) {
        ImpSet* M = nullptr;
        s = set_build({ctx}, st, &M);
        S->solo = M;
        if (s) return s;
    }
    ImpSet* M = (ImpSet*)S->solo;
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    Ctrl& c = *ctx->h_ctrl;
    const long long big = (1LL << 62);
    long long stop_at = nsteps > 0 ? c.iter + nsteps : big;
    c.stop_at = stop_at;
    CK(cudaMemcpyAsync(&ctx->ctrl->stop_at, &c.stop_at, sizeof(long long), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(ctx->ev_run0, st));
    launch_dt(ctx->mesh, ctx->phys, ctx->ctrl, ctx->sp, ctx->prim_buf[ctx->cur], ctx->dt_partial, ctx->dt_bad, st);
    launch_step_begin(ctx->ctrl, ctx->sp, ctx->dt_partial, ctx->dt_bad, ctx->nb_cells, st);
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int status = CCFD_OK;
    int ctl_status = 0;
    while (!c.done && c.active && c.iter < stop_at) {
        if ((status = set_step(M))) break;
        CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&ctl_status, S->ctl + CTL_STATUS, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (ctx->sp.hist && (s = ccfd_history_drain(ctx))) return s;
        if (ctl_status) {
            status = ctl_status;
            break;
        }
    }
    CK(cudaEventRecord(ctx->ev_run1, st));
    CK(cudaEventSynchronize(ctx->ev_run1));
    float run_ms = 0.0f;
    CK(cudaEventElapsedTime(&run_ms, ctx->ev_run0, ctx->ev_run1));
    if ((s = set_pull_counts(M))) return s;
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (report) {
        ccfd_fill_report(ctx, report);
        report->status = status ? status : report->status;
        report->device_ms = run_ms;
    }
    if (status) {
        // a failed step leaves the context usable: clear the stop flags the
        // device raised for it, as the single-case driver always did
        c.done = 0;
        c.active = 0;
        c.flags = 0;
        CK(cudaMemcpyAsync(ctx->ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        return status;
    }
    if (c.flags & FLAG_DT) return CCFD_ERR_DT;
    if (c.flags & FLAG_STATE) return CCFD_ERR_STATE;
    return CCFD_OK;
}

extern "C" int ccfd_run_implicit(ccfd_ctx* ctx, long nsteps, ccfd_report* report) {
    if (!ctx || !ctx->uploaded) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    return run_implicit(ctx, nsteps, report);
}

// the member set of a context alone (built on first use)
static int solo_set(ccfd_ctx* ctx, ImpSet** out) {
    ImpState* S = (ImpState*)ctx->implicit_state;
    if (!S || !S->ready) return CCFD_ERR_ARG;
    if (!S->solo) {
        ImpSet* M = nullptr;
        int s = set_build({ctx}, ctx->stream, &M);
        S->solo = M;
        if (s) return s;
    }
    *out = (ImpSet*)S->solo;
    return CCFD_OK;
}

// buildMatrix + calcDinv (src/linearSolver.c:136-252) at the context's state
// as at the first Newton iteration of an implicit step from t with time step
// dt, the blocks copied out in the reference's cell and half-side order.
extern "C" int ccfd_build_matrix(ccfd_ctx* ctx, double t, double dt, double* d_out, double* dinv_out,
                                 double* off_out) {
    if (!ctx || !ctx->uploaded || !ctx->params.implicit || !ctx->params.precond) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    CK(cudaSetDevice(ctx->device));
    ImpSet* M = nullptr;
    int s = solo_set(ctx, &M);
    if (s) return s;
    ImpState* S = (ImpState*)ctx->implicit_state;
    cudaStream_t st = ctx->stream;
    const long N = S->N, H = S->hs_off_h[N];
    // the step's control block (t, dt) and member words (Newton on, no GMRES
    // cycle), restored afterwards
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const Ctrl saved = *ctx->h_ctrl;
    Ctrl c = saved;
    c.t = t;
    c.dt = dt;
    c.active = 1;
    c.done = 0;
    int ctl[CTL_WORDS] = {0};
    ctl[CTL_NEWTON] = 1;
    ctl[CTL_SKIP_GMRES] = 1;
    CK(cudaMemcpyAsync(ctx->ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S->ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(S->flag, 0, sizeof(int) * 8, st));
    // boundary sides have no block: zero, as the reference's untouched
    // dense entries
    if (S->fp32) CK(cudaMemsetAsync(S->Of, 0, sizeof(float) * 16 * (size_t)H, st));
    else CK(cudaMemsetAsync(S->O, 0, sizeof(double) * 16 * (size_t)H, st));
    const dim3 gv(M->max_nb, M->n), g1(1, M->n);
    residuals(M, REC_NT);  // R_XK = R(U, t + dt)
    build_jacobian(M, st);
    CK(cudaGetLastError());
    std::vector<double> D(16 * N), Di(16 * N), O(16 * H);
    int flag[8];
    CK(cudaMemcpyAsync(D.data(), S->D, sizeof(double) * D.size(), cudaMemcpyDeviceToHost, st));
    if (S->fp32) {
        std::vector<float> a(16 * N), b(16 * H);
        CK(cudaMemcpyAsync(a.data(), S->Dinvf, sizeof(float) * a.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(b.data(), S->Of, sizeof(float) * b.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (size_t k = 0; k < a.size(); ++k) Di[k] = a[k];
        for (size_t k = 0; k < b.size(); ++k) O[k] = b[k];
    } else {
        CK(cudaMemcpyAsync(Di.data(), S->Dinv, sizeof(double) * Di.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(O.data(), S->O, sizeof(double) * O.size(), cudaMemcpyDeviceToHost, st));
    }
    CK(cudaMemcpyAsync(flag, S->flag, sizeof(flag), cudaMemcpyDeviceToHost, st));
    int zero[CTL_WORDS] = {0};
    CK(cudaMemcpyAsync(ctx->ctrl, &saved, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S->ctl, zero, sizeof(zero), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    *ctx->h_ctrl = saved;
    S->jac_built = true;
    // device order -> reference order (cells keep their side order)
    long ho = 0;
    for (long cr = 0; cr < N; ++cr) {
        const int d = ctx->dev_of_cell[cr];
        const int h0 = S->hs_off_h[d], nh = S->hs_off_h[d + 1] - h0;
        if (d_out) memcpy(d_out + 16 * cr, &D[16 * (size_t)d], sizeof(double) * 16);
        if (dinv_out) memcpy(dinv_out + 16 * cr, &Di[16 * (size_t)d], sizeof(double) * 16);
        if (off_out) memcpy(off_out + 16 * ho, &O[16 * (size_t)h0], sizeof(double) * 16 * nh);
        ho += nh;
    }
    return flag[2] ? CCFD_ERR_SINGULAR : CCFD_OK;
}

// LUSGS (src/linearSolver.c:261-333) of b with the blocks of the last
// ccfd_build_matrix, in the reference's cell order.
extern "C" int ccfd_lusgs(ccfd_ctx* ctx, const double* b, double* x) {
    if (!ctx || !b || !x || !ctx->uploaded) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    ImpState* S = (ImpState*)ctx->implicit_state;
    if (!S || !S->jac_built) return CCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    ImpSet* M = nullptr;
    int s = solo_set(ctx, &M);
    if (s) return s;
    cudaStream_t st = ctx->stream;
    const long N = S->N;
    std::vector<double> h(4 * N);
    for (long d = 0; d < N; ++d) memcpy(&h[4 * d], b + 4 * (size_t)ctx->cell_of_dev[d], sizeof(double) * 4);
    std::vector<float> hf;
    if (S->fp32) {
        hf.assign(h.begin(), h.end());
        CK(cudaMemcpyAsync(S->Vf, hf.data(), sizeof(float) * hf.size(), cudaMemcpyHostToDevice, st));
    } else {
        CK(cudaMemcpyAsync(S->V, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, st));
    }
    int ctl[CTL_WORDS] = {0};  // GMRES "on": the sweep runs
    CK(cudaMemcpyAsync(S->ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, st));
    if (S->fp32) {
        kb_lusgs<kSweepThreads, float><<<M->n, kSweepThreads, 0, st>>>(M->dev, 0);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hf.data(), S->Zf, sizeof(float) * hf.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (size_t k = 0; k < hf.size(); ++k) h[k] = hf[k];
    } else {
        kb_lusgs<kSweepThreads, double><<<M->n, kSweepThreads, 0, st>>>(M->dev, 0);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h.data(), S->Z, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    for (long d = 0; d < N; ++d) memcpy(x + 4 * (size_t)ctx->cell_of_dev[d], &h[4 * d], sizeof(double) * 4);
    return CCFD_OK;
}

// ---------------------------------------------------------------- batching
// The implicit members of a batch form one lockstep set on the batch stream
// (rebuilt when the membership changes).
// The implicit members of a batch are split into a few lockstep sets, each
// driven by its own host thread on its own stream: the latency-bound work of
// one set (LU-SGS sweeps, reductions) overlaps on the device with the
// throughput-bound residual evaluations of the others.  Rebuilt when the
// membership changes.
struct BatchImp {
    std::vector<ImpSet*> sets;
    std::vector<cudaStream_t> streams;
    std::vector<ccfd_ctx*> key;
};
static std::map<const ccfd_batch*, BatchImp> g_batch_imp;

static void batch_imp_free(BatchImp& bi) {
    for (ImpSet* M : bi.sets) set_free(M);
    for (cudaStream_t st : bi.streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    bi.sets.clear();
    bi.streams.clear();
    bi.key.clear();
}

cudaStream_t ccfd_batch_stream(ccfd_batch* b);

int ccfd_implicit_batch_join(ccfd_batch* b, ccfd_ctx* ctx) {
    ImpState* S = (ImpState*)ctx->implicit_state;
    if (!S || !S->ready) return CCFD_ERR_ARG;
    cudaStream_t st = ccfd_batch_stream(b);
    launch_dt(ctx->mesh, ctx->phys, ctx->ctrl, ctx->sp, ctx->prim_buf[ctx->cur], ctx->dt_partial, ctx->dt_bad, st);
    launch_step_begin(ctx->ctrl, ctx->sp, ctx->dt_partial, ctx->dt_bad, ctx->nb_cells, st);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    return CCFD_OK;
}

int ccfd_implicit_batch_leave(ccfd_batch* b, ccfd_ctx* ctx) {
    auto it = g_batch_imp.find(b);
    if (it != g_batch_imp.end()) {
        for (ImpSet* M : it->second.sets) set_pull_counts(M);
        batch_imp_free(it->second);
        g_batch_imp.erase(it);
    }
    (void)ctx;
    return CCFD_OK;
}

void ccfd_implicit_batch_release(ccfd_batch* b) {
    auto it = g_batch_imp.find(b);
    if (it == g_batch_imp.end()) return;
    batch_imp_free(it->second);
    g_batch_imp.erase(it);
}

// up to `steps` implicit time steps of one lockstep set
static int set_steps(ImpSet* M, int device, int steps) {
    if (cudaSetDevice(device) != cudaSuccess) return CCFD_ERR_CUDA;
    for (int k = 0; k < steps; ++k) {
        // members that can still step
        int any = 0;
        for (ccfd_ctx* ctx : M->members)
            CKM(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, M->stream));
        CKM(cudaStreamSynchronize(M->stream));
        for (ccfd_ctx* ctx : M->members) any |= ctx->h_ctrl->active && !ctx->h_ctrl->done;
        if (!any) break;
        int s = set_step(M);
        if (s) return s;
    }
    return set_pull_counts(M);
}

int ccfd_implicit_batch_steps(ccfd_batch* b, const std::vector<ccfd_ctx*>& members, int steps) {
    BatchImp& bi = g_batch_imp[b];
    if (bi.key != members) {
        batch_imp_free(bi);
        bi.key = members;
        // sets balanced by cell count (largest first onto the lightest set);
        // at most CCFD_IMPLICIT_SETS (default 8) sets of at least 4 members
        // (256 airfoils: 2 / 4 / 8 / 16 sets 3.17 / 2.93 / 2.75 / 2.87 s;
        // 32 airfoils: 4 and 8 sets alike)
        int max_sets = 8;
        if (const char* e = getenv("CCFD_IMPLICIT_SETS")) max_sets = std::max(1, std::min(64, atoi(e)));
        const int nsets = std::max(1, std::min(max_sets, (int)members.size() / 4));
        std::vector<int> idx(members.size());
        for (size_t k = 0; k < idx.size(); ++k) idx[k] = (int)k;
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) { return members[a]->N > members[c]->N; });
        std::vector<std::vector<ccfd_ctx*>> parts(nsets);
        std::vector<long> load(nsets, 0);
        for (int k : idx) {
            int j = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            parts[j].push_back(members[k]);
            load[j] += members[k]->N;
        }
        for (int j = 0; j < nsets; ++j) {
            cudaStream_t st;
            if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return CCFD_ERR_CUDA;
            bi.streams.push_back(st);
            ImpSet* M = nullptr;
            int s = set_build(parts[j], st, &M);
            bi.sets.push_back(M);
            if (s) return s;
        }
    }
    int device = members[0]->device;
    std::vector<int> status(bi.sets.size(), CCFD_OK);
    std::vector<std::thread> threads;
    for (size_t j = 1; j < bi.sets.size(); ++j)
        threads.emplace_back([&, j] { status[j] = set_steps(bi.sets[j], device, steps); });
    status[0] = set_steps(bi.sets[0], device, steps);
    for (auto& t : threads) t.join();
    for (int s : status)
        if (s) return s;
    return CCFD_OK;
}
