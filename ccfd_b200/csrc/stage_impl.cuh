// Kernels of the residual-and-update path (templates shared by the
// per-flux translation units stage_fNN.cu and by stage.cu).
//
//   k_stage  per tile (one CTA), fused: stage the primitive states of the
//            tile, two neighbour rings and the adjacent ghost cells (ghost
//            states at the mirrored barycentres, setBCatBarys, src/boundary.c:
//            320-331) in shared memory; least-squares
//            gradients with Barth-Jespersen / Venkatakrishnan limiting for the
//            tile and ring 1 (spatialReconstruction, src/reconstruction.c:
//            198-314); limited linear reconstruction, convective and viscous
//            flux of every face of the tile, ghost states at boundary faces
//            (setBCatSides, src/boundary.c:300-314; fluxCalculation,
//            src/fluxCalculation.c:882-998); per-cell sum of the face fluxes
//            in the reference's side order, no atomics (src/finiteVolume.c:
//            96-120); Runge-Kutta stage update with consPrim
//            (src/timeDiscretization.c:362-398); at the last stage the local
//            time step of the new state and the global-residual partial sums;
//            the CTA that finishes last reduces the partials in a fixed order
//            and performs the end-of-step bookkeeping of timeDisc
//            (src/timeDiscretization.c:595-731), the wing coefficients of
//            calcCoef (src/analyze.c:292-387) and the next time step
//   k_dt / k_step_begin   calcTimeStep (src/timeDiscretization.c:249-329)
//            for the first step of a run
//
// Gradients and face fluxes live only in shared memory.  Floating-point
// operations keep the reference's operand order; the library is compiled
// with -fmad=false, so the FP64 results equal the reference's.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>

#include "kernels.cuh"

namespace ccfd {

// CTA shape per arithmetic type (one CTA per tile; measured): FP64 stages
// run 384 threads, 2 CTAs per SM (gradient cells and faces of a 256-cell
// tile in about one pass each); the FP32 kernels need half the shared
// memory and run 256 threads, 3 CTAs per SM.
// Dynamic shared memory limit of one kernel, raised as launches need more:
// per device, only ever raised, and safe when host threads (the lockstep
// implicit sets, several serving contexts) launch the same kernel at once.
struct SmemLimit {
    std::mutex mu;
    std::atomic<int> bytes[64];
    SmemLimit() {
        for (auto& b : bytes) b.store(0);
    }
    template <typename K>
    void ensure(K kern, int smem) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
        if (bytes[dev].load(std::memory_order_acquire) >= smem) return;
        std::lock_guard<std::mutex> lk(mu);
        if (bytes[dev].load(std::memory_order_relaxed) >= smem) return;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess)
            bytes[dev].store(smem, std::memory_order_release);
    }
};

// Launch bounds of the stage kernels (threads, CTAs per SM: they fix the
// registers, 80 in FP64) and the CTA size of a single-instance launch when
// the context sets none: in FP64 256 threads, three CTAs of a 256-cell tile
// per SM (0.147 against 0.151 ms per stage at 384 threads on the
// 500k-triangle double Mach reflection; 320 threads: 0.169); with FP32
// staging 128 threads on 192-cell tiles (the context's default tile size
// in that precision), six CTAs per SM.
template <typename FT> struct StageShape;
template <> struct StageShape<double> { static constexpr int threads = 384, min_blocks = 2, single = 256; };
template <> struct StageShape<float> { static constexpr int threads = 256, min_blocks = 3, single = 128; };

__device__ __forceinline__ double stage_time(const Ctrl* ctrl, double tfix, double a_time) {
    return ctrl ? ctrl->t + a_time * ctrl->dt : tfix;
}

__device__ __forceinline__ bool inactive(const Ctrl* ctrl) { return ctrl && !ctrl->active; }

__device__ __forceinline__ void ld4(const double4& v, double q[4]) {
    q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
}
__device__ __forceinline__ void ld4(const float4& v, float q[4]) {
    q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
}
__device__ __forceinline__ double4 mk4(const double q[4]) {
    return make_double4(q[0], q[1], q[2], q[3]);
}
__device__ __forceinline__ float4 mk4(const float q[4]) {
    return make_float4(q[0], q[1], q[2], q[3]);
}

// shared-memory vector types of the stage kernel: FP64 throughout, or FP32
// reconstruction and face fluxes (mixed precision; state, residual sums and
// the update stay FP64)
template <typename T> struct Vec;
template <> struct Vec<double> { using v4 = double4; using v2 = double2; };
template <> struct Vec<float> { using v4 = float4; using v2 = float2; };

template <typename T>
__device__ __forceinline__ typename Vec<T>::v4 cvt4(const double4& v) {
    if constexpr (sizeof(T) == 8) return v;
    else return make_float4(float(v.x), float(v.y), float(v.z), float(v.w));
}
template <typename T>
__device__ __forceinline__ typename Vec<T>::v2 cvt2(double a, double b) {
    if constexpr (sizeof(T) == 8) return make_double2(a, b);
    else return make_float2(float(a), float(b));
}
__device__ __forceinline__ double4 to_d4(const double4& v) { return v; }
__device__ __forceinline__ double4 to_d4(const float4& v) {
    return make_double4(v.x, v.y, v.z, v.w);
}

// Limited least-squares gradient of one cell (src/reconstruction.c:25-192,
// 252-312).  nbr(k, qn) fetches the k-th neighbour state in side order,
// gw(k) the side's (GP.x, GP.y, w.x, w.y), gp(k) the side's GP again for
// the limiter.  The limiter runs side by side (each side's offset is
// fetched once and only two of its values are live); the minimum over
// sides and variables does not depend on the order, so the result is the
// reference's.
template <typename T, class Nbr, class GW, class GP>
__device__ __forceinline__ void cell_gradient(int limiter, const T q[4], int nh, T eps2, Nbr nbr,
                                              GW gw, GP gp, T ux[4], T uy[4]) {
    T umin[4] = {q[0], q[1], q[2], q[3]}, umax[4] = {q[0], q[1], q[2], q[3]};
#pragma unroll
    for (int v = 0; v < 4; ++v) ux[v] = uy[v] = T(0.0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k < nh) {
            double4 g = gw(k);
            const T wx = T(g.z), wy = T(g.w);
            T qn[4];
            nbr(k, qn);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                T d = qn[v] - q[v];
                ux[v] += wx * d;
                uy[v] += wy * d;
                umin[v] = fmin(umin[v], qn[v]);
                umax[v] = fmax(umax[v], qn[v]);
            }
        }
    }
    T phi[4] = {T(1.0), T(1.0), T(1.0), T(1.0)};
    T mn[4], mx[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        mn[v] = umin[v] - q[v];
        mx[v] = umax[v] - q[v];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k < nh) {
            T gpx, gpy;
            gp(k, gpx, gpy);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                T uD = ux[v] * gpx + uy[v] * gpy;
                T pl = T(1.0);
                if (limiter == 1) {
                    if (uD > T(0.0)) pl = fmin(T(1.0), mx[v] / uD);
                    else if (uD < T(0.0)) pl = fmin(T(1.0), mn[v] / uD);
                } else {
                    T uD2 = uD * uD;
                    if (uD > T(0.0)) {
                        const T mx2 = mx[v] * mx[v];
                        pl = T(1.0) / uD * (((mx2 + eps2) * uD + T(2.0) * uD2 * mx[v]) /
                                            (mx2 + T(2.0) * uD2 + uD * mx[v] + eps2));
                    } else if (uD < T(0.0)) {
                        const T mn2 = mn[v] * mn[v];
                        pl = T(1.0) / uD * (((mn2 + eps2) * uD + T(2.0) * uD2 * mn[v]) /
                                            (mn2 + T(2.0) * uD2 + uD * mn[v] + eps2));
                    }
                }
                phi[v] = fmin(phi[v], pl);
            }
        }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        ux[v] *= phi[v];
        uy[v] *= phi[v];
    }
}

// Face flux from the two reconstructed states, rotated into the face frame
// and back, with the viscous contribution, scaled by the face length
// (src/fluxCalculation.c:885-996).  q0 / q1 are the cell-centre states and
// g0x..g1y the cell gradients (Navier-Stokes only).
template <int FLUX, int NS, typename T>
__device__ __forceinline__ void face_flux(const Phys& P, T nx, T ny, T len, const T L[4], const T R[4],
                                          const T q0[4], const T q1[4], const T g0x[4],
                                          const T g0y[4], const T g1x[4], const T g1y[4], double4 bbd,
                                          T F[4], unsigned* flags) {
    FluxIn<T> s;
    s.rL = L[0]; s.uL = nx * L[1] + ny * L[2]; s.vL = -ny * L[1] + nx * L[2]; s.pL = L[3];
    s.rR = R[0]; s.uR = nx * R[1] + ny * R[2]; s.vR = -ny * R[1] + nx * R[2]; s.pR = R[3];
    T fc[4];
    convective_flux<FLUX, T>(P, s, fc, flags);
    F[0] = fc[0];
    F[1] = nx * fc[1] - ny * fc[2];
    F[2] = ny * fc[1] + nx * fc[2];
    F[3] = fc[3];
    if (NS) {
        T st[4], gx[4], gy[4];
        const T bbz = T(bbd.z);
        T bx = T(bbd.x) / bbz, by = T(bbd.y) / bbz;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            st[v] = T(0.5) * (R[v] + L[v]);
            T gxm = T(0.5) * (g0x[v] + g1x[v]);
            T gym = T(0.5) * (g0y[v] + g1y[v]);
            T corr = gxm * bx + gym * by - (q1[v] - q0[v]) / bbz;
            gx[v] = gxm - corr * bx;
            gy[v] = gym - corr * by;
        }
        T fdx[4], fdy[4];
        diffusion_flux<T>(P, st, gx, gy, fdx, fdy);
#pragma unroll
        for (int v = 0; v < 4; ++v) F[v] -= (fdx[v] * nx + fdy[v] * ny);
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) F[v] *= len;
}

// ghost state at the mirrored barycentre of ghost g from interior state q
// (kept out of line: the boundary code is rare and heavy, the hot face code
// should not carry its registers)
static __device__ __noinline__ double4 ghost_bary(const int* __restrict__ gbc, const double4* __restrict__ ggn,
                                           const Phys* __restrict__ Pg, int g, double time, double4 qv,
                                           unsigned* flags) {
    const Phys& P = *Pg;
    double4 gn = ggn[g];
    double x[2] = {gn.x, gn.y};
    double q[4] = {qv.x, qv.y, qv.z, qv.w}, out[4];
    boundary_state(P, P.bc[gbc[g]], gn.z, gn.w, time, q, out, x, flags);
    return make_double4(out[0], out[1], out[2], out[3]);
}

// ghost state at a boundary face from the reconstructed interior face state
static __device__ __noinline__ double4 ghost_face(const int* __restrict__ gbc, const double4* __restrict__ ggn,
                                           const double4* __restrict__ gml, const Phys* __restrict__ Pg,
                                           int g, double time, double4 Lv, unsigned* flags) {
    const Phys& P = *Pg;
    double4 gn = ggn[g], ml = gml[g];
    double x[2] = {ml.x, ml.y};
    double Lq[4] = {Lv.x, Lv.y, Lv.z, Lv.w}, R[4];
    boundary_state(P, P.bc[gbc[g]], gn.z, gn.w, time, Lq, R, x, flags);
    return make_double4(R[0], R[1], R[2], R[3]);
}

template <int NV>
__device__ __forceinline__ void block_sum(double v[NV], double* out) {
    __shared__ double sh[NV][32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? sh[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) out[k] = x;
        }
    }
}

__device__ __forceinline__ void block_min2(double a, double b, int bad, double2* out, int* bad_out) {
    __shared__ double sa[32], sb[32];
    __shared__ int sbad[32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = fmin(a, __shfl_down_sync(0xffffffffu, a, o));
        b = fmin(b, __shfl_down_sync(0xffffffffu, b, o));
        bad |= __shfl_down_sync(0xffffffffu, bad, o);
    }
    if (lane == 0) { sa[warp] = a; sb[warp] = b; sbad[warp] = bad; }
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        a = lane < nw ? sa[lane] : 1e150;
        b = lane < nw ? sb[lane] : 1e150;
        bad = lane < nw ? sbad[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a = fmin(a, __shfl_down_sync(0xffffffffu, a, o));
            b = fmin(b, __shfl_down_sync(0xffffffffu, b, o));
            bad |= __shfl_down_sync(0xffffffffu, bad, o);
        }
        if (lane == 0) { *out = make_double2(a, b); *bad_out = bad; }
    }
}

// local convective / viscous time step of one cell (calcTimeStep,
// src/timeDiscretization.c:253-308) at CFL number cfl; returns false if not
// finite
__device__ __forceinline__ bool local_dt(const Phys& P, const StepParams& sp, double cfl, double dfl,
                                         const double q[4], double4 geo, double* dc, double* dv) {
    double a = sqrt(P.gam * q[3] / q[0]);
    *dv = 1e150;
    if (sp.ts1d) {
        *dc = cfl * geo.w / (fabs(q[1]) + a);
        return isfinite(*dc);
    }
    double ssr = (fabs(q[1]) + a) * geo.z + (fabs(q[2]) + a) * geo.w;
    *dc = cfl * geo.x / ssr;
    bool ok = isfinite(*dc);
    if (sp.visc) {
        double ssv = sp.gam_pr_max * P.mu * geo.z * geo.z + sp.gam_pr_max * P.mu * geo.w * geo.w;
        *dv = dfl * q[0] * q[0] * geo.x * geo.x / (4.0 * ssv);
        ok = ok && isfinite(*dv);
    }
    return ok;
}

// global dt from the partial minima with the output / end-time clamp
// (src/timeDiscretization.c:310-321)
__device__ __forceinline__ void finish_dt(Ctrl* ctrl, const StepParams& sp, double dtc, double dtv,
                                          int bad) {
    if (bad) {
        ctrl->flags |= FLAG_DT;
        ctrl->done = 1;
        ctrl->active = 0;
        return;
    }
    double dt = sp.ts1d ? dtc : fmin(dtc, dtv);
    ctrl->visc_dominates = (!sp.ts1d && dtv < dtc) ? 1.0 : 0.0;
    double t = ctrl->t, pT = ctrl->print_time, sT = ctrl->stop_time;
    if ((t + dt > pT) || (t + dt > sT)) dt = fmin(pT, sT) - t;
    else if ((t + 1.5 * dt > pT) || (t + 1.5 * dt > sT)) dt = 0.5 * (fmin(pT, sT) - t);
    ctrl->dt = dt;
}

// End of a step, executed by one whole block: global residual (fixed-order
// reduction of the per-tile partials), wing coefficients, t += dt, the stop
// tests of timeDisc (src/timeDiscretization.c:609-731), the CFL number of
// the next step under switched evolution relaxation and, with with_dt, the
// next dt from the partial minima (otherwise a later k_step_dt computes it
// at the new CFL number).
__device__ __forceinline__ void step_end_block(Ctrl* ctrl, const StepParams& sp, const double* res_partial,
                               int nres, const double2* dt_partial, const int* dt_bad, int ndt,
                               const int* wall_ghost, const double* wall_nl,
                               const double* ghost_pface, const double4* prim_new,
                               bool with_dt = true) {
    __shared__ double s_res[4];
    __shared__ double2 s_dt;
    __shared__ int s_bad;
    const int tid = threadIdx.x;
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    double a = 1e150, b = 1e150;
    int bad = 0;
    for (int i = tid; i < nres; i += blockDim.x)
#pragma unroll
        for (int v = 0; v < 4; ++v) r[v] += __ldcg(&res_partial[4 * i + v]);
    for (int i = tid; i < ndt; i += blockDim.x) {
        double2 d = __ldcg(&dt_partial[i]);
        a = fmin(a, d.x);
        b = fmin(b, d.y);
        bad |= __ldcg(&dt_bad[i]);
    }
    block_sum<4>(r, s_res);
    block_min2(a, b, bad, &s_dt, &s_bad);
    __syncthreads();
    if (tid != 0) return;
    double res[6];
#pragma unroll
    for (int v = 0; v < 4; ++v) res[v] = sqrt(s_res[v] * sp.total_area_q);
    res[4] = res[5] = 0.0;
    double dt = ctrl->dt;
    ctrl->t += dt;
    long long iter = ctrl->iter + 1;
    ctrl->iter = iter;
    if (sp.calc_wing) {
        double cl_old = ctrl->cl, cd_old = ctrl->cd;
        double cl = 0.0, cd = 0.0;
        for (int k = 0; k < sp.n_wall; ++k) {
            double p0 = __ldcg(&ghost_pface[wall_ghost[k]]);
            double wnx = wall_nl[3 * k], wny = wall_nl[3 * k + 1], wl = wall_nl[3 * k + 2];
            cl += wny * p0 * wl;
            cd += wnx * p0 * wl;
        }
        cl *= sp.q_inf_lq;
        cd *= sp.q_inf_lq;
        ctrl->cl = cl * sp.cos_a - cd * sp.sin_a;
        ctrl->cd = cd * sp.cos_a + cl * sp.sin_a;
        res[4] = fabs(cl_old - ctrl->cl) / dt;
        res[5] = fabs(cd_old - ctrl->cd) / dt;
    }
#pragma unroll
    for (int v = 0; v < 6; ++v) ctrl->res[v] = res[v];
    if (sp.hist) {
        // the row of this step; the state of other CTAs is read around L1
        double* row = sp.hist + (size_t)((iter - 1) % sp.hist_cap) * sp.hist_width;
        row[0] = (double)iter;
        row[1] = ctrl->t;
        row[2] = dt;
#pragma unroll
        for (int v = 0; v < 6; ++v) row[3 + v] = res[v];
        row[9] = ctrl->cl;
        row[10] = ctrl->cd;
        for (int k = 0; k < sp.n_rec; ++k) {
            const double2* q = reinterpret_cast<const double2*>(&prim_new[sp.rec_cell[k]]);
            double2 a = __ldcg(q), b = __ldcg(q + 1);
            row[kHistHead + 4 * k] = a.x;
            row[kHistHead + 4 * k + 1] = a.y;
            row[kHistHead + 4 * k + 2] = b.x;
            row[kHistHead + 4 * k + 3] = b.y;
        }
    }
    if (!ctrl->have_first) {
#pragma unroll
        for (int v = 0; v < 4; ++v) ctrl->res_first[v] = res[v];
        ctrl->have_first = 1;
    }
    // switched evolution relaxation (Mulder and van Leer, 1985): the CFL
    // number of the next step from the first and the latest residual
    if (sp.ser && res[sp.abort_variable] > 0.0) {
        ctrl->cfl = fmin(sp.ser_cfl_max, sp.cfl * ctrl->res_first[sp.abort_variable] / res[sp.abort_variable]);
        ctrl->dfl = sp.dfl * ctrl->cfl / sp.cfl;
    }
    bool nonfinite = false;
#pragma unroll
    for (int v = 0; v < 4; ++v) nonfinite |= !isfinite(res[v]);
    ctrl->active = 0;
    if (nonfinite) {
        ctrl->flags |= FLAG_STATE;
        ctrl->done = 1;
        return;
    }
    double t = ctrl->t;
    if (ctrl->stop_time - t <= 1e-15) {
        ctrl->finished = 1;
        ctrl->done = 1;
        return;
    }
    if (sp.stationary) {
        double ra = res[sp.abort_variable];
        bool conv = false;
        if (fabs(ra) <= sp.abort_residual) {
            if (sp.abort_on_cl) conv = fabs(res[4]) <= sp.cl_abort;
            else if (sp.abort_on_cd) conv = fabs(res[5]) <= sp.cd_abort;
            else conv = true;
        }
        if (sp.rel_abort > 0.0 && ra <= sp.rel_abort * ctrl->res_first[sp.abort_variable])
            conv = true;
        if (conv) {
            ctrl->converged = 1;
            ctrl->done = 1;
            return;
        }
    }
    if ((ctrl->print_time - t <= 1e-15) || (iter == ctrl->print_iter)) {
        if (ctrl->print_time - t <= 1e-15) ctrl->print_time += ctrl->io_time_interval;
        if (iter == ctrl->print_iter) ctrl->print_iter += ctrl->io_iter_interval;
    }
    if (iter >= ctrl->max_iter) {
        ctrl->max_iter_hit = 1;
        ctrl->done = 1;
        return;
    }
    if (iter >= ctrl->stop_at) return;
    ctrl->active = 1;
    if (with_dt) finish_dt(ctrl, sp, s_dt.x, s_dt.y, s_bad);
}

// fused residual evaluation (+ RK stage) of tile t by one CTA; FT is the
// arithmetic type of the reconstruction and the face fluxes
template <int FLUX, int ORDER, int NS, typename FT>
__device__ __forceinline__ void stage_body(const StageLaunch& L, const int t) {
    using V4 = typename Vec<FT>::v4;
    using V2 = typename Vec<FT>::v2;
    extern __shared__ double4 smem[];
    const DevMesh& m = L.mesh;
    const TileDev& T = L.tiles;
    const Phys& P = L.phys;
    const int tid = threadIdx.x;
    // CTA size: the precision's default shape, or a smaller one chosen for the
    // context (the launch bounds fix the registers; work is strided by it)
    const int nthr = blockDim.x;
    const int4 cnt = T.counts[t];
    const int nT = cnt.x, nG = cnt.y, nEc = cnt.z, nE = cnt.w;
    const int e0 = T.e_off[t];
    // the tile's own cells are consecutive device cells (staged entries
    // 0..nT-1): their indices need no lookup
    const int d_first = T.e_ref[e0];
    const double time = stage_time(L.ctrl, L.tfix, L.a_time);
    V4* ps = reinterpret_cast<V4*>(smem);             // [max_e] states
    V4* gs = ps + T.max_e;                            // [2 max_g] gradients
    V2* hgp = reinterpret_cast<V2*>(gs + 2 * T.max_g);  // [max_hs] GP
    V4* fs = reinterpret_cast<V4*>(hgp + T.max_hs + (T.max_hs & 1));  // [max_f]

    // source term of the tile's cells (calcSource), evaluated first, while
    // few registers are live, into a per-cell buffer that the same thread
    // reads back in D (same cell-to-thread mapping)
    if (m.cell_src)
        for (int i = tid; i < nT; i += nthr) {
            const int d = d_first + i;
            m.src_buf[d] = cell_source(P, m.hs_gw, m.hs_off[d], m.hs_off[d + 1], m.cell_src[d],
                                       m.cell_geo[d].x, time);
        }

    // A: stage the states of the tile and its rings; ghost cells get the
    // boundary state at their mirrored barycentre (second order only: the
    // reference sets ghost cell states in its second-order reconstruction
    // and leaves them zero otherwise)
    for (int e = tid; e < nEc; e += nthr)
        ps[e] = cvt4<FT>(L.prim_in[e < nT ? d_first + e : T.e_ref[e0 + e]]);
    for (int e = nEc + tid; e < nE; e += nthr) {
        int g = -1 - T.e_ref[e0 + e];
        double4 gq = make_double4(0.0, 0.0, 0.0, 0.0);
        if (ORDER == 2)
            gq = ghost_bary(L.ghosts.bc, L.ghosts.gn, L.phys_g, g, time, L.prim_in[L.ghosts.cell[g]],
                            L.flags);
        ps[e] = cvt4<FT>(gq);
    }
    __syncthreads();

    // B: limited gradients of the tile and ring-1 cells
    const int hb = T.hs_off[t], gb = T.gl_off[t];
    if (ORDER == 2) {
        for (int i = tid; i < nG; i += nthr) {
            int d = i < nT ? d_first + i : T.e_ref[e0 + i];
            int h0 = m.hs_off[d], nh = m.hs_off[d + 1] - h0;
            int lo = T.hs_loc[gb + i];
            FT q[4], ux[4], uy[4];
            ld4(ps[i], q);
            FT eps2 = L.limiter == 2 ? FT(m.venk_eps2[d]) : FT(0.0);
            auto nbr = [&](int k, FT qn[4]) { ld4(ps[T.hs_nbl[hb + lo + k]], qn); };
            auto gw = [&](int k) {
                double4 g = m.hs_gw[h0 + k];
                hgp[lo + k] = cvt2<FT>(g.x, g.y);
                return g;
            };
            auto gp = [&](int k, FT& x, FT& y) {
                const V2 g = hgp[lo + k];
                x = g.x;
                y = g.y;
            };
            cell_gradient<FT>(L.limiter, q, nh, eps2, nbr, gw, gp, ux, uy);
            gs[2 * i] = mk4(ux);
            gs[2 * i + 1] = mk4(uy);
        }
        __syncthreads();
    }

    // C: fluxes of the tile's faces (interior faces, then boundary faces)
    const int f0 = T.f_off[t], nF = T.f_off[t + 1] - f0;
    for (int j = tid; j < nF; j += nthr) {
        int fid = T.f_id[f0 + j];
        int lr = T.f_lr[f0 + j];
        int il = lr & 0xffff, ir = lr >> 16;
        FT q0[4], q1[4], Lf[4], Rf[4];
        FT g0x[4] = {0, 0, 0, 0}, g0y[4] = {0, 0, 0, 0}, g1x[4] = {0, 0, 0, 0}, g1y[4] = {0, 0, 0, 0};
        ld4(ps[il], q0);
        ld4(ps[ir], q1);
        int hh = T.f_hs[f0 + j];
        if (ORDER == 2) {
            V2 gpl = hgp[hh & 0xffff];
            ld4(gs[2 * il], g0x);
            ld4(gs[2 * il + 1], g0y);
#pragma unroll
            for (int v = 0; v < 4; ++v) Lf[v] = q0[v] + gpl.x * g0x[v] + gpl.y * g0y[v];
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v) Lf[v] = q0[v];
        }
        FT nx, ny, len;
        double4 bb = make_double4(0, 0, 1, 0);
        if (fid >= 0) {
            if (ORDER == 2) {
                V2 gpr = hgp[hh >> 16];
                ld4(gs[2 * ir], g1x);
                ld4(gs[2 * ir + 1], g1y);
#pragma unroll
                for (int v = 0; v < 4; ++v) Rf[v] = q1[v] + gpr.x * g1x[v] + gpr.y * g1y[v];
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) Rf[v] = q1[v];
            }
            double4 nl = m.face_nl[fid];
            nx = FT(nl.x); ny = FT(nl.y); len = FT(nl.z);
            if (NS) bb = m.face_bb[fid];
        } else {
            int g = -1 - fid;
            double4 Rd = ghost_face(L.ghosts.bc, L.ghosts.gn, L.ghosts.ml, L.phys_g, g, time,
                                    to_d4(mk4(Lf)), L.flags);
            ld4(cvt4<FT>(Rd), Rf);
            if (L.ghost_pface) L.ghost_pface[g] = double(Lf[3]);
            double4 gn = L.ghosts.gn[g];
            nx = FT(gn.z); ny = FT(gn.w); len = FT(L.ghosts.ml[g].z);
            if (NS) bb = L.ghosts.bb[g];
        }
        FT F[4];
        face_flux<FLUX, NS, FT>(P, nx, ny, len, Lf, Rf, q0, q1, g0x, g0y, g1x, g1y, bb, F, L.flags);
        fs[j] = mk4(F);
    }
    __syncthreads();

    // D: per-cell flux sum in side order, update
    double r[4] = {0, 0, 0, 0};
    double dconv = 1e150, dvisc = 1e150;
    int bad = 0;
    const bool rk = L.mode == 1;
    for (int i = tid; i < nT; i += nthr) {
        int d = d_first + i;
        int h0 = m.hs_off[d], h1 = m.hs_off[d + 1];
        double s[4] = {0.0, 0.0, 0.0, 0.0};
        for (int h = h0; h < h1; ++h) {
            int code = T.u_code[h];
            FT F[4];
            ld4(fs[code >> 1], F);
            if (code & 1) {
#pragma unroll
                for (int v = 0; v < 4; ++v) s[v] += -double(F[v]);
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) s[v] += double(F[v]);
            }
        }
        double4 geo = m.cell_geo[d];
        const double4 sv = m.cell_src ? m.src_buf[d] : make_double4(0.0, 0.0, 0.0, 0.0);
        const double src[4] = {sv.x, sv.y, sv.z, sv.w};
        double ut[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) ut[v] = (src[v] - s[v]) * geo.y;
        if (L.u_t) L.u_t[d] = mk4(ut);
        if (!rk && L.grad_out) {
            L.grad_out[2 * d] = ORDER == 2 ? to_d4(gs[2 * i]) : make_double4(0, 0, 0, 0);
            L.grad_out[2 * d + 1] = ORDER == 2 ? to_d4(gs[2 * i + 1]) : make_double4(0, 0, 0, 0);
        }
        if (rk) {
            double c0[4], cn[4], pn[4];
            ld4(L.cons0[d], c0);
            double adt = L.rk * L.ctrl->dt;
#pragma unroll
            for (int v = 0; v < 4; ++v) cn[v] = c0[v] + adt * ut[v];
            cons_prim(P.gam1, cn, pn);
            L.prim_out[d] = mk4(pn);
            if (L.last_stage) {
                L.cons0[d] = mk4(cn);
                double a, b;
                if (!local_dt(P, L.sp, L.sp.cfl, L.sp.dfl, pn, geo, &a, &b)) bad = 1;
                else {
                    dconv = fmin(dconv, a);
                    dvisc = fmin(dvisc, b);
                }
            }
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) r[v] += geo.x * ut[v] * ut[v];
    }
    if (L.res_partial) {
        double out[4];
        block_sum<4>(r, out);
        if (tid == 0)
#pragma unroll
            for (int v = 0; v < 4; ++v) L.res_partial[4 * t + v] = out[v];
    }
    if (L.dt_partial) block_min2(dconv, dvisc, bad, &L.dt_partial[t], &L.dt_bad[t]);
    if (rk && L.last_stage) {
        // the CTA that finishes last closes the step
        __shared__ int s_last;
        __threadfence();
        __syncthreads();
        if (tid == 0) s_last = atomicAdd(L.ticket, 1u) == (unsigned)(T.n_tiles - 1);
        __syncthreads();
        if (s_last) {
            __threadfence();
            Ctrl* ctrl = const_cast<Ctrl*>(L.ctrl);
            step_end_block(ctrl, L.sp, L.res_partial, T.n_tiles, L.dt_partial, L.dt_bad, T.n_tiles,
                           L.wall_ghost, L.wall_nl, L.ghost_pface, L.prim_out);
            if (tid == 0) {
                ctrl->par ^= (L.sp.nrk & 1);  // buffer holding the state after this step
                *L.ticket = 0u;
            }
        }
    }
}


// one instance: one tile per CTA, launch parameters in the parameter space
template <int FLUX, int ORDER, int NS, typename FT>
__global__ void __launch_bounds__(StageShape<FT>::threads, StageShape<FT>::min_blocks) k_stage(StageLaunch L) {
    if (inactive(L.ctrl)) return;
    stage_body<FLUX, ORDER, NS, FT>(L, blockIdx.x);
}

// Many instances in one persistent launch over their concatenated tiles:
// each CTA claims the next entry of the tile map from a counter (entry b is
// tile tmap[b].y of instance tmap[b].x) until none is left, so uneven
// instances share one grid sized to the device, and CTAs that cannot start
// at once (SMs held by other work of the device) leave their share to the
// running ones instead of holding the launch back.  ctr[0] is the next
// entry, ctr[1] the CTAs done; the last CTA to finish resets both for the
// next launch on the stream.  An RK stage takes the instance's launch
// record for the stage and the buffer parity in its control block
// (Ls[inst][par][stage]); a residual evaluation (stride 1) takes Ls[inst]
// and is skipped while *skip is nonzero.
template <int FLUX, int ORDER, int NS, typename FT>
__global__ void __launch_bounds__(StageShape<FT>::threads, StageShape<FT>::min_blocks)
    k_stage_batch(const StageLaunch* __restrict__ Ls, const int2* __restrict__ tmap, int n_tiles, int rk_mode,
                  int stage, int* __restrict__ ctr) {
    // The member's launch record goes to shared memory.  In RK mode the
    // records of both buffer parities are copied while one thread reads the
    // member's control block, so resolving the record costs one round trip
    // after the tile map instead of a chain of dependent loads.
    static_assert(sizeof(StageLaunch) % 16 == 0, "launch record copied in 16-byte words");
    constexpr int W = (int)(sizeof(StageLaunch) / 16);
    __shared__ int4 s_rec[2 * W];
    __shared__ int s_go, s_sel, s_b;
    for (;;) {
        __syncthreads();  // the previous entry's record is no longer read
        if (threadIdx.x == 0) s_b = atomicAdd(&ctr[0], 1);
        __syncthreads();
        const int b = s_b;
        if (b >= n_tiles) break;
        const int2 tm = tmap[b];
        if (rk_mode) {
            const StageLaunch* rec = Ls + (size_t)tm.x * 2 * kBatchStages;
            const int4* a = reinterpret_cast<const int4*>(rec + stage);
            const int4* c = reinterpret_cast<const int4*>(rec + kBatchStages + stage);
            for (int k = threadIdx.x; k < 2 * W; k += blockDim.x) s_rec[k] = k < W ? a[k] : c[k - W];
            if (threadIdx.x == 0) {
                const Ctrl* cb = rec[0].ctrl;
                s_go = cb->active;
                s_sel = cb->par;
            }
        } else {
            const int4* a = reinterpret_cast<const int4*>(Ls + tm.x);
            for (int k = threadIdx.x; k < W; k += blockDim.x) s_rec[k] = a[k];
            if (threadIdx.x == 0) {
                const int* skip = Ls[tm.x].skip;
                s_go = !(skip && *skip);
                s_sel = 0;
            }
        }
        __syncthreads();
        if (!s_go) continue;
        const StageLaunch& L = *reinterpret_cast<const StageLaunch*>(s_rec + s_sel * W);
        if (L.mode < 0) continue;
        stage_body<FLUX, ORDER, NS, FT>(L, tm.y);
    }
    if (threadIdx.x == 0 && atomicAdd(&ctr[1], 1) == (int)gridDim.x - 1) {
        atomicExch(&ctr[0], 0);
        atomicExch(&ctr[1], 0);
    }
}


// grid of a persistent launch: as many CTAs as the device holds at once
// (SMs x resident CTAs per SM), at most one per tile; the occupancy is
// looked up once per kernel, shared-memory size and device
template <typename K>
inline int persistent_grid(K kern, int threads, int smem, int n_tiles) {
    struct Key {
        const void* k;
        int smem, dev;
        bool operator<(const Key& o) const {
            return k != o.k ? k < o.k : smem != o.smem ? smem < o.smem : dev < o.dev;
        }
    };
    static std::mutex mu;
    static std::map<Key, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const Key key{reinterpret_cast<const void*>(kern), smem, dev};
    int slots;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it == cache.end()) {
            int sms = 1, per = 1;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem) != cudaSuccess || per < 1)
                per = 1;
            it = cache.emplace(key, sms * per).first;
        }
        slots = it->second;
    }
    return n_tiles < slots ? n_tiles : slots;
}

template <typename FT>
inline int stage_smem_bytes_t(const TileDev& T) {
    using V4 = typename Vec<FT>::v4;
    using V2 = typename Vec<FT>::v2;
    return (int)(sizeof(V4) * (T.max_e + 2 * T.max_g) + sizeof(V2) * (T.max_hs + (T.max_hs & 1)) +
                 sizeof(V4) * T.max_f);
}

// per-flux entry points (stage_fNN.cu)
#define CCFD_DECLARE_FLUX(ID)                                             \
    void launch_stage_f##ID(const StageLaunch& L, cudaStream_t st);       \
    void launch_stage_batch_f##ID(const BatchLaunch& B, cudaStream_t st);
CCFD_DECLARE_FLUX(1) CCFD_DECLARE_FLUX(2) CCFD_DECLARE_FLUX(3) CCFD_DECLARE_FLUX(4)
CCFD_DECLARE_FLUX(5) CCFD_DECLARE_FLUX(6) CCFD_DECLARE_FLUX(7) CCFD_DECLARE_FLUX(8)
CCFD_DECLARE_FLUX(9) CCFD_DECLARE_FLUX(10) CCFD_DECLARE_FLUX(11)
#undef CCFD_DECLARE_FLUX

}  // namespace ccfd
