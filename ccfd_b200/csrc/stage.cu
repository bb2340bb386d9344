// Kernels of the residual-and-update path.
//
//   k_bnd    per ghost (boundary face), small: ghost state at the mirrored
//            barycentre (setBCatBarys, src/boundary.c:320-331), limited
//            gradient of the interior cell, ghost state at the face
//            (setBCatSides, :300-314) and the boundary-face flux
//   k_stage  per tile (one CTA), fused: stage the primitive states of the
//            tile and two neighbour rings in shared memory; least-squares
//            gradients with Barth-Jespersen / Venkatakrishnan limiting for the
//            tile and ring 1 (spatialReconstruction, src/reconstruction.c:
//            198-314); limited linear reconstruction, convective and viscous
//            flux of every interior face of the tile (fluxCalculation,
//            src/fluxCalculation.c:882-998); per-cell sum of the face fluxes
//            in the reference's side order, no atomics (src/finiteVolume.c:
//            96-120); Runge-Kutta stage update with consPrim
//            (src/timeDiscretization.c:362-398); at the last stage the local
//            time step of the new state and the global-residual partial sums
//   k_dt / k_step_begin / k_step_end   calcTimeStep (src/timeDiscretization.c:
//            249-329), the per-step bookkeeping of timeDisc (:595-731) and the
//            wing coefficients of calcCoef (src/analyze.c:292-387)
//
// Gradients and face fluxes live only in shared memory.  Floating-point
// operations keep the reference's operand order; the library is compiled
// with -fmad=false, so the FP64 results equal the reference's.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace ccfd {

constexpr int kThreads = 256;

__device__ __forceinline__ double stage_time(const Ctrl* ctrl, double tfix, double a_time) {
    return ctrl ? ctrl->t + a_time * ctrl->dt : tfix;
}

__device__ __forceinline__ bool inactive(const Ctrl* ctrl) { return ctrl && !ctrl->active; }

__device__ __forceinline__ void ld4(const double4& v, double q[4]) {
    q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
}

__device__ __forceinline__ double4 mk4(const double q[4]) {
    return make_double4(q[0], q[1], q[2], q[3]);
}

// Limited least-squares gradient of one cell (src/reconstruction.c:25-192,
// 252-312).  nbr(k, qn) fetches the k-th neighbour state in side order,
// gw(k) the side's (GP.x, GP.y, w.x, w.y).
template <class Nbr, class GW>
__device__ __forceinline__ void cell_gradient(int limiter, const double q[4], int nh, double eps2,
                                              Nbr nbr, GW gw, double ux[4], double uy[4]) {
    double umin[4] = {q[0], q[1], q[2], q[3]}, umax[4] = {q[0], q[1], q[2], q[3]};
    double gpx[4] = {0, 0, 0, 0}, gpy[4] = {0, 0, 0, 0};
#pragma unroll
    for (int v = 0; v < 4; ++v) ux[v] = uy[v] = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k < nh) {
            double4 g = gw(k);
            gpx[k] = g.x;
            gpy[k] = g.y;
            double qn[4];
            nbr(k, qn);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                double d = qn[v] - q[v];
                ux[v] += g.z * d;
                uy[v] += g.w * d;
                umin[v] = fmin(umin[v], qn[v]);
                umax[v] = fmax(umax[v], qn[v]);
            }
        }
    }
    double phi[4] = {1.0, 1.0, 1.0, 1.0};
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        double mn = umin[v] - q[v], mx = umax[v] - q[v];
        double mn2 = mn * mn, mx2 = mx * mx;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < nh) {
                double uD = ux[v] * gpx[k] + uy[v] * gpy[k];
                double pl = 1.0;
                if (limiter == 1) {
                    if (uD > 0.0) pl = fmin(1.0, mx / uD);
                    else if (uD < 0.0) pl = fmin(1.0, mn / uD);
                } else {
                    double uD2 = uD * uD;
                    if (uD > 0.0)
                        pl = 1.0 / uD * (((mx2 + eps2) * uD + 2.0 * uD2 * mx) /
                                         (mx2 + 2.0 * uD2 + uD * mx + eps2));
                    else if (uD < 0.0)
                        pl = 1.0 / uD * (((mn2 + eps2) * uD + 2.0 * uD2 * mn) /
                                         (mn2 + 2.0 * uD2 + uD * mn + eps2));
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
template <int FLUX, int NS>
__device__ __forceinline__ void face_flux(const Phys& P, double nx, double ny, double len,
                                          const double L[4], const double R[4], const double q0[4],
                                          const double q1[4], const double g0x[4],
                                          const double g0y[4], const double g1x[4],
                                          const double g1y[4], double4 bb, double F[4],
                                          unsigned* flags) {
    FluxIn<double> s;
    s.rL = L[0]; s.uL = nx * L[1] + ny * L[2]; s.vL = -ny * L[1] + nx * L[2]; s.pL = L[3];
    s.rR = R[0]; s.uR = nx * R[1] + ny * R[2]; s.vR = -ny * R[1] + nx * R[2]; s.pR = R[3];
    double fc[4];
    convective_flux<FLUX, double>(P, s, fc, flags);
    F[0] = fc[0];
    F[1] = nx * fc[1] - ny * fc[2];
    F[2] = ny * fc[1] + nx * fc[2];
    F[3] = fc[3];
    if (NS) {
        double st[4], gx[4], gy[4];
        double bx = bb.x / bb.z, by = bb.y / bb.z;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            st[v] = 0.5 * (R[v] + L[v]);
            double gxm = 0.5 * (g0x[v] + g1x[v]);
            double gym = 0.5 * (g0y[v] + g1y[v]);
            double corr = gxm * bx + gym * by - (q1[v] - q0[v]) / bb.z;
            gx[v] = gxm - corr * bx;
            gy[v] = gym - corr * by;
        }
        double fdx[4], fdy[4];
        diffusion_flux(P, st, gx, gy, fdx, fdy);
#pragma unroll
        for (int v = 0; v < 4; ++v) F[v] -= (fdx[v] * nx + fdy[v] * ny);
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) F[v] *= len;
}

template <int NS>
__device__ void bnd_flux_dispatch(int flux, const Phys& P, double nx, double ny, double len,
                                  const double L[4], const double R[4], const double q0[4],
                                  const double q1[4], const double g0x[4], const double g0y[4],
                                  const double g1x[4], const double g1y[4], double4 bb,
                                  double F[4], unsigned* flags) {
#define CCFD_BF(ID) \
    case ID: face_flux<ID, NS>(P, nx, ny, len, L, R, q0, q1, g0x, g0y, g1x, g1y, bb, F, flags); break;
    switch (flux) {
        CCFD_BF(1) CCFD_BF(2) CCFD_BF(3) CCFD_BF(4) CCFD_BF(5) CCFD_BF(6)
        CCFD_BF(7) CCFD_BF(8) CCFD_BF(9) CCFD_BF(10) CCFD_BF(11)
    }
#undef CCFD_BF
}

// ghost state at the mirrored barycentre of ghost g from interior state q
__device__ __forceinline__ void ghost_bary(const GhostDev& G, const Phys& P, int g, double time,
                                           const double q[4], double out[4], unsigned* flags) {
    double4 gn = G.gn[g];
    double x[2] = {gn.x, gn.y};
    boundary_state(P, P.bc[G.bc[g]], gn.z, gn.w, time, q, out, x, flags);
}

// one thread per ghost / boundary face
template <int NS>
__global__ void __launch_bounds__(128) k_bnd(StageLaunch L) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    const DevMesh& m = L.mesh;
    if (g >= m.B || inactive(L.ctrl)) return;
    const Phys& P = L.phys;
    double time = stage_time(L.ctrl, L.tfix, L.a_time);
    int c = L.ghosts.cell[g];
    double q0[4];
    ld4(L.prim_in[c], q0);
    double gb[4];
    ghost_bary(L.ghosts, P, g, time, q0, gb, L.flags);
    L.ghost_prim[g] = mk4(gb);
    double ux[4] = {0, 0, 0, 0}, uy[4] = {0, 0, 0, 0};
    double Lf[4];
    if (L.order == 2) {
        int h0 = m.hs_off[c], nh = m.hs_off[c + 1] - h0;
        double eps2 = L.limiter == 2 ? m.venk_eps2[c] : 0.0;
        auto nbr = [&](int k, double qn[4]) {
            int nb = m.hs_nb[h0 + k];
            if (nb >= 0) ld4(L.prim_in[nb], qn);
            else ghost_bary(L.ghosts, P, -1 - nb, time, q0, qn, L.flags);
        };
        auto gw = [&](int k) { return m.hs_gw[h0 + k]; };
        cell_gradient(L.limiter, q0, nh, eps2, nbr, gw, ux, uy);
        double4 gp = m.hs_gw[L.ghosts.hs[g]];
#pragma unroll
        for (int v = 0; v < 4; ++v) Lf[v] = q0[v] + gp.x * ux[v] + gp.y * uy[v];
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) Lf[v] = q0[v];
        // the ghost cell state is only set by the second-order
        // reconstruction; it is zero otherwise (calloc'd ghost element)
        gb[0] = gb[1] = gb[2] = gb[3] = 0.0;
    }
    double4 gn = L.ghosts.gn[g], ml = L.ghosts.ml[g];
    double R[4];
    double xm[2] = {ml.x, ml.y};
    boundary_state(P, P.bc[L.ghosts.bc[g]], gn.z, gn.w, time, Lf, R, xm, L.flags);
    if (L.ghost_pface) L.ghost_pface[g] = Lf[3];
    double zero[4] = {0, 0, 0, 0}, F[4];
    double4 bb = NS ? L.ghosts.bb[g] : make_double4(0, 0, 1, 0);
    bnd_flux_dispatch<NS>(L.flux_id, P, gn.z, gn.w, ml.z, Lf, R, q0, gb, ux, uy, zero, zero, bb, F,
                          L.flags);
    L.bc_flux[g] = mk4(F);
}

template <int NV>
__device__ __forceinline__ void block_sum(double v[NV], double* out) {
    __shared__ double sh[NV][32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
// src/timeDiscretization.c:253-308); returns false if not finite
__device__ __forceinline__ bool local_dt(const Phys& P, const StepParams& sp, const double q[4],
                                         double4 geo, double* dc, double* dv) {
    double a = sqrt(P.gam * q[3] / q[0]);
    *dv = 1e150;
    if (sp.ts1d) {
        *dc = sp.cfl * geo.w / (fabs(q[1]) + a);
        return isfinite(*dc);
    }
    double ssr = (fabs(q[1]) + a) * geo.z + (fabs(q[2]) + a) * geo.w;
    *dc = sp.cfl * geo.x / ssr;
    bool ok = isfinite(*dc);
    if (sp.visc) {
        double ssv = sp.gam_pr_max * P.mu * geo.z * geo.z + sp.gam_pr_max * P.mu * geo.w * geo.w;
        *dv = sp.dfl * q[0] * q[0] * geo.x * geo.x / (4.0 * ssv);
        ok = ok && isfinite(*dv);
    }
    return ok;
}

// fused residual evaluation (+ RK stage) of one tile per CTA
template <int FLUX, int ORDER, int NS>
__global__ void __launch_bounds__(kThreads, 2) k_stage(StageLaunch L) {
    extern __shared__ double4 smem[];
    if (inactive(L.ctrl)) return;
    const DevMesh& m = L.mesh;
    const TileDev& T = L.tiles;
    const Phys& P = L.phys;
    const int t = blockIdx.x, tid = threadIdx.x;
    const int4 cnt = T.counts[t];
    const int nT = cnt.x, nG = cnt.y, nE = cnt.w;
    const int e0 = T.e_off[t];
    double4* ps = smem;                                   // [max_e] states
    double4* gs = ps + T.max_e;                           // [2 max_g] gradients
    double2* hgp = reinterpret_cast<double2*>(gs + 2 * T.max_g);  // [max_hs] GP
    double4* fs = reinterpret_cast<double4*>(hgp + T.max_hs + (T.max_hs & 1));  // [max_f]

    // A: stage the states of the tile, its rings and ghosts
    for (int e = tid; e < nE; e += kThreads) {
        int r = T.e_ref[e0 + e];
        ps[e] = r >= 0 ? L.prim_in[r] : L.ghost_prim[-1 - r];
    }
    __syncthreads();

    // B: limited gradients of the tile and ring-1 cells
    const int hb = T.hs_off[t], gb = T.gl_off[t];
    if (ORDER == 2) {
        for (int i = tid; i < nG; i += kThreads) {
            int d = T.e_ref[e0 + i];
            int h0 = m.hs_off[d], nh = m.hs_off[d + 1] - h0;
            int lo = T.hs_loc[gb + i];
            double q[4], ux[4], uy[4];
            ld4(ps[i], q);
            double eps2 = L.limiter == 2 ? m.venk_eps2[d] : 0.0;
            auto nbr = [&](int k, double qn[4]) { ld4(ps[T.hs_nbl[hb + lo + k]], qn); };
            auto gw = [&](int k) {
                double4 g = m.hs_gw[h0 + k];
                hgp[lo + k] = make_double2(g.x, g.y);
                return g;
            };
            cell_gradient(L.limiter, q, nh, eps2, nbr, gw, ux, uy);
            gs[2 * i] = mk4(ux);
            gs[2 * i + 1] = mk4(uy);
        }
        __syncthreads();
    }

    // C: interior face fluxes of the tile
    const int f0 = T.f_off[t], nF = T.f_off[t + 1] - f0;
    for (int j = tid; j < nF; j += kThreads) {
        int fid = T.f_id[f0 + j];
        int lr = T.f_lr[f0 + j];
        int il = lr & 0xffff, ir = lr >> 16;
        double q0[4], q1[4], Lf[4], Rf[4];
        double g0x[4] = {0, 0, 0, 0}, g0y[4] = {0, 0, 0, 0}, g1x[4] = {0, 0, 0, 0}, g1y[4] = {0, 0, 0, 0};
        ld4(ps[il], q0);
        ld4(ps[ir], q1);
        if (ORDER == 2) {
            int hh = T.f_hs[f0 + j];
            double2 gpl = hgp[hh & 0xffff], gpr = hgp[hh >> 16];
            ld4(gs[2 * il], g0x);
            ld4(gs[2 * il + 1], g0y);
            ld4(gs[2 * ir], g1x);
            ld4(gs[2 * ir + 1], g1y);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                Lf[v] = q0[v] + gpl.x * g0x[v] + gpl.y * g0y[v];
                Rf[v] = q1[v] + gpr.x * g1x[v] + gpr.y * g1y[v];
            }
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                Lf[v] = q0[v];
                Rf[v] = q1[v];
            }
        }
        double4 nl = m.face_nl[fid];
        double4 bb = NS ? m.face_bb[fid] : make_double4(0, 0, 1, 0);
        double F[4];
        face_flux<FLUX, NS>(P, nl.x, nl.y, nl.z, Lf, Rf, q0, q1, g0x, g0y, g1x, g1y, bb, F, L.flags);
        fs[j] = mk4(F);
    }
    __syncthreads();

    // D: per-cell flux sum in side order, update
    double r[4] = {0, 0, 0, 0};
    double dconv = 1e150, dvisc = 1e150;
    int bad = 0;
    const bool rk = L.mode == 1;
    for (int i = tid; i < nT; i += kThreads) {
        int d = T.e_ref[e0 + i];
        int h0 = m.hs_off[d], h1 = m.hs_off[d + 1];
        double s[4] = {0.0, 0.0, 0.0, 0.0};
        for (int h = h0; h < h1; ++h) {
            int code = T.u_code[h];
            double F[4];
            if (code >= 0) {
                ld4(fs[code >> 1], F);
                if (code & 1) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) s[v] += -F[v];
                } else {
#pragma unroll
                    for (int v = 0; v < 4; ++v) s[v] += F[v];
                }
            } else {
                ld4(L.bc_flux[-1 - code], F);
#pragma unroll
                for (int v = 0; v < 4; ++v) s[v] += F[v];
            }
        }
        double4 geo = m.cell_geo[d];
        double ut[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) ut[v] = (0.0 - s[v]) * geo.y;
        if (L.u_t) L.u_t[d] = mk4(ut);
        if (!rk && L.grad_out) {
            L.grad_out[2 * d] = gs[2 * i];
            L.grad_out[2 * d + 1] = gs[2 * i + 1];
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
                if (!local_dt(P, L.sp, pn, geo, &a, &b)) bad = 1;
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
}

// per-block minima of the convective and viscous time steps
__global__ void __launch_bounds__(256) k_dt(DevMesh m, Phys P, const Ctrl* ctrl, StepParams sp,
                                            const double4* __restrict__ prim,
                                            double2* __restrict__ partial, int* bad_partial) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double dconv = 1e150, dvisc = 1e150;
    int bad = 0;
    if (c < m.N) {
        double q[4];
        ld4(prim[c], q);
        if (!local_dt(P, sp, q, m.cell_geo[c], &dconv, &dvisc)) {
            bad = 1;
            dconv = dvisc = 1e150;
        }
    }
    block_min2(dconv, dvisc, bad, &partial[blockIdx.x], &bad_partial[blockIdx.x]);
}

// global dt from the partial minima with the output / end-time clamp
// (src/timeDiscretization.c:310-321)
__device__ void finish_dt(Ctrl* ctrl, const StepParams& sp, double dtc, double dtv, int bad) {
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

__device__ void reduce_min2(const double2* partial, const int* bad_partial, int nb, double* a_out,
                            double* b_out, int* bad_out) {
    __shared__ double sa[256], sb[256];
    __shared__ int sbad[256];
    int tid = threadIdx.x;
    double a = 1e150, b = 1e150;
    int bad = 0;
    for (int i = tid; i < nb; i += blockDim.x) {
        a = fmin(a, partial[i].x);
        b = fmin(b, partial[i].y);
        bad |= bad_partial[i];
    }
    sa[tid] = a; sb[tid] = b; sbad[tid] = bad;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s) {
            sa[tid] = fmin(sa[tid], sa[tid + s]);
            sb[tid] = fmin(sb[tid], sb[tid + s]);
            sbad[tid] |= sbad[tid + s];
        }
        __syncthreads();
    }
    *a_out = sa[0];
    *b_out = sb[0];
    *bad_out = sbad[0];
}

// first step of a run: dt of the current state, whether the step runs
__global__ void k_step_begin(Ctrl* ctrl, StepParams sp, const double2* __restrict__ partial,
                             const int* __restrict__ bad_partial, int nb) {
    double a, b;
    int bad;
    reduce_min2(partial, bad_partial, nb, &a, &b, &bad);
    if (threadIdx.x != 0) return;
    if (ctrl->done || ctrl->iter >= ctrl->stop_at) {
        ctrl->active = 0;
        return;
    }
    ctrl->active = 1;
    finish_dt(ctrl, sp, a, b, bad);
}

// end of a step: global residual, wing coefficients, t += dt, the stop tests
// of timeDisc (src/timeDiscretization.c:609-731) and the next step's dt
__global__ void k_step_end(Ctrl* ctrl, StepParams sp, const double* __restrict__ res_partial,
                           const double2* __restrict__ dt_partial, const int* __restrict__ dt_bad,
                           int nb, const int* __restrict__ wall_ghost,
                           const double* __restrict__ wall_nl,
                           const double* __restrict__ ghost_pface) {
    __shared__ double sh[4][256];
    int tid = threadIdx.x;
    if (!ctrl->active) return;
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = tid; i < nb; i += blockDim.x)
#pragma unroll
        for (int v = 0; v < 4; ++v) r[v] += res_partial[4 * i + v];
#pragma unroll
    for (int v = 0; v < 4; ++v) sh[v][tid] = r[v];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s)
#pragma unroll
            for (int v = 0; v < 4; ++v) sh[v][tid] += sh[v][tid + s];
        __syncthreads();
    }
    double dta, dtb;
    int dbad;
    reduce_min2(dt_partial, dt_bad, nb, &dta, &dtb, &dbad);
    if (tid != 0) return;
    double res[6];
#pragma unroll
    for (int v = 0; v < 4; ++v) res[v] = sqrt(sh[v][0] * sp.total_area_q);
    res[4] = res[5] = 0.0;
    double dt = ctrl->dt;
    ctrl->t += dt;
    long long iter = ctrl->iter + 1;
    ctrl->iter = iter;
    if (sp.calc_wing) {
        double cl_old = ctrl->cl, cd_old = ctrl->cd;
        double cl = 0.0, cd = 0.0;
        for (int k = 0; k < sp.n_wall; ++k) {
            double p0 = ghost_pface[wall_ghost[k]];
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
    if (!ctrl->have_first) {
#pragma unroll
        for (int v = 0; v < 4; ++v) ctrl->res_first[v] = res[v];
        ctrl->have_first = 1;
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
    // next step: dt of the new state (computed by the last stage)
    ctrl->active = 1;
    finish_dt(ctrl, sp, dta, dtb, dbad);
}

// ------------------------------------------------------------ dispatchers
template <int FLUX, int ORDER, int NS>
static void launch_k_stage(const StageLaunch& L, cudaStream_t st) {
    auto kern = k_stage<FLUX, ORDER, NS>;
    static int configured = 0;
    if (configured < L.tiles.smem_bytes) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.tiles.smem_bytes);
        configured = L.tiles.smem_bytes;
    }
    kern<<<L.tiles.n_tiles, kThreads, L.tiles.smem_bytes, st>>>(L);
}

template <int FLUX>
static void launch_flux(const StageLaunch& L, cudaStream_t st) {
    if (L.order == 2) {
        if (L.ns) launch_k_stage<FLUX, 2, 1>(L, st);
        else launch_k_stage<FLUX, 2, 0>(L, st);
    } else {
        if (L.ns) launch_k_stage<FLUX, 1, 1>(L, st);
        else launch_k_stage<FLUX, 1, 0>(L, st);
    }
}

void launch_stage(const StageLaunch& L, cudaStream_t st) {
    if (L.mesh.B > 0) {
        int nb = (L.mesh.B + 127) / 128;
        if (L.ns) k_bnd<1><<<nb, 128, 0, st>>>(L);
        else k_bnd<0><<<nb, 128, 0, st>>>(L);
    }
#define CCFD_FLUX_CASE(ID) \
    case ID: launch_flux<ID>(L, st); break;
    switch (L.flux_id) {
        CCFD_FLUX_CASE(1) CCFD_FLUX_CASE(2) CCFD_FLUX_CASE(3) CCFD_FLUX_CASE(4)
        CCFD_FLUX_CASE(5) CCFD_FLUX_CASE(6) CCFD_FLUX_CASE(7) CCFD_FLUX_CASE(8)
        CCFD_FLUX_CASE(9) CCFD_FLUX_CASE(10) CCFD_FLUX_CASE(11)
    }
#undef CCFD_FLUX_CASE
}

void launch_dt(const DevMesh& m, const Phys& P, const Ctrl* ctrl, const StepParams& sp,
               const double4* prim, double2* partial, int* bad_partial, cudaStream_t st) {
    k_dt<<<(m.N + 255) / 256, 256, 0, st>>>(m, P, ctrl, sp, prim, partial, bad_partial);
}

void launch_step_begin(Ctrl* ctrl, const StepParams& sp, const double2* partial,
                       const int* bad_partial, int nb, cudaStream_t st) {
    k_step_begin<<<1, 256, 0, st>>>(ctrl, sp, partial, bad_partial, nb);
}

void launch_step_end(Ctrl* ctrl, const StepParams& sp, const double* res_partial,
                     const double2* dt_partial, const int* dt_bad, int nb, const int* wall_ghost,
                     const double* wall_nl, const double* ghost_pface, cudaStream_t st) {
    k_step_end<<<1, 256, 0, st>>>(ctrl, sp, res_partial, dt_partial, dt_bad, nb, wall_ghost,
                                  wall_nl, ghost_pface);
}

}  // namespace ccfd
