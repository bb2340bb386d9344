// Kernels of the explicit residual-and-update path.
//
//   k_grad    per cell: ghost states at the mirrored barycentres, least-squares
//             gradient of the primitive variables over the cell's half-sides
//             in the reference's side order, Barth-Jespersen / Venkatakrishnan
//             limiting  (spatialReconstruction, src/reconstruction.c:198-314;
//             setBCatBarys, src/boundary.c:320-331)
//   k_face    per face: limited linear reconstruction of both states at the
//             face midpoint, ghost state at boundary faces, rotation into the
//             face frame, convective flux, viscous flux, rotation back, length
//             scaling  (setBCatSides src/boundary.c:300-314; fluxCalculation
//             src/fluxCalculation.c:882-998)
//   k_update  per cell: deterministic CSR sum of the face fluxes in the
//             reference's side order (no atomics), division by the area
//             (src/finiteVolume.c:96-120), fused Runge-Kutta stage update and
//             consPrim (src/timeDiscretization.c:362-398), partial sums of the
//             global residual (src/analyze.c:521-539)
//   k_dt / k_step_begin / k_step_end   calcTimeStep (src/timeDiscretization.c:
//             249-329), the per-step bookkeeping of timeDisc (:595-731) and the
//             wing coefficients of calcCoef (src/analyze.c:292-387), on device
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace ccfd {

__device__ __forceinline__ double stage_time(const Ctrl* ctrl, double tfix, double a_time) {
    return ctrl ? ctrl->t + a_time * ctrl->dt : tfix;
}

__device__ __forceinline__ bool inactive(const Ctrl* ctrl) {
    return ctrl && !ctrl->active;
}

__device__ __forceinline__ void ld4(const double4* p, int i, double q[4]) {
    double4 v = p[i];
    q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
}

__device__ __forceinline__ void st4(double4* p, int i, const double q[4]) {
    p[i] = make_double4(q[0], q[1], q[2], q[3]);
}

// ghost state at the mirrored barycentre of ghost g from the interior cell
// state q (setBCatBarys, src/boundary.c:320-331)
__device__ __forceinline__ void ghost_bary_state(const DevMesh& m, const Phys& P, int g,
                                                 double time, const double q[4], double out[4],
                                                 unsigned* flags) {
    double4 gn = m.ghost_gn[g];
    double x[2] = {gn.x, gn.y};
    boundary_state(P, P.bc[m.ghost_bc[g]], gn.z, gn.w, time, q, out, x, flags);
}

template <int LIM>
__global__ void __launch_bounds__(256) k_grad(DevMesh m, Phys P, const Ctrl* ctrl, double tfix,
                                              double a_time, const double4* __restrict__ prim,
                                              double4* __restrict__ grad, unsigned* flags) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.N || inactive(ctrl)) return;
    double time = stage_time(ctrl, tfix, a_time);
    double q[4];
    ld4(prim, c, q);
    int h0 = m.hs_off[c], nh = m.hs_off[c + 1] - h0;
    double ux[4] = {0.0, 0.0, 0.0, 0.0}, uy[4] = {0.0, 0.0, 0.0, 0.0};
    double umin[4] = {q[0], q[1], q[2], q[3]}, umax[4] = {q[0], q[1], q[2], q[3]};
    double gpx[4], gpy[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k < nh) {
            int h = h0 + k;
            int nb = m.hs_nb[h];
            double4 gw = m.hs_gw[h];
            gpx[k] = gw.x;
            gpy[k] = gw.y;
            double qn[4];
            if (nb >= 0) ld4(prim, nb, qn);
            else ghost_bary_state(m, P, -1 - nb, time, q, qn, flags);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                double d = qn[v] - q[v];
                ux[v] += gw.z * d;
                uy[v] += gw.w * d;
                umin[v] = fmin(umin[v], qn[v]);
                umax[v] = fmax(umax[v], qn[v]);
            }
        }
    }
    double minD[4], maxD[4], phi[4] = {1.0, 1.0, 1.0, 1.0};
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        minD[v] = umin[v] - q[v];
        maxD[v] = umax[v] - q[v];
    }
    if (LIM == 1) {
        // limiterBarthJespersen, src/reconstruction.c:25-96
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < nh) {
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    double uD = ux[v] * gpx[k] + uy[v] * gpy[k];
                    double pl = 1.0;
                    if (uD > 0.0) pl = fmin(1.0, maxD[v] / uD);
                    else if (uD < 0.0) pl = fmin(1.0, minD[v] / uD);
                    phi[v] = fmin(phi[v], pl);
                }
            }
        }
    } else {
        // limiterVenkatakrishnan, src/reconstruction.c:103-192
        double eps2 = m.venk_eps2[c];
        double minD2[4], maxD2[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            minD2[v] = minD[v] * minD[v];
            maxD2[v] = maxD[v] * maxD[v];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < nh) {
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    double uD = ux[v] * gpx[k] + uy[v] * gpy[k];
                    double uD2 = uD * uD;
                    double pl = 1.0;
                    if (uD > 0.0)
                        pl = 1.0 / uD * (((maxD2[v] + eps2) * uD + 2.0 * uD2 * maxD[v]) /
                                         (maxD2[v] + 2.0 * uD2 + uD * maxD[v] + eps2));
                    else if (uD < 0.0)
                        pl = 1.0 / uD * (((minD2[v] + eps2) * uD + 2.0 * uD2 * minD[v]) /
                                         (minD2[v] + 2.0 * uD2 + uD * minD[v] + eps2));
                    phi[v] = fmin(phi[v], pl);
                }
            }
        }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        ux[v] *= phi[v];
        uy[v] *= phi[v];
    }
    st4(grad, 2 * c, ux);
    st4(grad, 2 * c + 1, uy);
}

template <int FLUX, int ORDER, int NS>
__global__ void __launch_bounds__(256) k_face(DevMesh m, Phys P, const Ctrl* ctrl, double tfix,
                                              double a_time, const double4* __restrict__ prim,
                                              const double4* __restrict__ grad,
                                              double4* __restrict__ flux,
                                              double* __restrict__ ghost_pface, unsigned* flags) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.F || inactive(ctrl)) return;
    double time = stage_time(ctrl, tfix, a_time);
    int2 fc = m.face_c[f];
    double4 nl = m.face_nl[f];
    const double nx = nl.x, ny = nl.y;
    double q0[4], L[4], R[4];
    double g0x[4] = {0, 0, 0, 0}, g0y[4] = {0, 0, 0, 0}, g1x[4] = {0, 0, 0, 0}, g1y[4] = {0, 0, 0, 0};
    ld4(prim, fc.x, q0);
    double4 gp;
    if (ORDER == 2) {
        gp = m.face_gp[f];
        ld4(grad, 2 * fc.x, g0x);
        ld4(grad, 2 * fc.x + 1, g0y);
#pragma unroll
        for (int v = 0; v < 4; ++v) L[v] = q0[v] + gp.x * g0x[v] + gp.y * g0y[v];
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) L[v] = q0[v];
    }
    double q1[4];
    if (fc.y >= 0) {
        ld4(prim, fc.y, q1);
        if (ORDER == 2) {
            ld4(grad, 2 * fc.y, g1x);
            ld4(grad, 2 * fc.y + 1, g1y);
#pragma unroll
            for (int v = 0; v < 4; ++v) R[v] = q1[v] + gp.z * g1x[v] + gp.w * g1y[v];
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v) R[v] = q1[v];
        }
    } else {
        int g = -1 - fc.y;
        double2 mid = m.ghost_mid[g];
        double x[2] = {mid.x, mid.y};
        boundary_state(P, P.bc[m.ghost_bc[g]], nx, ny, time, L, R, x, flags);
        if (ghost_pface) ghost_pface[g] = L[3];
        if (NS) {
            // ghost cell state at its barycentre: set by setBCatBarys in the
            // second-order reconstruction only; zero (calloc) otherwise
            if (ORDER == 2) ghost_bary_state(m, P, g, time, q0, q1, flags);
            else q1[0] = q1[1] = q1[2] = q1[3] = 0.0;
        }
    }
    FluxIn<double> s;
    s.rL = L[0]; s.uL = nx * L[1] + ny * L[2]; s.vL = -ny * L[1] + nx * L[2]; s.pL = L[3];
    s.rR = R[0]; s.uR = nx * R[1] + ny * R[2]; s.vR = -ny * R[1] + nx * R[2]; s.pR = R[3];
    double fcv[4];
    convective_flux<FLUX, double>(P, s, fcv, flags);
    double F[4];
    F[0] = fcv[0];
    F[1] = nx * fcv[1] - ny * fcv[2];
    F[2] = ny * fcv[1] + nx * fcv[2];
    F[3] = fcv[3];
    if (NS) {
        // viscous flux with the compact-stencil gradient correction,
        // src/fluxCalculation.c:915-957 and :978-984
        double4 bb = m.face_bb[f];
        double st[4], gxm[4], gym[4], gx[4], gy[4];
        double bx = bb.x / bb.z, by = bb.y / bb.z;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            st[v] = 0.5 * (R[v] + L[v]);
            gxm[v] = 0.5 * (g0x[v] + g1x[v]);
            gym[v] = 0.5 * (g0y[v] + g1y[v]);
            double corr = gxm[v] * bx + gym[v] * by - (q1[v] - q0[v]) / bb.z;
            gx[v] = gxm[v] - corr * bx;
            gy[v] = gym[v] - corr * by;
        }
        double fdx[4], fdy[4];
        diffusion_flux(P, st, gx, gy, fdx, fdy);
#pragma unroll
        for (int v = 0; v < 4; ++v) F[v] -= (fdx[v] * nx + fdy[v] * ny);
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) F[v] *= nl.z;
    st4(flux, f, F);
}

// block-wide sum of NV values per thread into one partial per block (fixed
// tree, so the result is independent of timing)
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

// MODE 0: residual only (u_t written); MODE 1: Runge-Kutta stage update
template <int MODE>
__global__ void __launch_bounds__(256) k_update(DevMesh m, Phys P, const Ctrl* ctrl,
                                                const double4* __restrict__ flux,
                                                double4* __restrict__ cons0,
                                                double4* __restrict__ prim,
                                                double4* __restrict__ u_t_out, double rk,
                                                int last_stage, double* __restrict__ res_partial) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (inactive(ctrl)) return;
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    if (c < m.N) {
        double s[4] = {0.0, 0.0, 0.0, 0.0};
        int h0 = m.hs_off[c], h1 = m.hs_off[c + 1];
        for (int h = h0; h < h1; ++h) {
            int fs = m.hs_fs[h];
            double F[4];
            if (fs >= 0) {
                ld4(flux, fs, F);
#pragma unroll
                for (int v = 0; v < 4; ++v) s[v] += F[v];
            } else {
                ld4(flux, ~fs, F);
#pragma unroll
                for (int v = 0; v < 4; ++v) s[v] += -F[v];
            }
        }
        double4 geo = m.cell_geo[c];
        double ut[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) ut[v] = (0.0 - s[v]) * geo.y;
        if (u_t_out) st4(u_t_out, c, ut);
        if (MODE == 1) {
            double c0[4], cn[4], pn[4];
            ld4(cons0, c, c0);
            double adt = rk * ctrl->dt;
#pragma unroll
            for (int v = 0; v < 4; ++v) cn[v] = c0[v] + adt * ut[v];
            cons_prim(P.gam1, cn, pn);
            st4(prim, c, pn);
            if (last_stage) st4(cons0, c, cn);
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) r[v] = geo.x * ut[v] * ut[v];
    }
    if (res_partial) {
        double out[4];
        block_sum<4>(r, out);
        if (threadIdx.x == 0)
#pragma unroll
            for (int v = 0; v < 4; ++v) res_partial[4 * blockIdx.x + v] = out[v];
    }
}

// per-block minima of the convective and viscous time steps
__global__ void __launch_bounds__(256) k_dt(DevMesh m, Phys P, const Ctrl* ctrl, StepParams sp,
                                            const double4* __restrict__ prim,
                                            double2* __restrict__ partial, int* bad_partial) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (ctrl && (ctrl->done || ctrl->iter >= ctrl->stop_at)) return;
    double dconv = 1e150, dvisc = 1e150;
    int bad = 0;
    if (c < m.N) {
        double q[4];
        ld4(prim, c, q);
        double4 geo = m.cell_geo[c];
        double a = sqrt(P.gam * q[3] / q[0]);
        if (sp.ts1d) {
            dconv = sp.cfl * geo.w / (fabs(q[1]) + a);
            if (!isfinite(dconv)) bad = 1;
        } else {
            double ssr = (fabs(q[1]) + a) * geo.z + (fabs(q[2]) + a) * geo.w;
            dconv = sp.cfl * geo.x / ssr;
            if (!isfinite(dconv)) bad = 1;
            if (sp.visc) {
                double ssv = sp.gam_pr_max * P.mu * geo.z * geo.z + sp.gam_pr_max * P.mu * geo.w * geo.w;
                dvisc = sp.dfl * q[0] * q[0] * geo.x * geo.x / (4.0 * ssv);
                if (!isfinite(dvisc)) bad = 1;
            }
        }
        if (bad) { dconv = 1e150; dvisc = 1e150; }
    }
    block_min2(dconv, dvisc, bad, &partial[blockIdx.x], &bad_partial[blockIdx.x]);
}

// global time step with the output / end-time clamp; decides whether the
// step runs (src/timeDiscretization.c:249-329, 595-596)
__global__ void k_step_begin(Ctrl* ctrl, StepParams sp, const double2* __restrict__ partial,
                             const int* __restrict__ bad_partial, int nb) {
    __shared__ double sa[256], sb[256];
    __shared__ int sbad[256];
    int tid = threadIdx.x;
    bool run = !ctrl->done && ctrl->iter < ctrl->stop_at;
    double a = 1e150, b = 1e150;
    int bad = 0;
    if (run)
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
    if (tid != 0) return;
    if (!run) {
        ctrl->active = 0;
        return;
    }
    if (sbad[0]) {
        ctrl->flags |= FLAG_DT;
        ctrl->done = 1;
        ctrl->active = 0;
        return;
    }
    double dtc = sa[0], dtv = sb[0];
    double dt = sp.ts1d ? dtc : fmin(dtc, dtv);
    ctrl->visc_dominates = (!sp.ts1d && dtv < dtc) ? 1.0 : 0.0;
    double t = ctrl->t, pT = ctrl->print_time, sT = ctrl->stop_time;
    if ((t + dt > pT) || (t + dt > sT)) dt = fmin(pT, sT) - t;
    else if ((t + 1.5 * dt > pT) || (t + 1.5 * dt > sT)) dt = 0.5 * (fmin(pT, sT) - t);
    ctrl->dt = dt;
    ctrl->active = 1;
}

// end of a step: global residual, wing coefficients, t += dt and the stop
// tests of timeDisc (src/timeDiscretization.c:609-731)
__global__ void k_step_end(Ctrl* ctrl, StepParams sp, const double* __restrict__ res_partial,
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
    bool bad = false;
#pragma unroll
    for (int v = 0; v < 4; ++v) bad |= !isfinite(res[v]);
    if (bad) {
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
    }
}

// ------------------------------------------------------------ dispatchers
template <int FLUX>
static void launch_face_flux(int order, int ns, dim3 g, dim3 b, cudaStream_t st, const DevMesh& m,
                             const Phys& P, const Ctrl* ctrl, double tfix, double a_time,
                             const double4* prim, const double4* grad, double4* flux,
                             double* ghost_pface, unsigned* flags) {
    if (order == 2) {
        if (ns) k_face<FLUX, 2, 1><<<g, b, 0, st>>>(m, P, ctrl, tfix, a_time, prim, grad, flux, ghost_pface, flags);
        else k_face<FLUX, 2, 0><<<g, b, 0, st>>>(m, P, ctrl, tfix, a_time, prim, grad, flux, ghost_pface, flags);
    } else {
        if (ns) k_face<FLUX, 1, 1><<<g, b, 0, st>>>(m, P, ctrl, tfix, a_time, prim, grad, flux, ghost_pface, flags);
        else k_face<FLUX, 1, 0><<<g, b, 0, st>>>(m, P, ctrl, tfix, a_time, prim, grad, flux, ghost_pface, flags);
    }
}

void launch_residual(const ResidualLaunch& L, cudaStream_t st) {
    const DevMesh& m = L.mesh;
    dim3 b(256);
    dim3 gc((m.N + 255) / 256), gf((m.F + 255) / 256);
    if (L.order == 2) {
        if (L.limiter == 2)
            k_grad<2><<<gc, b, 0, st>>>(m, L.phys, L.ctrl, L.tfix, L.a_time, L.prim, L.grad, L.flags);
        else
            k_grad<1><<<gc, b, 0, st>>>(m, L.phys, L.ctrl, L.tfix, L.a_time, L.prim, L.grad, L.flags);
    }
#define CCFD_FACE_CASE(ID)                                                                  \
    case ID:                                                                                \
        launch_face_flux<ID>(L.order, L.ns, gf, b, st, m, L.phys, L.ctrl, L.tfix, L.a_time, \
                             L.prim, L.grad, L.flux, L.ghost_pface, L.flags);               \
        break;
    switch (L.flux_id) {
        CCFD_FACE_CASE(1)
        CCFD_FACE_CASE(2)
        CCFD_FACE_CASE(3)
        CCFD_FACE_CASE(4)
        CCFD_FACE_CASE(5)
        CCFD_FACE_CASE(6)
        CCFD_FACE_CASE(7)
        CCFD_FACE_CASE(8)
        CCFD_FACE_CASE(9)
        CCFD_FACE_CASE(10)
        CCFD_FACE_CASE(11)
    }
#undef CCFD_FACE_CASE
    if (L.update_mode == 1)
        k_update<1><<<gc, b, 0, st>>>(m, L.phys, L.ctrl, L.flux, L.cons0, L.prim_out, L.u_t,
                                      L.rk, L.last_stage, L.res_partial);
    else
        k_update<0><<<gc, b, 0, st>>>(m, L.phys, L.ctrl, L.flux, nullptr, nullptr, L.u_t, 0.0, 0,
                                      L.res_partial);
}

void launch_dt(const DevMesh& m, const Phys& P, const Ctrl* ctrl, const StepParams& sp,
               const double4* prim, double2* partial, int* bad_partial, cudaStream_t st) {
    k_dt<<<(m.N + 255) / 256, 256, 0, st>>>(m, P, ctrl, sp, prim, partial, bad_partial);
}

void launch_step_begin(Ctrl* ctrl, const StepParams& sp, const double2* partial,
                       const int* bad_partial, int nb, cudaStream_t st) {
    k_step_begin<<<1, 256, 0, st>>>(ctrl, sp, partial, bad_partial, nb);
}

void launch_step_end(Ctrl* ctrl, const StepParams& sp, const double* res_partial, int nb,
                     const int* wall_ghost, const double* wall_nl, const double* ghost_pface,
                     cudaStream_t st) {
    k_step_end<<<1, 256, 0, st>>>(ctrl, sp, res_partial, nb, wall_ghost, wall_nl, ghost_pface);
}

}  // namespace ccfd
