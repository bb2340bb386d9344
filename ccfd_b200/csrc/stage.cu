// Non-template kernels of the residual-and-update path and the dispatch of
// the stage kernels to the per-flux translation units (stage_fNN.cu):
//   k_dt / k_step_begin   calcTimeStep (src/timeDiscretization.c:249-329)
//            for the first step of a run
//   k_step_end_sep        end of an implicit time step
#include <cuda_runtime.h>

#include "stage_impl.cuh"

namespace ccfd {

// per-block minima of the convective and viscous time steps; the CFL
// number is the control block's under switched evolution relaxation
__global__ void __launch_bounds__(256) k_dt(DevMesh m, Phys P, const Ctrl* ctrl, StepParams sp,
                                            const double4* __restrict__ prim,
                                            double2* __restrict__ partial, int* bad_partial) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double dconv = 1e150, dvisc = 1e150;
    int bad = 0;
    const double cfl = (ctrl && sp.ser) ? ctrl->cfl : sp.cfl;
    const double dfl = (ctrl && sp.ser) ? ctrl->dfl : sp.dfl;
    if (c < m.N) {
        double q[4];
        ld4(prim[c], q);
        if (!local_dt(P, sp, cfl, dfl, q, m.cell_geo[c], &dconv, &dvisc)) {
            bad = 1;
            dconv = dvisc = 1e150;
        }
    }
    block_min2(dconv, dvisc, bad, &partial[blockIdx.x], &bad_partial[blockIdx.x]);
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

// end of an implicit step (the residual partials come from the last
// residual evaluation): global residual, stop tests and the CFL number of
// the next step; its dt follows from k_dt and k_step_dt
__global__ void k_step_end_sep(Ctrl* ctrl, StepParams sp, const double* res_partial, int nres,
                               const int* wall_ghost, const double* wall_nl,
                               const double* ghost_pface, const double4* prim_new) {
    if (!ctrl->active) return;
    step_end_block(ctrl, sp, res_partial, nres, nullptr, nullptr, 0, wall_ghost, wall_nl, ghost_pface,
                   prim_new, false);
}

// dt of the next step of a member that steps on (calcTimeStep of the new
// state, src/timeDiscretization.c:249-329)
__global__ void k_step_dt(Ctrl* ctrl, StepParams sp, const double2* __restrict__ partial,
                          const int* __restrict__ bad_partial, int nb) {
    double a, b;
    int bad;
    reduce_min2(partial, bad_partial, nb, &a, &b, &bad);
    if (threadIdx.x != 0 || !ctrl->active) return;
    finish_dt(ctrl, sp, a, b, bad);
}

void imp_step_end_launch(Ctrl* ctrl, const DevMesh& m, const Phys& P, const StepParams& sp,
                         const double* res_partial, int nres, double2* dt_partial, int* dt_bad, int ndt,
                         const int* wall_ghost, const double* wall_nl, const double* ghost_pface,
                         const double4* prim_new, cudaStream_t st) {
    k_step_end_sep<<<1, 256, 0, st>>>(ctrl, sp, res_partial, nres, wall_ghost, wall_nl, ghost_pface, prim_new);
    launch_dt(m, P, ctrl, sp, prim_new, dt_partial, dt_bad, st);
    k_step_dt<<<1, 256, 0, st>>>(ctrl, sp, dt_partial, dt_bad, ndt);
}


// ------------------------------------------------------------ dispatchers
int stage_smem_bytes(const TileDev& T, int fp32) {
    return fp32 ? stage_smem_bytes_t<float>(T) : stage_smem_bytes_t<double>(T);
}

void launch_stage(const StageLaunch& L, cudaStream_t st) {
#define CCFD_FLUX_CASE(ID) \
    case ID: launch_stage_f##ID(L, st); break;
    switch (L.flux_id) {
        CCFD_FLUX_CASE(1) CCFD_FLUX_CASE(2) CCFD_FLUX_CASE(3) CCFD_FLUX_CASE(4)
        CCFD_FLUX_CASE(5) CCFD_FLUX_CASE(6) CCFD_FLUX_CASE(7) CCFD_FLUX_CASE(8)
        CCFD_FLUX_CASE(9) CCFD_FLUX_CASE(10) CCFD_FLUX_CASE(11)
    }
#undef CCFD_FLUX_CASE
}

void launch_stage_batch(const BatchLaunch& B, cudaStream_t st) {
    if (B.n_tiles <= 0) return;
#define CCFD_FLUX_CASE(ID) \
    case ID: launch_stage_batch_f##ID(B, st); break;
    switch (B.flux_id) {
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

}  // namespace ccfd
