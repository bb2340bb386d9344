// Host-side launch interface of the explicit-path kernels.
#pragma once

#include "solver.cuh"

namespace ccfd {

// One residual evaluation R(U) (optionally fused with a Runge-Kutta stage).
struct ResidualLaunch {
    DevMesh mesh;
    Phys phys;
    const Ctrl* ctrl;      // device control block, or nullptr (fixed time)
    double tfix;           // time when ctrl == nullptr
    double a_time;         // stage time = t + a_time * dt
    int order, limiter, flux_id, ns;
    const double4* prim;   // [N] input primitive state
    double4* grad;         // [2N] limited gradients (scratch)
    double4* flux;         // [F] face fluxes (scratch)
    double* ghost_pface;   // [B] interior face pressure at boundary faces
    unsigned* flags;       // device error bits
    int update_mode;       // 0: write u_t only; 1: RK stage
    double4* cons0;        // [N] stage-start conservative state (RK)
    double4* prim_out;     // [N] updated primitive state (RK)
    double4* u_t;          // [N] residual output (may be nullptr in RK mode)
    double rk;             // RK coefficient of this stage
    int last_stage;
    double* res_partial;   // [4 * nblocks] residual partial sums or nullptr
};

void launch_residual(const ResidualLaunch& L, cudaStream_t st);
void launch_dt(const DevMesh& m, const Phys& P, const Ctrl* ctrl, const StepParams& sp,
               const double4* prim, double2* partial, int* bad_partial, cudaStream_t st);
void launch_step_begin(Ctrl* ctrl, const StepParams& sp, const double2* partial,
                       const int* bad_partial, int nb, cudaStream_t st);
void launch_step_end(Ctrl* ctrl, const StepParams& sp, const double* res_partial, int nb,
                     const int* wall_ghost, const double* wall_nl, const double* ghost_pface,
                     cudaStream_t st);

}  // namespace ccfd
