// Host-side launch interface of the residual-and-update kernels.
#pragma once

#include "solver.cuh"

namespace ccfd {

// Tiles of the fused stage kernel in device memory (see tiles.h).
struct TileDev {
    int n_tiles;
    int smem_bytes;
    int max_e, max_g, max_hs, max_f;
    int threads;          // CTA size of the single-instance stage kernel (0: the precision's default)
    int pad_[3];          // launch records stay a whole number of 16-byte words
    const int* e_off;     // [n_tiles + 1]
    const int4* counts;   // [n_tiles] (nT, nG, nE cells, nE)
    const int* e_ref;     // staged entries: device cell or -1-g
    const int* hs_off;    // [n_tiles + 1] into hs_nbl
    const short* hs_nbl;  // local E index of the neighbour of each gradient half-side
    const int* gl_off;    // [n_tiles + 1] into hs_loc
    const short* hs_loc;  // local half-side start per gradient cell (nG + 1 per tile)
    const int* f_off;     // [n_tiles + 1]
    const int* f_id;      // device interior face id
    const int* f_lr;      // packed local cell indices
    const int* f_hs;      // packed local half-side indices
    const int* u_code;    // [H] per device half-side: 2 * local face + neighbour flag, or -1-g
};

// Per-ghost data of the boundary kernel (device order of ghosts = BCside order).
struct GhostDev {
    const int* cell;       // interior device cell
    const int* hs;         // device half-side of the interior side
    const int* bc;         // BC table index
    const double4* gn;     // (ghost bary x, y, n.x, n.y)
    const double4* ml;     // (face midpoint x, y, len, 0)
    const double4* bb;     // (baryBaryVec x, y, baryBaryDist, 0) of the interior side
};

// One residual evaluation (optionally fused with a Runge-Kutta stage).
struct StageLaunch {
    DevMesh mesh;
    TileDev tiles;
    GhostDev ghosts;
    Phys phys;
    const Phys* phys_g;    // the same constants in global memory (boundary code)
    StepParams sp;
    const Ctrl* ctrl;      // device control block, or nullptr (fixed time)
    double tfix;           // time when ctrl == nullptr
    double a_time;         // stage time = t + a_time * dt
    int order, limiter, flux_id, ns;
    int fp32;              // 1: FP32 reconstruction and face fluxes (mixed precision)
    int mode;              // 0: residual u_t only; 1: RK stage; -1: no-op (batched stage slot)
    const int* skip;       // batched residual evaluations: skipped while *skip != 0
    const double4* prim_in;
    double4* prim_out;     // RK: updated primitive state
    double4* cons0;        // RK: stage-start conservative state (updated in place at the last stage)
    double* ghost_pface;   // [B] interior face pressure at boundary faces
    double4* u_t;          // [N] residual (mode 0, or RK last stage), may be nullptr
    double4* grad_out;     // [2N] limited gradients (mode 0 only), may be nullptr
    double rk;
    int last_stage;
    double* res_partial;   // [4 * n_tiles] or nullptr
    double2* dt_partial;   // [n_tiles] (last RK stage) or nullptr
    int* dt_bad;           // [n_tiles]
    unsigned* flags;
    unsigned* ticket;      // CTA completion counter of the last stage (zero between launches)
    const int* wall_ghost; // wing surface ghosts in calcCoef summation order
    const double* wall_nl; // their (n.x, n.y, len)
};

// Stage slots per instance and buffer parity in a batched RK launch record
// array (RK schemes have at most 5 stages).
constexpr int kBatchStages = 6;

// One launch of the stage kernel over the concatenated tiles of several
// instances that share the kernel variant (flux, order, equations, precision).
struct BatchLaunch {
    const StageLaunch* recs;  // rk_mode: [inst][2][kBatchStages], else [inst]
    const int2* tmap;         // [n_tiles] (instance, tile)
    int n_tiles, smem_bytes;
    int rk_mode, stage;
    int flux_id, order, ns, fp32;
    int* ctr;                 // [2] tile claim counter and finished CTAs, zero between launches
};

void launch_stage(const StageLaunch& L, cudaStream_t st);
void launch_stage_batch(const BatchLaunch& B, cudaStream_t st);
int stage_smem_bytes(const TileDev& T, int fp32);
void launch_dt(const DevMesh& m, const Phys& P, const Ctrl* ctrl, const StepParams& sp,
               const double4* prim, double2* partial, int* bad_partial, cudaStream_t st);
void launch_step_begin(Ctrl* ctrl, const StepParams& sp, const double2* partial,
                       const int* bad_partial, int nb, cudaStream_t st);
int error_blocks(int n_cells);
void launch_exact_state(int n, const double4* xq, const Phys* phys_g, int which, double time, double4* out,
                        unsigned* flags, cudaStream_t st);
void launch_errors(const DevMesh& m, const double4* xq, const double4* prim, const double4* grad,
                   const Phys* phys_g, int which, double time, double* partial, unsigned* flags,
                   cudaStream_t st);
void imp_step_end_launch(Ctrl* ctrl, const DevMesh& m, const Phys& P, const StepParams& sp,
                         const double* res_partial, int nres, double2* dt_partial, int* dt_bad, int ndt,
                         const int* wall_ghost, const double* wall_nl, const double* ghost_pface,
                         const double4* prim_new, cudaStream_t st);

}  // namespace ccfd
