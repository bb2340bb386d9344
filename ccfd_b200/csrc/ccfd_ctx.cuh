// Device context of one solver instance (one mesh, one state) on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "ccfd_b200.h"
#include "kernels.cuh"
#include "solver.cuh"

struct ccfd_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    ccfd_params params;
    ccfd::Phys phys;
    ccfd::StepParams sp;
    ccfd::DevMesh mesh;
    ccfd::TileDev tiles;
    ccfd::GhostDev ghosts;
    int tile_cells = 256;
    int stage_threads = 0;  // CTA size of the stage kernel, 0: the precision's default
    ccfd_exact exact;
    double rk[6];
    double total_area_q = 0.0;
    long N = 0, F = 0, B = 0;
    bool uploaded = false;
    int last_cuda_error = 0;
    size_t device_bytes = 0;
    std::vector<void*> allocs;
    std::vector<int> cell_of_dev;  // device cell -> reference cell
    std::vector<int> dev_of_cell;  // reference cell -> device cell
    // state (primitive state ping-pong: a stage reads one buffer and writes
    // the other, because neighbouring tiles still read the old state)
    double4* prim_buf[2] = {nullptr, nullptr};
    int cur = 0;
    double4* cons0 = nullptr;
    double4* u_t = nullptr;
    double4* grad = nullptr;
    const double4* cell_xq = nullptr;  // [N] (bary, fifth quad point): source term and error norms
    const int* d_cell_of_dev = nullptr;  // [N] on the device: state transfers permute there
    const int* d_dev_of_cell = nullptr;
    double4* xfer = nullptr;             // [N] state in the reference's cell order (transfers)
    unsigned* ticket = nullptr;
    ccfd::Phys* phys_g = nullptr;
    double* ghost_pface = nullptr;
    unsigned* flags = nullptr;
    ccfd::Ctrl* ctrl = nullptr;
    ccfd::Ctrl* h_ctrl = nullptr;
    double2* dt_partial = nullptr;
    int* dt_bad = nullptr;
    double* res_partial = nullptr;
    int nb_cells = 0;
    int nb_part = 0;  // partial-array length: max(cell blocks, tiles)
    int* wall_ghost = nullptr;
    double* wall_nl = nullptr;
    int n_wall = 0;
    int n_wall_pressure = 0;       // pressure-side entries lead the wall list
    std::vector<double> wall_xy;   // wall face points (x, y) in wall-list order
    // step graphs per start buffer parity: [parity][0: one step, 1: many]
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    std::vector<cudaEvent_t> prof_ev[2][2];
    long newton_total = 0, gmres_total = 0;
    // profiling: event pairs around each residual evaluation in the graphs
    bool profiling = false;
    double prof_ms = 0.0;
    long prof_count = 0;
    cudaEvent_t ev_run0 = nullptr, ev_run1 = nullptr;
    cudaEvent_t ev_xfer = nullptr;  // end of a state upload's host-to-device copy
    // per-step history: device ring (sp.hist), rows drained to the host
    // after each synchronisation of a run
    long long hist_read = 0;         // last iteration drained
    std::vector<double> h_hist;      // drained rows not yet fetched
    void* implicit_state = nullptr;  // owned by the implicit solver
    void* batch = nullptr;           // the batch this context is stepped by, if any
};

// launch record of a residual evaluation / RK stage of this context with
// the fields common to all stages filled in (abi.cu)
void ccfd_fill_stage(ccfd_ctx* ctx, ccfd::StageLaunch& L);
// status code of device error flags; report from the host copy of the
// control block (abi.cu)
int ccfd_status_from_flags(unsigned f);
void ccfd_fill_report(ccfd_ctx* ctx, ccfd_report* r);
// stream-ordered device allocation from the library's memory pool of the
// current device (abi.cu); free with cudaFreeAsync
cudaError_t ccfd_malloc_async(void** p, size_t bytes, cudaStream_t st);
// copy the history rows recorded since the last drain (up to the
// iteration in ctx->h_ctrl, which the caller has refreshed) to the host
int ccfd_history_drain(ccfd_ctx* ctx);
// device-side residual of the current state into ctx->u_t (abi.cu)
int ccfd_residual_device(ccfd_ctx* ctx, double time);
// residual of an arbitrary primitive state into ut (abi.cu)
int ccfd_residual_of(ccfd_ctx* ctx, const double4* prim, double time, double4* ut);
// implicit solver set-up / release (implicit.cu); the device buffers are
// owned by the context's allocation list
int ccfd_implicit_setup(ccfd_ctx* ctx, const std::vector<int>& hs_off, const std::vector<int>& hs_nb);
void ccfd_implicit_free(ccfd_ctx* ctx);
