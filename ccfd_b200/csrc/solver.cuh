// Device data layout and kernel declarations of the residual-and-update path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "physics.cuh"

namespace ccfd {

// Mesh in device memory, uploaded once: cells in Hilbert order, 32-bit
// indices, 32-byte records so that every gather of a record is one sector.
struct DevMesh {
    int N, F, B, H;           // cells, interior faces, ghosts, half-sides
    const int* hs_off;        // [N+1] CSR offsets of the per-cell half-sides
    const int* hs_nb;         // [H] neighbour cell, or -1-g for ghost g
    const double4* hs_gw;     // [H] (GP.x, GP.y, w.x, w.y)
    const double4* cell_geo;  // [N] (area, 1/area, sx, sy)
    const double* venk_eps2;  // [N] Venkatakrishnan epsilon^2
    const double4* face_nl;   // [F] (n.x, n.y, len, 0) of interior faces
    const double4* face_bb;   // [F] (baryBaryVec.x, .y, baryBaryDist, 0)
    const double4* cell_src;  // [N] (bary, fifth quad point) when the source term is on, else nullptr
    double4* src_buf;         // [N] the cells' source term of the running evaluation (with cell_src)
};

// Time-loop control block in device memory.  The time step, simulation time,
// output clamps and stop tests of timeDisc (src/timeDiscretization.c:
// 595-731) run on the device so that many steps are replayed as one CUDA
// graph without host round trips.
struct Ctrl {
    double t, dt, print_time, stop_time;
    double io_time_interval;
    long long iter, print_iter, io_iter_interval, max_iter, stop_at;
    int active;      // this step runs
    int done;        // no further steps (finished / converged / error / maxIter)
    int finished;    // stopTime reached
    int converged;   // stationary abort criterion met
    int max_iter_hit;
    unsigned flags;  // DevFlag bits
    double res[6];
    double res_first[4];
    int have_first;
    double cl, cd;
    double visc_dominates;
    int par;         // primitive buffer holding the current state (batched RK runs)
    double cfl, dfl; // CFL / DFL numbers of the next time step (switched evolution relaxation)
};

// Run parameters of the explicit integrator (kernel argument).
struct StepParams {
    double cfl, dfl, gam_pr_max;
    double rk[6];
    int nrk;
    int ts1d;
    int visc;             // mu > 1e-10
    int stationary;
    int abort_variable;
    double abort_residual, cl_abort, cd_abort, rel_abort;
    int abort_on_cl, abort_on_cd;
    int calc_wing;
    int n_wall;           // wall faces in CL/CD summation order
    double q_inf_lq, cos_a, sin_a;
    double total_area_q;
    // per-step history (the residual-file rows of analyze and the record
    // points, src/analyze.c:393-433): ring of hist_cap rows of hist_width
    // doubles, nullptr when off
    double* hist;
    int hist_cap, hist_width, n_rec;
    const int* rec_cell;  // [n_rec] device cell of each record point
    // switched evolution relaxation of the CFL number (implicit runs):
    // Ctrl::cfl = min(ser_cfl_max, cfl * r_1 / r_n) after step n,
    // Ctrl::dfl = dfl * Ctrl::cfl / cfl
    double ser_cfl_max;
    int ser, ser_pad;
};

// history row: iteration, t after the step, dt, residuals [6], CL, CD, then
// (rho, vx, vy, p) of each record point
constexpr int kHistHead = 11;

}  // namespace ccfd
