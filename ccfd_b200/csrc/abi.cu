// C ABI of the device path: context, one-time mesh upload, state transfer,
// residual evaluation and explicit time stepping under CUDA graphs.
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "ccfd_b200.h"
#include "ccfd_ctx.cuh"
#include "host/ccfd_host.h"
#include "kernels.cuh"
#include "tiles.h"

using namespace ccfd;

#define CK(x)                               \
    do {                                    \
        cudaError_t e_ = (x);               \
        if (e_ != cudaSuccess) {            \
            ctx->last_cuda_error = (int)e_; \
            return CCFD_ERR_CUDA;           \
        }                                   \
    } while (0)

int ccfd_status_from_flags(unsigned f) {
    if (f & FLAG_DT) return CCFD_ERR_DT;
    if (f & FLAG_VACUUM) return CCFD_ERR_VACUUM;
    if (f & FLAG_STATE) return CCFD_ERR_STATE;
    if (f & FLAG_SINGULAR) return CCFD_ERR_SINGULAR;
    if (f & FLAG_GMRES) return CCFD_ERR_GMRES;
    if (f & FLAG_NEWTON) return CCFD_ERR_NEWTON;
    return CCFD_OK;
}

// One memory pool per device for all of the library's device buffers.  The
// default pool hands freed memory back to the driver at synchronisations,
// which made releasing a context take up to a second in a serving loop;
// this pool keeps up to CCFD_POOL_KEEP_BYTES (default: all) of freed
// memory for the next contexts.
static std::mutex g_pool_mu;
static cudaMemPool_t g_pool[64];

cudaError_t ccfd_malloc_async(void** p, size_t bytes, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, st);
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (!g_pool[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            if ((e = cudaMemPoolCreate(&g_pool[dev], &props)) != cudaSuccess) {
                g_pool[dev] = nullptr;
                return e;
            }
            unsigned long long keep = ~0ull;
            if (const char* v = getenv("CCFD_POOL_KEEP_BYTES")) keep = strtoull(v, nullptr, 10);
            cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool = g_pool[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

template <typename T>
static int dalloc(ccfd_ctx* ctx, T** p, size_t n) {
    void* q = nullptr;
    if (n == 0) n = 1;
    // stream-ordered: allocating and freeing a context never waits for the
    // work of other contexts (a serving loop admits while others step)
    cudaError_t e = ccfd_malloc_async(&q, n * sizeof(T), ctx->stream);
    if (e != cudaSuccess) {
        ctx->last_cuda_error = (int)e;
        return CCFD_ERR_NOMEM;
    }
    ctx->allocs.push_back(q);
    ctx->device_bytes += n * sizeof(T);
    *p = (T*)q;
    return CCFD_OK;
}

template <typename T>
static int dupload(ccfd_ctx* ctx, T** p, const std::vector<T>& h) {
    int st = dalloc(ctx, p, h.size());
    if (st) return st;
    if (!h.empty())
        CK(cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return CCFD_OK;
}

template <typename T>
static int dupload_c(ccfd_ctx* ctx, const T** p, const std::vector<T>& h) {
    T* q = nullptr;
    int st = dupload(ctx, &q, h);
    *p = q;
    return st;
}

static void drop_graphs(ccfd_ctx* ctx) {
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            if (ctx->graph[a][b]) cudaGraphExecDestroy(ctx->graph[a][b]);
            ctx->graph[a][b] = nullptr;
            for (cudaEvent_t e : ctx->prof_ev[a][b]) cudaEventDestroy(e);
            ctx->prof_ev[a][b].clear();
        }
}

static void free_device(ccfd_ctx* ctx) {
    drop_graphs(ctx);
    ccfd_implicit_free(ctx);
    for (void* p : ctx->allocs) cudaFreeAsync(p, ctx->stream);
    ctx->allocs.clear();
    ctx->device_bytes = 0;
    ctx->uploaded = false;
}

extern "C" int ccfd_set_device(int device) {
    return cudaSetDevice(device) == cudaSuccess ? CCFD_OK : CCFD_ERR_CUDA;
}

extern "C" int ccfd_create(const ccfd_params* params, ccfd_ctx** out) {
    if (!params || !out) return CCFD_ERR_ARG;
    *out = nullptr;
    const ccfd_params& p = *params;
    if (p.flux < 1 || p.flux > 11 || p.spatial_order < 1 || p.spatial_order > 2 ||
        (p.spatial_order == 2 && p.limiter != 1 && p.limiter != 2) || p.time_order < 1 ||
        p.time_order > 3 ||
        (!(p.n_rk_stages == 1 && p.time_order == 1) && (p.n_rk_stages < 3 || p.n_rk_stages > 5)) ||
        p.source_func < 0 || p.source_func > 1)
        return CCFD_ERR_ARG;
    if (p.time_step_1d && p.mu > 1e-10 && p.eqn == CCFD_NAVIER_STOKES)
        return CCFD_ERR_ARG; /* src/timeDiscretization.c:264-267 */
    int dev = 0, ndev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CCFD_ERR_CUDA;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return CCFD_ERR_CUDA;
    ccfd_ctx* ctx = new ccfd_ctx();
    ctx->params = p;
    ctx->device = dev;
    // a context's own stream has the highest priority: its uploads, state
    // transfers and releases then do not queue behind the long stage
    // launches of a batch that steps other contexts (serving)
    int prio_least = 0, prio_greatest = 0;
    cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
    if (cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, prio_greatest) != cudaSuccess) {
        delete ctx;
        return CCFD_ERR_CUDA;
    }
    // host copy of the control block in ordinary memory: releasing pinned
    // memory would wait for all work on the device (other contexts included)
    ctx->h_ctrl = new Ctrl();
    if (cudaEventCreate(&ctx->ev_run0) != cudaSuccess || cudaEventCreate(&ctx->ev_run1) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_xfer, cudaEventDisableTiming) != cudaSuccess) {
        if (ctx->ev_run0) cudaEventDestroy(ctx->ev_run0);
        if (ctx->ev_run1) cudaEventDestroy(ctx->ev_run1);
        delete ctx->h_ctrl;
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return CCFD_ERR_CUDA;
    }
    memset(ctx->h_ctrl, 0, sizeof(Ctrl));
    // RK coefficient tables, src/timeDiscretization.c:94-169
    double* rk = ctx->rk;
    for (int i = 0; i < 6; ++i) rk[i] = 0.0;
    if (p.n_rk_stages == 1 && p.time_order == 1) {
        rk[1] = 1.0;
    } else {
        static const double t3[3][3] = {{0.1418, 0.4, 1.0}, {0.1918, 0.4929, 1.0}, {0.2884, 0.5010, 1.0}};
        static const double t4[3][4] = {
            {0.0833, 0.2069, 0.4265, 1.0}, {0.1084, 0.2602, 0.5052, 1.0}, {0.1666, 0.3027, 0.5275, 1.0}};
        static const double t5[3][5] = {{0.0533, 0.1263, 0.2375, 0.4414, 1.0},
                                        {0.0695, 0.1602, 0.2898, 0.5060, 1.0},
                                        {0.1067, 0.1979, 0.3232, 0.5201, 1.0}};
        int o = p.time_order - 1;
        for (int s = 0; s < p.n_rk_stages; ++s)
            rk[s + 1] = p.n_rk_stages == 3 ? t3[o][s] : p.n_rk_stages == 4 ? t4[o][s] : t5[o][s];
    }
    // explicit mixed precision (FP32 staging): smaller tiles and CTAs, six
    // per SM (0.366 against 0.393 ms per RK3 step at 256 x 256 on the
    // 500k-triangle double Mach reflection)
    if (p.precision == CCFD_MIXED && !p.implicit) ctx->tile_cells = 192;
    const char* tc = getenv("CCFD_TILE_CELLS");
    if (tc) ctx->tile_cells = std::max(32, std::min(2048, atoi(tc)));
    const char* th = getenv("CCFD_STAGE_THREADS");
    if (th) ctx->stage_threads = std::max(0, std::min(1024, atoi(th))) & ~31;
    *out = ctx;
    return CCFD_OK;
}

extern "C" void ccfd_destroy(ccfd_ctx* ctx) {
    if (!ctx) return;
    if (ctx->batch) ccfd_batch_remove((ccfd_batch*)ctx->batch, ctx);
    cudaStreamSynchronize(ctx->stream);
    free_device(ctx);
    if (ctx->ev_run0) cudaEventDestroy(ctx->ev_run0);
    if (ctx->ev_run1) cudaEventDestroy(ctx->ev_run1);
    if (ctx->ev_xfer) cudaEventDestroy(ctx->ev_xfer);
    delete ctx->h_ctrl;
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

// wing surface faces in the summation order of calcCoef: the pressure-side
// list then the suction-side list, each built by the insertion of initWing
// (src/analyze.c:95-184), keyed on the face midpoint x
static void build_wall_list(const ccfd_mesh* m, const ccfd_bc* bc, int wall_code,
                            std::vector<int>& order, int* n_pressure) {
    std::vector<int> pressure, suction;
    for (long g = 0; g < m->n_bc; ++g) {
        const ccfd_bc& b = bc[m->bc_index[g]];
        if (b.type * 100 + b.id != wall_code) continue;
        long f = m->bc_face[g];
        double ghost_ny = -m->face_n[2 * f + 1];
        std::vector<int>& L = ghost_ny <= 0.0 ? suction : pressure;
        double xi = m->bc_x[2 * g];
        size_t pos = L.size();
        for (size_t k = 0; k < L.size(); ++k)
            if (xi < m->bc_x[2 * L[k]]) {
                pos = k;
                break;
            }
        L.insert(L.begin() + pos, (int)g);
    }
    order = pressure;
    order.insert(order.end(), suction.begin(), suction.end());
    *n_pressure = (int)pressure.size();
}

// Host loop over [0, n) split across up to 16 threads (the gathers from the
// reference's cell order into the device order are memory-latency bound).
template <typename Fn>
static void par_for(long n, Fn fn) {
    unsigned hw = std::thread::hardware_concurrency();
    long nth = std::max(1L, std::min<long>(hw ? hw : 1, std::min(16L, n / 32768)));
    std::vector<std::thread> pool;
    for (long k = 0; k + 1 < nth; ++k) pool.emplace_back(fn, n * k / nth, n * (k + 1) / nth);
    fn(n * (nth - 1) / nth, n);
    for (std::thread& th : pool) th.join();
}

// Host staging of an upload, kept per thread from one upload to the next:
// filling a few hundred MB of freshly allocated host memory per upload cost
// more in page faults than the work itself.
struct UploadScratch {
    std::vector<int> cperm, cinv, fint, fdev, cnt, hs_off, hs_nb, hs_dev_of_ref;
    std::vector<int> g_cell, g_hs, g_bc, gl_off;
    std::vector<double4> hs_gw, cell_geo, cell_xq, face_nl, face_bb, g_gn, g_ml, g_bb;
    std::vector<double> venk, e2;
    std::vector<int4> counts;
    std::vector<short> hs_nbl, hs_loc;
    TileSet ts;
};
static thread_local UploadScratch tl_upload;

extern "C" int ccfd_upload_case(ccfd_ctx* ctx, const ccfd_mesh* m, const ccfd_bc* bc, int n_bc,
                                const ccfd_exact* ex, int reorder) {
    if (!ctx || !m || (!bc && n_bc > 0) || !ex || n_bc > kMaxBC) return CCFD_ERR_ARG;
    if (m->n_cells <= 0 || m->n_faces <= 0 || m->n_cells > (1L << 30) || m->n_faces > (1L << 30))
        return CCFD_ERR_ARG;
    for (long g = 0; g < m->n_bc; ++g)
        if (m->bc_index[g] < 0 || m->bc_index[g] >= n_bc) return CCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    free_device(ctx);
    const ccfd_params& p = ctx->params;
    const long N = m->n_cells, F = m->n_faces, B = m->n_bc;
    ctx->N = N;
    ctx->B = B;
    UploadScratch& S = tl_upload;

    // cell order: Hilbert curve of the barycentres (or the reference order);
    // results do not depend on it, only the storage order changes
    std::vector<int>& cperm = S.cperm;
    if (reorder == 2) ccfd_rcm_order(m, cperm);
    else if (reorder) ccfd_hilbert_order(m, cperm);
    else {
        cperm.resize(N);
        for (long i = 0; i < N; ++i) cperm[i] = (int)i;
    }
    std::vector<int>& cinv = S.cinv;
    cinv.resize(N);
    for (long i = 0; i < N; ++i) cinv[cperm[i]] = (int)i;
    ctx->cell_of_dev = cperm;
    ctx->dev_of_cell = cinv;

    // interior faces in the order of their owner's device index
    // (stable counting sort by the owner's device index)
    std::vector<int>& fint = S.fint;
    {
        std::vector<int>& cnt = S.cnt;
        cnt.assign(N + 1, 0);
        long nfi = 0;
        for (long f = 0; f < F; ++f)
            if (m->face_cells[2 * f + 1] >= 0) {
                ++cnt[cinv[m->face_cells[2 * f]] + 1];
                ++nfi;
            }
        for (long d = 0; d < N; ++d) cnt[d + 1] += cnt[d];
        fint.resize(nfi);
        for (long f = 0; f < F; ++f)
            if (m->face_cells[2 * f + 1] >= 0) fint[cnt[cinv[m->face_cells[2 * f]]]++] = (int)f;
    }
    std::vector<int>& fdev = S.fdev;
    fdev.assign(F, -1);
    for (size_t i = 0; i < fint.size(); ++i) fdev[fint[i]] = (int)i;
    const long FI = (long)fint.size();
    ctx->F = FI;

    // per-cell CSR in device order
    std::vector<int>& hs_off = S.hs_off;
    std::vector<int>& hs_nb = S.hs_nb;
    std::vector<double4>& hs_gw = S.hs_gw;
    std::vector<double4>& cell_geo = S.cell_geo;
    std::vector<double4>& cell_xq = S.cell_xq;
    std::vector<int>& hs_dev_of_ref = S.hs_dev_of_ref;
    hs_off.resize(N + 1);
    cell_geo.resize(N);
    cell_xq.resize(N);
    hs_dev_of_ref.resize(m->n_half_sides);
    hs_off[0] = 0;
    for (long d = 0; d < N; ++d) {
        long c = cperm[d];
        hs_off[d + 1] = hs_off[d] + (int)(m->hs_offset[c + 1] - m->hs_offset[c]);
    }
    hs_nb.resize(hs_off[N]);
    hs_gw.resize(hs_off[N]);
    std::vector<double>& venk = S.venk;
    venk.resize(N);
    const bool vk = p.spatial_order == 2 && p.limiter == 2;
    par_for(N, [&](long d0, long d1) {
        for (long d = d0; d < d1; ++d) {
            long c = cperm[d];
            long k = hs_off[d];
            for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h, ++k) {
                long nb = m->hs_nb[h];
                hs_dev_of_ref[h] = (int)k;
                hs_nb[k] = nb >= 0 ? cinv[nb] : (int)nb;
                hs_gw[k] = make_double4(m->hs_gp[2 * h], m->hs_gp[2 * h + 1], m->hs_w[2 * h], m->hs_w[2 * h + 1]);
            }
            cell_geo[d] = make_double4(m->cell_geo[4 * c], m->cell_geo[4 * c + 1], m->cell_geo[4 * c + 2],
                                       m->cell_geo[4 * c + 3]);
            const double* b = &m->cell_bary[2 * c];
            const double* q5 = m->cell_gp5 ? &m->cell_gp5[2 * c] : b;
            cell_xq[d] = make_double4(b[0], b[1], q5[0], q5[1]);
            // src/finiteVolume.c:47-52, as ccfd_venk_eps2
            const double a = m->cell_geo[4 * c];
            venk[d] = vk ? (p.venk_k * sqrt(a)) * (p.venk_k * sqrt(a)) * (p.venk_k * sqrt(a)) : 0.0;
        }
    });
    // face geometry; the barycentre vectors only for the viscous fluxes
    const bool ns = p.eqn == CCFD_NAVIER_STOKES;
    std::vector<double4>& face_nl = S.face_nl;
    std::vector<double4>& face_bb = S.face_bb;
    face_nl.resize(FI + 1);
    face_bb.resize(ns ? FI + 1 : 1);
    face_nl[FI] = face_bb[face_bb.size() - 1] = make_double4(0, 0, 0, 0);
    par_for(FI, [&](long i0, long i1) {
        for (long i = i0; i < i1; ++i) {
            long f = fint[i];
            face_nl[i] = make_double4(m->face_n[2 * f], m->face_n[2 * f + 1], m->face_len[f], 0.0);
            if (ns) face_bb[i] = make_double4(m->face_bb[3 * f], m->face_bb[3 * f + 1], m->face_bb[3 * f + 2], 0.0);
        }
    });
    // ghosts (BCside order)
    std::vector<int>& g_cell = S.g_cell;
    std::vector<int>& g_hs = S.g_hs;
    std::vector<int>& g_bc = S.g_bc;
    std::vector<double4>& g_gn = S.g_gn;
    std::vector<double4>& g_ml = S.g_ml;
    std::vector<double4>& g_bb = S.g_bb;
    g_cell.assign(B + 1, 0);
    g_hs.assign(B + 1, 0);
    g_bc.assign(B + 1, 0);
    g_gn.assign(B + 1, make_double4(0, 0, 0, 0));
    g_ml.assign(B + 1, make_double4(0, 0, 0, 0));
    g_bb.assign(B + 1, make_double4(0, 0, 0, 0));
    for (long g = 0; g < B; ++g) {
        long f = m->bc_face[g];
        g_cell[g] = cinv[m->face_cells[2 * f]];
        g_hs[g] = hs_dev_of_ref[m->face_hs[2 * f]];
        g_bc[g] = m->bc_index[g];
        g_gn[g] = make_double4(m->bc_ghost_bary[2 * g], m->bc_ghost_bary[2 * g + 1], m->face_n[2 * f],
                               m->face_n[2 * f + 1]);
        g_ml[g] = make_double4(m->bc_x[2 * g], m->bc_x[2 * g + 1], m->face_len[f], 0.0);
        g_bb[g] = make_double4(m->face_bb[3 * f], m->face_bb[3 * f + 1], m->face_bb[3 * f + 2], 0.0);
    }
    // tiles of the fused stage kernel
    TileSet& ts = S.ts;
    ccfd_build_tiles(m, cperm, cinv, fdev, ctx->tile_cells, ts);
    if (ts.max_e >= 32768 || ts.max_hs >= 32768) return CCFD_ERR_ARG;
    std::vector<int4>& counts = S.counts;
    std::vector<int>& gl_off = S.gl_off;
    counts.resize(ts.n_tiles);
    gl_off.assign(ts.n_tiles + 1, 0);
    for (int t = 0; t < ts.n_tiles; ++t) {
        counts[t] = make_int4(ts.counts[4 * t], ts.counts[4 * t + 1], ts.counts[4 * t + 2], ts.counts[4 * t + 3]);
        gl_off[t + 1] = gl_off[t] + ts.counts[4 * t + 1] + 1;
    }
    int st;
    DevMesh& dm = ctx->mesh;
    memset(&dm, 0, sizeof(dm));
    TileDev& td = ctx->tiles;
    memset(&td, 0, sizeof(td));
    GhostDev& gd = ctx->ghosts;
    memset(&gd, 0, sizeof(gd));
    std::vector<short>& hs_nbl = S.hs_nbl;
    std::vector<short>& hs_loc = S.hs_loc;
    hs_nbl.assign(ts.hs_nbl.begin(), ts.hs_nbl.end());
    hs_loc.assign(ts.hs_loc.begin(), ts.hs_loc.end());
    if ((st = dupload_c(ctx, &dm.hs_off, hs_off)) || (st = dupload_c(ctx, &dm.hs_nb, hs_nb)) ||
        (st = dupload_c(ctx, &dm.hs_gw, hs_gw)) || (st = dupload_c(ctx, &dm.cell_geo, cell_geo)) ||
        (st = dupload_c(ctx, &dm.venk_eps2, venk)) || (st = dupload_c(ctx, &dm.face_nl, face_nl)) ||
        (st = dupload_c(ctx, &dm.face_bb, face_bb)) || (st = dupload_c(ctx, &gd.cell, g_cell)) ||
        (st = dupload_c(ctx, &gd.hs, g_hs)) || (st = dupload_c(ctx, &gd.bc, g_bc)) ||
        (st = dupload_c(ctx, &gd.gn, g_gn)) || (st = dupload_c(ctx, &gd.ml, g_ml)) ||
        (st = dupload_c(ctx, &gd.bb, g_bb)) || (st = dupload_c(ctx, &td.e_off, ts.e_off)) ||
        (st = dupload_c(ctx, &td.counts, counts)) || (st = dupload_c(ctx, &td.e_ref, ts.e_ref)) ||
        (st = dupload_c(ctx, &td.hs_off, ts.hs_off)) || (st = dupload_c(ctx, &td.hs_nbl, hs_nbl)) ||
        (st = dupload_c(ctx, &td.gl_off, gl_off)) || (st = dupload_c(ctx, &td.hs_loc, hs_loc)) ||
        (st = dupload_c(ctx, &td.f_off, ts.f_off)) || (st = dupload_c(ctx, &td.f_id, ts.f_id)) ||
        (st = dupload_c(ctx, &td.f_lr, ts.f_lr)) || (st = dupload_c(ctx, &td.f_hs, ts.f_hs)) ||
        (st = dupload_c(ctx, &td.u_code, ts.u_code)) || (st = dupload_c(ctx, &ctx->cell_xq, cell_xq))) {
        free_device(ctx);
        return st;
    }
    if (p.source_func) {
        dm.cell_src = ctx->cell_xq;
        if ((st = dalloc(ctx, &dm.src_buf, (size_t)N))) {
            free_device(ctx);
            return st;
        }
    }
    dm.N = (int)N;
    dm.F = (int)FI;
    dm.B = (int)B;
    dm.H = hs_off[N];
    td.n_tiles = ts.n_tiles;
    td.max_e = ts.max_e;
    td.max_g = ts.max_g;
    td.max_hs = ts.max_hs;
    td.max_f = ts.max_f;
    td.smem_bytes = stage_smem_bytes(td, 0);  // FP64 staging: the larger of the two layouts
    td.threads = ctx->stage_threads;
    int smem_max = 0;
    CK(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    if (td.smem_bytes > smem_max) {
        free_device(ctx);
        return CCFD_ERR_ARG;
    }

    // physics constants (src/equation.c:572-578)
    Phys& P = ctx->phys;
    memset(&P, 0, sizeof(P));
    P.gam = p.gamma;
    P.gam1 = p.gamma - 1.0;
    P.gam1q = 1.0 / P.gam1;
    P.mu = p.eqn == CCFD_NAVIER_STOKES ? p.mu : 0.0;
    P.Pr = p.eqn == CCFD_NAVIER_STOKES ? p.Pr : 0.72;
    P.pi = acos(-1.0);
    P.sqrt3q = 1 / sqrt(3.0);
    P.nbc = n_bc;
    P.order = p.spatial_order;
    P.eqn = p.eqn;
    P.source_func = p.source_func;
    for (int i = 0; i < n_bc; ++i) {
        P.bc[i].type = bc[i].type;
        P.bc[i].exact_func = bc[i].exact_func;
        for (int v = 0; v < 4; ++v) P.bc[i].pvar[v] = bc[i].pvar[v];
    }
    memcpy(P.ex.ref_state, ex->ref_state, sizeof(P.ex.ref_state));
    P.ex.rp1d_interface = ex->rp1d_interface;
    P.ex.x_min = ex->x_min;
    P.ex.x_max = ex->x_max;
    P.ex.y_min = ex->y_min;
    P.ex.y_max = ex->y_max;
    P.ex.dx_ref = ex->dx_ref;
    ctx->total_area_q = m->total_area_q;
    ctx->exact = *ex;
    if ((st = dalloc(ctx, &ctx->phys_g, 1))) {
        free_device(ctx);
        return st;
    }
    CK(cudaMemcpyAsync(ctx->phys_g, &ctx->phys, sizeof(Phys), cudaMemcpyHostToDevice, ctx->stream));

    // wing surface list for CL / CD
    std::vector<int> wl;
    std::vector<double> wnl;
    ctx->n_wall_pressure = 0;
    ctx->wall_xy.clear();
    if (p.calc_wing) build_wall_list(m, bc, p.wall_id, wl, &ctx->n_wall_pressure);
    for (int g : wl) {
        long f = m->bc_face[g];
        ctx->wall_xy.push_back(m->bc_x[2 * g]);
        ctx->wall_xy.push_back(m->bc_x[2 * g + 1]);
        wnl.push_back(m->face_n[2 * f]);
        wnl.push_back(m->face_n[2 * f + 1]);
        wnl.push_back(m->face_len[f]);
    }
    ctx->n_wall = (int)wl.size();
    if ((st = dupload(ctx, &ctx->wall_ghost, wl)) || (st = dupload(ctx, &ctx->wall_nl, wnl))) {
        free_device(ctx);
        return st;
    }

    // state and scratch
    ctx->nb_cells = (int)((N + 255) / 256);
    ctx->nb_part = std::max(ctx->nb_cells, ts.n_tiles);
    if ((st = dupload_c(ctx, &ctx->d_cell_of_dev, ctx->cell_of_dev)) ||
        (st = dupload_c(ctx, &ctx->d_dev_of_cell, ctx->dev_of_cell)) || (st = dalloc(ctx, &ctx->xfer, N)) ||
        (st = dalloc(ctx, &ctx->prim_buf[0], N)) || (st = dalloc(ctx, &ctx->prim_buf[1], N)) ||
        (st = dalloc(ctx, &ctx->cons0, N)) || (st = dalloc(ctx, &ctx->u_t, N)) ||
        (st = dalloc(ctx, &ctx->grad, 2 * N)) || (st = dalloc(ctx, &ctx->ticket, 1)) ||
        (st = dalloc(ctx, &ctx->ghost_pface, B + 1)) ||
        (st = dalloc(ctx, &ctx->flags, 1)) || (st = dalloc(ctx, &ctx->ctrl, 1)) ||
        (st = dalloc(ctx, &ctx->dt_partial, ctx->nb_part)) || (st = dalloc(ctx, &ctx->dt_bad, ctx->nb_part)) ||
        (st = dalloc(ctx, &ctx->res_partial, 4 * (size_t)ctx->nb_part))) {
        free_device(ctx);
        return st;
    }
    ctx->cur = 0;
    CK(cudaMemsetAsync(ctx->flags, 0, sizeof(unsigned), ctx->stream));
    CK(cudaMemsetAsync(ctx->ticket, 0, sizeof(unsigned), ctx->stream));
    CK(cudaMemsetAsync(ctx->ghost_pface, 0, sizeof(double) * (B + 1), ctx->stream));
    CK(cudaMemsetAsync(ctx->grad, 0, sizeof(double4) * 2 * N, ctx->stream));
    CK(cudaMemsetAsync(ctx->res_partial, 0, sizeof(double) * 4 * ctx->nb_part, ctx->stream));

    // control block: t = 0, printTime / printIter of initTimeDisc
    // (src/timeDiscretization.c:238-239)
    Ctrl& c = *ctx->h_ctrl;
    memset(&c, 0, sizeof(Ctrl));
    c.t = 0.0;
    c.stop_time = p.t_end;
    c.io_time_interval = p.io_time_interval;
    c.io_iter_interval = p.io_iter_interval > 0 ? p.io_iter_interval : 1;
    c.print_time = (floor(0.0 / p.io_time_interval) + 1) * p.io_time_interval;
    c.print_iter = (0 / c.io_iter_interval + 1) * c.io_iter_interval;
    c.max_iter = p.max_iter;
    c.stop_at = 0;
    c.cfl = p.cfl;
    c.dfl = p.dfl;
    CK(cudaMemcpyAsync(ctx->ctrl, ctx->h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));

    // step parameters
    StepParams& sp = ctx->sp;
    memset(&sp, 0, sizeof(sp));
    sp.cfl = p.cfl;
    sp.dfl = p.dfl;
    sp.ser = p.implicit && p.ser_cfl_max > 0.0;
    sp.ser_cfl_max = p.ser_cfl_max;
    sp.gam_pr_max = fmax(4.0 / 3.0, P.gam / P.Pr);
    for (int i = 0; i < 6; ++i) sp.rk[i] = ctx->rk[i];
    sp.nrk = (p.n_rk_stages == 1 && p.time_order == 1) ? 1 : p.n_rk_stages;
    sp.ts1d = p.time_step_1d;
    sp.visc = P.mu > 1e-10;
    sp.stationary = p.stationary;
    sp.abort_variable = p.abort_variable;
    sp.abort_residual = p.abort_residual;
    sp.cl_abort = p.cl_abort_residual;
    sp.cd_abort = p.cd_abort_residual;
    sp.abort_on_cl = p.cl_abort_residual > 0.0;
    sp.abort_on_cd = !sp.abort_on_cl && p.cd_abort_residual > 0.0;
    sp.rel_abort = p.rel_abort_residual;
    sp.calc_wing = p.calc_wing && ctx->n_wall > 0;
    sp.n_wall = ctx->n_wall;
    {
        double pi = acos(-1.0);
        double v = ex->ref_state[0][1] / cos(ex->alpha * pi / 180.0);
        double q_inf_q = 1.0 / (ex->ref_state[0][0] * 0.5 * v * v);
        sp.q_inf_lq = q_inf_q / p.ref_length;
        double a = ex->alpha * pi / 180.0;
        sp.cos_a = cos(a);
        sp.sin_a = sin(a);
    }
    sp.total_area_q = m->total_area_q;
    if (p.implicit && (st = ccfd_implicit_setup(ctx, hs_off, hs_nb))) {
        free_device(ctx);
        return st;
    }
    ctx->uploaded = true;
    return CCFD_OK;
}

void ccfd_fill_stage(ccfd_ctx* ctx, StageLaunch& L) {
    memset(&L, 0, sizeof(L));
    L.mesh = ctx->mesh;
    L.tiles = ctx->tiles;
    L.ghosts = ctx->ghosts;
    L.phys = ctx->phys;
    L.phys_g = ctx->phys_g;
    L.sp = ctx->sp;
    L.order = ctx->params.spatial_order;
    L.limiter = ctx->params.limiter;
    L.flux_id = ctx->params.flux;
    L.ns = ctx->params.eqn == CCFD_NAVIER_STOKES;
    // mixed precision: FP32 face fluxes in the explicit scheme; the implicit
    // scheme keeps FP64 residuals (its finite-difference Jacobian-vector
    // products divide residual differences by a tiny perturbation)
    L.fp32 = ctx->params.precision == CCFD_MIXED && !ctx->params.implicit;
    L.ghost_pface = ctx->ghost_pface;
    L.flags = ctx->flags;
    L.ticket = ctx->ticket;
    L.wall_ghost = ctx->wall_ghost;
    L.wall_nl = ctx->wall_nl;
}

static int check_flags(ccfd_ctx* ctx) {
    unsigned f = 0;
    CK(cudaMemcpyAsync(&f, ctx->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (f) CK(cudaMemsetAsync(ctx->flags, 0, sizeof(unsigned), ctx->stream));
    return ccfd_status_from_flags(f);
}

// primitive buffer of the current state (a batch member's parity lives in
// its control block, whose host copy the batch refreshes after each call)
static double4* cur_prim(ccfd_ctx* ctx) {
    return ctx->prim_buf[ctx->batch ? ctx->h_ctrl->par : ctx->cur];
}

// State transfers move the caller's array as it is (reference cell order)
// and permute / convert on the device: a pinned caller buffer goes by DMA
// at full speed, and no host loop touches the cells.
__global__ void k_state_in(int n, const double4* __restrict__ src, const int* __restrict__ cell_of_dev,
                           int conservative, double gam1, double gam1q, double4* __restrict__ prim,
                           double4* __restrict__ cons) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const double4 v = src[cell_of_dev[d]];
    double a[4] = {v.x, v.y, v.z, v.w}, pv[4], cv[4];
    if (conservative) {
        for (int k = 0; k < 4; ++k) cv[k] = a[k];
        cons_prim(gam1, cv, pv);
    } else {
        for (int k = 0; k < 4; ++k) pv[k] = a[k];
        prim_cons(gam1q, pv, cv);
    }
    prim[d] = make_double4(pv[0], pv[1], pv[2], pv[3]);
    cons[d] = make_double4(cv[0], cv[1], cv[2], cv[3]);
}

__global__ void k_state_out(int n, const double4* __restrict__ src, const int* __restrict__ dev_of_cell,
                            double4* __restrict__ dst) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) dst[c] = src[dev_of_cell[c]];
}

extern "C" int ccfd_set_state(ccfd_ctx* ctx, const double* state, int kind) {
    if (!ctx || !state || !ctx->uploaded) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    CK(cudaSetDevice(ctx->device));
    const long N = ctx->N;
    CK(cudaMemcpyAsync(ctx->xfer, state, sizeof(double4) * N, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaEventRecord(ctx->ev_xfer, ctx->stream));
    k_state_in<<<(unsigned)((N + 255) / 256), 256, 0, ctx->stream>>>(
        (int)N, ctx->xfer, ctx->d_cell_of_dev, kind == CCFD_CONSERVATIVE, ctx->phys.gam1, ctx->phys.gam1q,
        cur_prim(ctx), ctx->cons0);
    CK(cudaGetLastError());
    // the caller's array is free once the copy is done; the permutation runs
    // on in stream order before anything else that reads the state (a batch
    // synchronises the context's stream when it takes the context in)
    CK(cudaEventSynchronize(ctx->ev_xfer));
    return CCFD_OK;
}

extern "C" int ccfd_get_state(ccfd_ctx* ctx, double* state, int kind) {
    if (!ctx || !state || !ctx->uploaded) return CCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    const long N = ctx->N;
    k_state_out<<<(unsigned)((N + 255) / 256), 256, 0, ctx->stream>>>(
        (int)N, kind == CCFD_CONSERVATIVE ? ctx->cons0 : cur_prim(ctx), ctx->d_dev_of_cell, ctx->xfer);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(state, ctx->xfer, sizeof(double4) * N, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CCFD_OK;
}

extern "C" int ccfd_set_time(ccfd_ctx* ctx, double t) {
    if (!ctx || !ctx->uploaded) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    Ctrl& c = *ctx->h_ctrl;
    c.t = t;
    c.print_time = (floor(t / ctx->params.io_time_interval) + 1) * ctx->params.io_time_interval;
    c.done = c.finished = c.converged = c.max_iter_hit = 0;
    c.flags = 0;
    CK(cudaMemcpyAsync(ctx->ctrl, ctx->h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CCFD_OK;
}

extern "C" int ccfd_get_time(ccfd_ctx* ctx, double* t) {
    if (!ctx || !t || !ctx->uploaded) return CCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *t = ctx->h_ctrl->t;
    return CCFD_OK;
}

// Residual of the current state into ctx->u_t (device); no host copies.
int ccfd_residual_device(ccfd_ctx* ctx, double time) {
    StageLaunch L;
    ccfd_fill_stage(ctx, L);
    L.ctrl = nullptr;
    L.tfix = time;
    L.mode = 0;
    L.prim_in = cur_prim(ctx);
    L.u_t = ctx->u_t;
    L.grad_out = ctx->params.spatial_order == 2 ? ctx->grad : nullptr;
    L.res_partial = ctx->res_partial;
    launch_stage(L, ctx->stream);
    CK(cudaGetLastError());
    return CCFD_OK;
}

int ccfd_residual_of(ccfd_ctx* ctx, const double4* prim, double time, double4* ut) {
    StageLaunch L;
    ccfd_fill_stage(ctx, L);
    L.ctrl = nullptr;
    L.tfix = time;
    L.mode = 0;
    L.prim_in = prim;
    L.u_t = ut;
    L.res_partial = ctx->res_partial;
    launch_stage(L, ctx->stream);
    CK(cudaGetLastError());
    return CCFD_OK;
}

extern "C" int ccfd_residual(ccfd_ctx* ctx, double time, double* u_t_out, double* grad_out) {
    if (!ctx || !ctx->uploaded) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    CK(cudaSetDevice(ctx->device));
    int st = ccfd_residual_device(ctx, time);
    if (st) return st;
    const long N = ctx->N;
    if (u_t_out) {
        std::vector<double4> h(N);
        CK(cudaMemcpyAsync(h.data(), ctx->u_t, sizeof(double4) * N, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (long d = 0; d < N; ++d) {
            double* s = &u_t_out[4 * ctx->cell_of_dev[d]];
            s[0] = h[d].x; s[1] = h[d].y; s[2] = h[d].z; s[3] = h[d].w;
        }
    }
    if (grad_out) {
        std::vector<double4> h(2 * N);
        CK(cudaMemcpyAsync(h.data(), ctx->grad, sizeof(double4) * 2 * N, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (long d = 0; d < N; ++d) {
            double* s = &grad_out[8 * ctx->cell_of_dev[d]];
            s[0] = h[2 * d].x; s[1] = h[2 * d].y; s[2] = h[2 * d].z; s[3] = h[2 * d].w;
            s[4] = h[2 * d + 1].x; s[5] = h[2 * d + 1].y; s[6] = h[2 * d + 1].z; s[7] = h[2 * d + 1].w;
        }
    }
    return check_flags(ctx);
}

// calcErrors (src/analyze.c:445-514) at the current time: the limited
// gradients of the current state (spatialReconstruction, as one residual
// evaluation that writes only the gradients), then the per-cell quadrature
// errors against exact function `exact_func` and the CTA partials summed
// here in CTA order.
extern "C" int ccfd_errors(ccfd_ctx* ctx, int exact_func, double out[12]) {
    if (!ctx || !out || !ctx->uploaded || exact_func < 1 || exact_func > 6) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    CK(cudaSetDevice(ctx->device));
    double t = 0.0;
    int st = ccfd_get_time(ctx, &t);
    if (st) return st;
    const bool second = ctx->params.spatial_order == 2;
    if (second) {
        StageLaunch L;
        ccfd_fill_stage(ctx, L);
        L.ctrl = nullptr;
        L.tfix = t;
        L.mode = 0;
        L.prim_in = cur_prim(ctx);
        L.u_t = nullptr;
        L.grad_out = ctx->grad;
        L.res_partial = nullptr;
        L.ghost_pface = nullptr;
        launch_stage(L, ctx->stream);
        CK(cudaGetLastError());
    }
    const int nb = error_blocks((int)ctx->N);
    double* part = nullptr;
    CK(ccfd_malloc_async((void**)&part, sizeof(double) * 12 * nb, ctx->stream));
    launch_errors(ctx->mesh, ctx->cell_xq, cur_prim(ctx), second ? ctx->grad : nullptr, ctx->phys_g, exact_func, t,
                  part, ctx->flags, ctx->stream);
    cudaError_t le = cudaGetLastError();
    std::vector<double> h(12 * (size_t)nb);
    cudaError_t ce = le == cudaSuccess ? cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(),
                                                         cudaMemcpyDeviceToHost, ctx->stream)
                                       : le;
    cudaFreeAsync(part, ctx->stream);
    CK(ce);
    CK(cudaStreamSynchronize(ctx->stream));
    double l1[4] = {0, 0, 0, 0}, l2[4] = {0, 0, 0, 0}, li[4] = {0, 0, 0, 0};
    for (int b = 0; b < nb; ++b)
        for (int v = 0; v < 4; ++v) {
            l1[v] += h[12 * b + v];
            l2[v] += h[12 * b + 4 + v];
            li[v] = fmax(li[v], h[12 * b + 8 + v]);
        }
    for (int v = 0; v < 4; ++v) {
        out[v] = l1[v] * ctx->total_area_q;
        out[4 + v] = sqrt(l2[v] * ctx->total_area_q);
        out[8 + v] = li[v];
    }
    return check_flags(ctx);
}

extern "C" int ccfd_exact_state(ccfd_ctx* ctx, int exact_func, double time, double* prim_out) {
    if (!ctx || !prim_out || !ctx->uploaded || exact_func < 1 || exact_func > 6) return CCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    const long N = ctx->N;
    double4* out = nullptr;
    CK(ccfd_malloc_async((void**)&out, sizeof(double4) * N, ctx->stream));
    launch_exact_state((int)N, ctx->cell_xq, ctx->phys_g, exact_func, time, out, ctx->flags, ctx->stream);
    cudaError_t le = cudaGetLastError();
    std::vector<double4> h(N);
    cudaError_t ce = le == cudaSuccess ? cudaMemcpyAsync(h.data(), out, sizeof(double4) * N,
                                                         cudaMemcpyDeviceToHost, ctx->stream)
                                       : le;
    cudaFreeAsync(out, ctx->stream);
    CK(ce);
    CK(cudaStreamSynchronize(ctx->stream));
    for (long d = 0; d < N; ++d) {
        double* s = &prim_out[4 * ctx->cell_of_dev[d]];
        s[0] = h[d].x; s[1] = h[d].y; s[2] = h[d].z; s[3] = h[d].w;
    }
    return check_flags(ctx);
}

// Per-step history (analyze, src/analyze.c:393-433): the step end writes a
// row per step into a device ring; runs drain it after each host
// synchronisation (every graph of at most 16 steps, every implicit step,
// every batch call), so the ring needs no more than those rows.
extern "C" int ccfd_set_history(ccfd_ctx* ctx, int capacity, const long* record_cells, int n_record) {
    if (!ctx || !ctx->uploaded || n_record < 0 || n_record > CCFD_MAX_RECORD || (n_record > 0 && !record_cells))
        return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    for (int k = 0; k < n_record; ++k)
        if (record_cells[k] < 0 || record_cells[k] >= ctx->N) return CCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    StepParams& sp = ctx->sp;
    drop_graphs(ctx);  // the step graphs hold the step parameters by value
    ctx->h_hist.clear();
    if (capacity <= 0) {
        sp.hist = nullptr;
        sp.n_rec = 0;
        sp.rec_cell = nullptr;
        return CCFD_OK;
    }
    if (capacity < 64) capacity = 64;
    const int width = kHistHead + 4 * n_record;
    std::vector<int> cells(n_record > 0 ? n_record : 1, 0);
    for (int k = 0; k < n_record; ++k) cells[k] = ctx->dev_of_cell[record_cells[k]];
    double* ring = nullptr;
    const int* rec = nullptr;
    int st;
    if ((st = dalloc(ctx, &ring, (size_t)capacity * width)) || (st = dupload_c(ctx, &rec, cells))) return st;
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->hist_read = ctx->h_ctrl->iter;
    sp.hist = ring;
    sp.hist_cap = capacity;
    sp.hist_width = width;
    sp.n_rec = n_record;
    sp.rec_cell = rec;
    return CCFD_OK;
}

int ccfd_history_drain(ccfd_ctx* ctx) {
    const StepParams& sp = ctx->sp;
    const long long now = ctx->h_ctrl->iter;
    if (!sp.hist || now <= ctx->hist_read) {
        ctx->hist_read = now > ctx->hist_read ? now : ctx->hist_read;
        return CCFD_OK;
    }
    long long first = ctx->hist_read + 1;
    if (now - first + 1 > sp.hist_cap) first = now - sp.hist_cap + 1;  // older rows were overwritten
    const size_t w = (size_t)sp.hist_width, old = ctx->h_hist.size();
    const long long n = now - first + 1;
    ctx->h_hist.resize(old + (size_t)n * w);
    // one copy per contiguous run of ring slots (at most two)
    long long it = first;
    double* dst = ctx->h_hist.data() + old;
    while (it <= now) {
        long long slot = (it - 1) % sp.hist_cap;
        long long run = std::min<long long>(now - it + 1, sp.hist_cap - slot);
        CK(cudaMemcpyAsync(dst, sp.hist + slot * w, sizeof(double) * w * run, cudaMemcpyDeviceToHost, ctx->stream));
        dst += run * w;
        it += run;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->hist_read = now;
    return CCFD_OK;
}

extern "C" int ccfd_get_history(ccfd_ctx* ctx, double* rows, long max_rows, long* n_rows, int* width) {
    if (!ctx || !n_rows) return CCFD_ERR_ARG;
    const long w = ctx->sp.hist ? ctx->sp.hist_width : kHistHead;
    if (width) *width = (int)w;
    const long have = (long)(ctx->h_hist.size() / (size_t)w);
    if (!rows) {
        *n_rows = have;
        return CCFD_OK;
    }
    const long n = std::min(have, max_rows < 0 ? 0L : max_rows);
    std::copy(ctx->h_hist.begin(), ctx->h_hist.begin() + n * w, rows);
    ctx->h_hist.erase(ctx->h_hist.begin(), ctx->h_hist.begin() + n * w);
    *n_rows = n;
    return CCFD_OK;
}

// Autotuner of the stage kernel's launch shape: cells per tile (which sets
// the CTA's faces and gradient cells per thread) and the cell ordering
// (Hilbert curve or the reference's numbering).  Every candidate is uploaded
// and timed over a few residual evaluations of the given state; the context
// keeps the fastest.  Results do not depend on the choice (the arithmetic
// and the summation order per cell are the same for every tiling).
extern "C" int ccfd_autotune(ccfd_ctx* ctx, const ccfd_mesh* m, const ccfd_bc* bc, int n_bc,
                             const ccfd_exact* ex, const double* prim, int* tile_cells_out,
                             int* reorder_out, int* threads_out, double* ms_out) {
    if (!ctx || !m || !ex || !prim) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    CK(cudaSetDevice(ctx->device));
    static const int kTiles[] = {128, 192, 256, 320, 384};
    // CTA sizes at or below the precision's launch bounds (FP64 384, FP32 256)
    static const int kThreads64[] = {256, 320, 384}, kThreads32[] = {128, 192, 256};
    const bool fp32 = ctx->params.precision == CCFD_MIXED && !ctx->params.implicit;
    const int* thr_list = fp32 ? kThreads32 : kThreads64;
    const int kReps = 5;
    // the two timing events are released on every return path
    struct Events {
        cudaEvent_t a = nullptr, b = nullptr;
        ~Events() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } ev;
    CK(cudaEventCreate(&ev.a));
    CK(cudaEventCreate(&ev.b));
    double best = 1e300;
    int best_tile = ctx->tile_cells, best_order = 1, best_threads = ctx->stage_threads;
    for (int order = 1; order >= 0; --order)
        for (int tc : kTiles) {
            ctx->tile_cells = tc;
            int st = ccfd_upload_case(ctx, m, bc, n_bc, ex, order);
            if (st == CCFD_ERR_ARG) continue;  // tile too large for shared memory
            if (st || (st = ccfd_set_state(ctx, prim, CCFD_PRIMITIVE))) return st;
            // the CTA size changes the launch only: time each on the same tiles
            for (int k = 0; k < 3; ++k) {
                ctx->tiles.threads = thr_list[k];
                if ((st = ccfd_residual_device(ctx, 0.0))) return st;  // warm-up
                CK(cudaEventRecord(ev.a, ctx->stream));
                for (int r = 0; r < kReps; ++r)
                    if ((st = ccfd_residual_device(ctx, 0.0))) return st;
                CK(cudaEventRecord(ev.b, ctx->stream));
                CK(cudaEventSynchronize(ev.b));
                float ms = 0.0f;
                CK(cudaEventElapsedTime(&ms, ev.a, ev.b));
                if (ms / kReps < best) {
                    best = ms / kReps;
                    best_tile = tc;
                    best_order = order;
                    best_threads = thr_list[k];
                }
            }
        }
    ctx->tile_cells = best_tile;
    ctx->stage_threads = best_threads;
    int st = ccfd_upload_case(ctx, m, bc, n_bc, ex, best_order);
    if (!st) st = ccfd_set_state(ctx, prim, CCFD_PRIMITIVE);
    if (tile_cells_out) *tile_cells_out = best_tile;
    if (reorder_out) *reorder_out = best_order;
    if (threads_out) *threads_out = best_threads;
    if (ms_out) *ms_out = best;
    return st;
}

extern "C" int ccfd_global_residual(ccfd_ctx* ctx, double res[4]) {
    if (!ctx || !res || !ctx->uploaded) return CCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    std::vector<double> h(4 * (size_t)ctx->tiles.n_tiles);
    CK(cudaMemcpyAsync(h.data(), ctx->res_partial, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double s[4] = {0, 0, 0, 0};
    for (int b = 0; b < ctx->tiles.n_tiles; ++b)
        for (int v = 0; v < 4; ++v) s[v] += h[4 * b + v];
    for (int v = 0; v < 4; ++v) res[v] = sqrt(s[v] * ctx->total_area_q);
    return CCFD_OK;
}

extern "C" int ccfd_time_step(ccfd_ctx* ctx, double* dt_out) {
    if (!ctx || !dt_out || !ctx->uploaded) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    CK(cudaSetDevice(ctx->device));
    launch_dt(ctx->mesh, ctx->phys, ctx->ctrl, ctx->sp, cur_prim(ctx), ctx->dt_partial, ctx->dt_bad, ctx->stream);
    CK(cudaGetLastError());
    std::vector<double2> part(ctx->nb_cells);
    std::vector<int> bad(ctx->nb_cells);
    CK(cudaMemcpyAsync(part.data(), ctx->dt_partial, sizeof(double2) * part.size(), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaMemcpyAsync(bad.data(), ctx->dt_bad, sizeof(int) * bad.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double a = 1e150, b = 1e150;
    for (int i = 0; i < ctx->nb_cells; ++i) {
        if (bad[i]) return CCFD_ERR_DT;
        a = fmin(a, part[i].x);
        b = fmin(b, part[i].y);
    }
    double dt = ctx->sp.ts1d ? a : fmin(a, b);
    const Ctrl& c = *ctx->h_ctrl;
    double t = c.t, pT = c.print_time, sT = c.stop_time;
    if ((t + dt > pT) || (t + dt > sT)) dt = fmin(pT, sT) - t;
    else if ((t + 1.5 * dt > pT) || (t + 1.5 * dt > sT)) dt = 0.5 * (fmin(pT, sT) - t);
    *dt_out = dt;
    return CCFD_OK;
}

// Record one explicit time step starting from primitive buffer `par` into
// the stream (graph capture); returns the parity after the step.  With
// profiling, each stage is bracketed by two event-record nodes.
static int record_step(ccfd_ctx* ctx, int par, const std::vector<cudaEvent_t>* ev, size_t* ev_next) {
    const StepParams& sp = ctx->sp;
    for (int s = 1; s <= sp.nrk; ++s) {
        StageLaunch L;
        ccfd_fill_stage(ctx, L);
        L.ctrl = ctx->ctrl;
        L.a_time = sp.rk[s - 1];
        L.mode = 1;
        L.prim_in = ctx->prim_buf[par];
        L.prim_out = ctx->prim_buf[par ^ 1];
        L.cons0 = ctx->cons0;
        L.rk = sp.rk[s];
        L.last_stage = s == sp.nrk;
        L.res_partial = L.last_stage ? ctx->res_partial : nullptr;
        L.dt_partial = L.last_stage ? ctx->dt_partial : nullptr;
        L.dt_bad = ctx->dt_bad;
        if (ev) cudaEventRecordWithFlags((*ev)[(*ev_next)++], ctx->stream, cudaEventRecordExternal);
        launch_stage(L, ctx->stream);
        if (ev) cudaEventRecordWithFlags((*ev)[(*ev_next)++], ctx->stream, cudaEventRecordExternal);
        par ^= 1;
    }
    return par;
}

static int build_graph(ccfd_ctx* ctx, int par, int steps, cudaGraphExec_t* exec, std::vector<cudaEvent_t>* ev) {
    cudaGraph_t g;
    if (ev) {
        // events are created before the capture begins
        size_t need = (size_t)steps * ctx->sp.nrk * 2;
        while (ev->size() < need) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            ev->push_back(e);
        }
    }
    size_t ev_next = 0;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < steps; ++i) par = record_step(ctx, par, ev, &ev_next);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (e != cudaSuccess) {
        ctx->last_cuda_error = (int)e;
        return CCFD_ERR_CUDA;
    }
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        ctx->last_cuda_error = (int)e;
        return CCFD_ERR_CUDA;
    }
    return CCFD_OK;
}

void ccfd_fill_report(ccfd_ctx* ctx, ccfd_report* r) {
    const Ctrl& c = *ctx->h_ctrl;
    memset(r, 0, sizeof(*r));
    r->t = c.t;
    r->dt = c.dt;
    r->iterations = c.iter;
    for (int v = 0; v < 6; ++v) r->residual[v] = c.res[v];
    for (int v = 0; v < 4; ++v) r->first_residual[v] = c.res_first[v];
    r->cl = c.cl;
    r->cd = c.cd;
    r->converged = c.converged;
    r->finished = c.finished;
    r->newton_iterations = ctx->newton_total;
    r->gmres_iterations = ctx->gmres_total;
    r->status = ccfd_status_from_flags(c.flags);
}

// accumulate the stage times of the steps that ran (their event pairs come
// first in the graph)
static int collect_profile(ccfd_ctx* ctx, const std::vector<cudaEvent_t>& ev, size_t pairs) {
    for (size_t i = 0; i < pairs && 2 * i + 1 < ev.size(); ++i) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]));
        ctx->prof_ms += ms;
        ctx->prof_count += 1;
    }
    return CCFD_OK;
}

extern "C" int ccfd_set_profiling(ccfd_ctx* ctx, int on) {
    if (!ctx) return CCFD_ERR_ARG;
    if ((bool)on != ctx->profiling) {
        CK(cudaSetDevice(ctx->device));
        drop_graphs(ctx);
        ctx->profiling = on != 0;
    }
    ctx->prof_ms = 0.0;
    ctx->prof_count = 0;
    return CCFD_OK;
}

extern "C" int ccfd_get_profile(ccfd_ctx* ctx, double* residual_ms, long* residual_count, int reset) {
    if (!ctx || !residual_ms || !residual_count) return CCFD_ERR_ARG;
    *residual_ms = ctx->prof_ms;
    *residual_count = ctx->prof_count;
    if (reset) {
        ctx->prof_ms = 0.0;
        ctx->prof_count = 0;
    }
    return CCFD_OK;
}

extern "C" int ccfd_run_explicit(ccfd_ctx* ctx, long nsteps, ccfd_report* report) {
    if (!ctx || !ctx->uploaded) return CCFD_ERR_ARG;
    if (ctx->batch) return CCFD_ERR_BUSY;
    if (ctx->params.implicit) return ccfd_run_implicit(ctx, nsteps, report);
    CK(cudaSetDevice(ctx->device));
    int st;
    const int kMany = 16;
    const bool prof = ctx->profiling;
    const int nrk = ctx->sp.nrk;
    // read the control block, set the step budget of this call
    CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    Ctrl& c = *ctx->h_ctrl;
    const long long big = (1LL << 62);
    long long stop_at = nsteps > 0 ? c.iter + nsteps : big;
    c.stop_at = stop_at;
    CK(cudaMemcpyAsync(&ctx->ctrl->stop_at, &c.stop_at, sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaEventRecord(ctx->ev_run0, ctx->stream));
    // dt of the current state for the first step; later steps get theirs
    // from the last stage of the step before
    launch_dt(ctx->mesh, ctx->phys, ctx->ctrl, ctx->sp, cur_prim(ctx), ctx->dt_partial, ctx->dt_bad, ctx->stream);
    launch_step_begin(ctx->ctrl, ctx->sp, ctx->dt_partial, ctx->dt_bad, ctx->nb_cells, ctx->stream);
    CK(cudaGetLastError());
    // each graph launch is followed by the end event and the reads of the
    // control block and the flags, so the synchronisation after the last
    // graph also ends the run
    unsigned f = 0;
    bool ended = false;
    while (!c.done && c.iter < stop_at) {
        long long remaining = stop_at - c.iter;
        int which = remaining >= kMany ? 1 : 0;
        int steps = which ? kMany : 1;
        int par = ctx->cur;
        if (!ctx->graph[par][which] &&
            (st = build_graph(ctx, par, steps, &ctx->graph[par][which], prof ? &ctx->prof_ev[par][which] : nullptr)))
            return st;
        long long iter0 = c.iter;
        CK(cudaGraphLaunch(ctx->graph[par][which], ctx->stream));
        CK(cudaEventRecord(ctx->ev_run1, ctx->stream));
        CK(cudaMemcpyAsync(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(&f, ctx->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        ended = true;
        // steps after a stop inside the graph do not run: the state is in
        // the buffer the last executed stage wrote
        long long ran = c.iter - iter0;
        if ((ran * nrk) & 1) ctx->cur ^= 1;
        if (ctx->sp.hist && (st = ccfd_history_drain(ctx))) return st;
        if (prof && (st = collect_profile(ctx, ctx->prof_ev[par][which], (size_t)ran * nrk))) return st;
        if (ran == 0) break;  // error in the first stage of the graph
    }
    if (!ended) {  // no graph ran: end after the time-step kernels
        CK(cudaEventRecord(ctx->ev_run1, ctx->stream));
        CK(cudaMemcpyAsync(&f, ctx->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    float run_ms = 0.0f;
    CK(cudaEventElapsedTime(&run_ms, ctx->ev_run0, ctx->ev_run1));
    if (report) {
        ccfd_fill_report(ctx, report);
        report->device_ms = run_ms;
    }
    return ccfd_status_from_flags(c.flags | f);
}

// Pressure coefficient along the wing (the CP part of calcCoef,
// src/analyze.c:296-367): for each wall face in calcCoef's order (pressure
// side by increasing x, then suction side) its point x, y and
// cp = (p_face - p_inf) / (rho_inf v_inf^2 / 2) of the last residual
// evaluation.  Arrays of at least *n entries; with x == NULL only the counts
// are returned.
extern "C" int ccfd_wall_cp(ccfd_ctx* ctx, double* x, double* y, double* cp, int* n, int* n_pressure) {
    if (!ctx || !ctx->uploaded || !n) return CCFD_ERR_ARG;
    if (!ctx->params.calc_wing || ctx->n_wall == 0) return CCFD_ERR_ARG;
    *n = ctx->n_wall;
    if (n_pressure) *n_pressure = ctx->n_wall_pressure;
    if (!x) return CCFD_OK;
    if (!y || !cp) return CCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    std::vector<double> pf(ctx->B + 1);
    std::vector<int> wl(ctx->n_wall);
    CK(cudaMemcpyAsync(pf.data(), ctx->ghost_pface, sizeof(double) * pf.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(wl.data(), ctx->wall_ghost, sizeof(int) * wl.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double pi = acos(-1.0);
    const double* ref = ctx->exact.ref_state[0];
    const double v = ref[1] / cos(ctx->exact.alpha * pi / 180.0);
    const double q_inf_q = 1.0 / (ref[0] * 0.5 * v * v);
    const double p_inf = ref[3];
    for (int k = 0; k < ctx->n_wall; ++k) {
        x[k] = ctx->wall_xy[2 * k];
        y[k] = ctx->wall_xy[2 * k + 1];
        cp[k] = (pf[wl[k]] - p_inf) * q_inf_q;
    }
    return CCFD_OK;
}

// The reference's CP files: <base>_CP_pressureSide.csv and
// <base>_CP_suctionSide.csv with rows x, y, phi = atan2(y, x), cp
extern "C" int ccfd_write_cp(ccfd_ctx* ctx, const char* base) {
    if (!base) return CCFD_ERR_ARG;
    int n = 0, np = 0;
    int st = ccfd_wall_cp(ctx, nullptr, nullptr, nullptr, &n, &np);
    if (st) return st;
    std::vector<double> x(n), y(n), cp(n);
    if ((st = ccfd_wall_cp(ctx, x.data(), y.data(), cp.data(), &n, &np))) return st;
    for (int side = 0; side < 2; ++side) {
        const char* tag = side ? "suctionSide" : "pressureSide";
        std::string name = std::string(base) + "_CP_" + tag + ".csv";
        FILE* f = fopen(name.c_str(), "w");
        if (!f) return CCFD_ERR_ARG;
        fprintf(f, "x, y, phi, CP_%s\n", tag);
        for (int k = side ? np : 0; k < (side ? n : np); ++k)
            fprintf(f, "%15.7f,%15.7f,%15.7f,%15.7f\n", x[k], y[k], atan2(y[k], x[k]), cp[k]);
        fclose(f);
    }
    // the gnuplot script of the CP files, written once (src/analyze.c:370-386)
    std::string dem = std::string(base) + "_CP.dem";
    FILE* d = fopen(dem.c_str(), "r");
    if (!d) {
        if (!(d = fopen(dem.c_str(), "w"))) return CCFD_ERR_ARG;
        fprintf(d, "unset key\n");
        fprintf(d, "set xlabel 'x'\n");
        fprintf(d, "set ylabel 'cp'\n");
        fprintf(d, "set yrange [*:*] reverse\n");
        fprintf(d, "plot '%s_CP_pressureSide.csv' using 1:4 w l lc rgb 'black', \\\n", base);
        fprintf(d, "     '%s_CP_suctionSide.csv' using 1:4 w l lc rgb 'black'\n", base);
        fprintf(d, "pause -1");
    }
    fclose(d);
    return CCFD_OK;
}

extern "C" int ccfd_clcd(ccfd_ctx* ctx, double* cl, double* cd) {
    if (!ctx || !ctx->uploaded || !cl || !cd) return CCFD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    if (!ctx->params.calc_wing || ctx->n_wall == 0) return CCFD_ERR_ARG;
    std::vector<double> pf(ctx->B + 1);
    std::vector<int> wl(ctx->n_wall);
    std::vector<double> wnl(3 * ctx->n_wall);
    CK(cudaMemcpyAsync(pf.data(), ctx->ghost_pface, sizeof(double) * pf.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(wl.data(), ctx->wall_ghost, sizeof(int) * wl.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(wnl.data(), ctx->wall_nl, sizeof(double) * wnl.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double l = 0.0, d = 0.0;
    for (int k = 0; k < ctx->n_wall; ++k) {
        double p0 = pf[wl[k]];
        l += wnl[3 * k + 1] * p0 * wnl[3 * k + 2];
        d += wnl[3 * k] * p0 * wnl[3 * k + 2];
    }
    l *= ctx->sp.q_inf_lq;
    d *= ctx->sp.q_inf_lq;
    *cl = l * ctx->sp.cos_a - d * ctx->sp.sin_a;
    *cd = d * ctx->sp.cos_a + l * ctx->sp.sin_a;
    return CCFD_OK;
}
