// Batched stepping of many solver instances on one GPU.
//
// Every member is an ordinary context (its own mesh, state, control block and
// scratch, all resident in device memory).  Explicit members are advanced
// together: each Runge-Kutta stage is one launch per kernel variant (flux,
// order, equations, precision) over the concatenated tiles of all members of
// that variant, so small and uneven meshes fill the GPU together.  Each
// member keeps its own time step, CFL, stop tests and convergence flags in
// its control block; a member that stops simply returns from its CTAs.  A
// CUDA graph holds a fixed number of batched steps and is rebuilt only when
// the membership changes.  Implicit members are advanced by the batched
// Newton-Krylov driver (implicit_batch in implicit.cu).
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "ccfd_ctx.cuh"

using namespace ccfd;

namespace {

struct VariantGroup {
    int flux, order, ns, fp32;
    std::vector<int> members;  // indices into ccfd_batch::inst
    int n_tiles = 0, smem_bytes = 0;
    StageLaunch* d_recs = nullptr;
    int2* d_tmap = nullptr;
    int* d_ctr = nullptr;  // tile claim counters of the group's launches
};

__global__ void k_gather_ctrl(const Ctrl* const* __restrict__ src, Ctrl* __restrict__ dst, int n) {
    int i = blockIdx.x;
    if (i >= n) return;
    const int* s = reinterpret_cast<const int*>(src[i]);
    int* d = reinterpret_cast<int*>(dst + i);
    for (int k = threadIdx.x; k < (int)(sizeof(Ctrl) / sizeof(int)); k += blockDim.x) d[k] = s[k];
}

}  // namespace

struct ccfd_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    int last_cuda_error = 0;
    std::vector<ccfd_ctx*> inst;
    std::vector<VariantGroup> groups;
    bool dirty = true;
    int max_nrk = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // [0]: one step, [1]: kMany steps
    const Ctrl** d_ctrl_ptr = nullptr;
    Ctrl* d_ctrl = nullptr;
    Ctrl* h_ctrl = nullptr;
    int ctrl_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double device_ms = 0.0;
    // kernel variants and the implicit members run on streams of their own
    // so that their launches overlap on the device (fork / join by events)
    std::vector<cudaStream_t> gstream;
    std::vector<cudaEvent_t> gdone;
    cudaEvent_t fork = nullptr;
    cudaStream_t istream = nullptr;
    cudaEvent_t idone = nullptr;
};

#define CKB(x)                              \
    do {                                    \
        cudaError_t e_ = (x);               \
        if (e_ != cudaSuccess) {            \
            b->last_cuda_error = (int)e_;   \
            return CCFD_ERR_CUDA;           \
        }                                   \
    } while (0)

static constexpr int kMany = 16;

static void drop_group_memory(ccfd_batch* b) {
    for (auto& g : b->groups) {
        if (g.d_recs) cudaFreeAsync(g.d_recs, b->stream);
        if (g.d_tmap) cudaFreeAsync(g.d_tmap, b->stream);
        if (g.d_ctr) cudaFreeAsync(g.d_ctr, b->stream);
    }
    b->groups.clear();
    for (auto& g : b->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// launch records of member ctx: [parity][stage] for the RK stages
static void member_records(ccfd_ctx* ctx, StageLaunch* out) {
    const StepParams& sp = ctx->sp;
    for (int par = 0; par < 2; ++par)
        for (int s = 0; s < kBatchStages; ++s) {
            StageLaunch& L = out[par * kBatchStages + s];
            ccfd_fill_stage(ctx, L);
            L.ctrl = ctx->ctrl;
            if (s >= sp.nrk) {
                L.mode = -1;
                continue;
            }
            int pin = par ^ (s & 1);
            L.mode = 1;
            L.a_time = sp.rk[s];
            L.rk = sp.rk[s + 1];
            L.prim_in = ctx->prim_buf[pin];
            L.prim_out = ctx->prim_buf[pin ^ 1];
            L.cons0 = ctx->cons0;
            L.last_stage = s == sp.nrk - 1;
            L.res_partial = L.last_stage ? ctx->res_partial : nullptr;
            L.dt_partial = L.last_stage ? ctx->dt_partial : nullptr;
            L.dt_bad = ctx->dt_bad;
        }
}

// group the explicit members by kernel variant, upload their launch records
// and tile maps
static int rebuild(ccfd_batch* b) {
    drop_group_memory(b);
    std::map<std::tuple<int, int, int, int>, int> key_of;
    b->max_nrk = 0;
    for (int i = 0; i < (int)b->inst.size(); ++i) {
        ccfd_ctx* c = b->inst[i];
        if (c->params.implicit) continue;
        StageLaunch probe;
        ccfd_fill_stage(c, probe);
        auto key = std::make_tuple(probe.flux_id, probe.order, probe.ns, probe.fp32);
        auto it = key_of.find(key);
        if (it == key_of.end()) {
            VariantGroup g;
            g.flux = probe.flux_id;
            g.order = probe.order;
            g.ns = probe.ns;
            g.fp32 = probe.fp32;
            key_of[key] = (int)b->groups.size();
            b->groups.push_back(g);
            it = key_of.find(key);
        }
        b->groups[it->second].members.push_back(i);
        b->max_nrk = std::max(b->max_nrk, c->sp.nrk);
    }
    for (auto& g : b->groups) {
        std::vector<StageLaunch> recs(g.members.size() * 2 * kBatchStages);
        std::vector<int2> tmap;
        TileDev big;
        memset(&big, 0, sizeof(big));
        for (size_t k = 0; k < g.members.size(); ++k) {
            ccfd_ctx* c = b->inst[g.members[k]];
            member_records(c, &recs[k * 2 * kBatchStages]);
            for (int t = 0; t < c->tiles.n_tiles; ++t) tmap.push_back(make_int2((int)k, t));
            big.max_e = std::max(big.max_e, c->tiles.max_e);
            big.max_g = std::max(big.max_g, c->tiles.max_g);
            big.max_hs = std::max(big.max_hs, c->tiles.max_hs);
            big.max_f = std::max(big.max_f, c->tiles.max_f);
        }
        g.n_tiles = (int)tmap.size();
        g.smem_bytes = stage_smem_bytes(big, g.fp32);
        CKB(ccfd_malloc_async((void**)&g.d_recs, sizeof(StageLaunch) * recs.size(), b->stream));
        CKB(ccfd_malloc_async((void**)&g.d_tmap, sizeof(int2) * tmap.size(), b->stream));
        CKB(ccfd_malloc_async((void**)&g.d_ctr, sizeof(int) * 2, b->stream));
        CKB(cudaMemsetAsync(g.d_ctr, 0, sizeof(int) * 2, b->stream));
        CKB(cudaMemcpyAsync(g.d_recs, recs.data(), sizeof(StageLaunch) * recs.size(), cudaMemcpyHostToDevice,
                            b->stream));
        CKB(cudaMemcpyAsync(g.d_tmap, tmap.data(), sizeof(int2) * tmap.size(), cudaMemcpyHostToDevice,
                            b->stream));
    }
    while (b->gstream.size() < b->groups.size()) {
        cudaStream_t gs;
        cudaEvent_t ge;
        CKB(cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking));
        CKB(cudaEventCreateWithFlags(&ge, cudaEventDisableTiming));
        b->gstream.push_back(gs);
        b->gdone.push_back(ge);
    }
    // control-block gather list
    const int n = (int)b->inst.size();
    if (n > b->ctrl_cap) {
        if (b->d_ctrl_ptr) cudaFree((void*)b->d_ctrl_ptr);
        if (b->d_ctrl) cudaFree(b->d_ctrl);
        if (b->h_ctrl) cudaFreeHost(b->h_ctrl);
        b->ctrl_cap = std::max(n, 2 * b->ctrl_cap);
        CKB(cudaMalloc((void**)&b->d_ctrl_ptr, sizeof(Ctrl*) * b->ctrl_cap));
        CKB(cudaMalloc(&b->d_ctrl, sizeof(Ctrl) * b->ctrl_cap));
        CKB(cudaMallocHost(&b->h_ctrl, sizeof(Ctrl) * b->ctrl_cap));
    }
    std::vector<const Ctrl*> ptrs(n);
    for (int i = 0; i < n; ++i) ptrs[i] = b->inst[i]->ctrl;
    if (n) CKB(cudaMemcpyAsync((void*)b->d_ctrl_ptr, ptrs.data(), sizeof(Ctrl*) * n, cudaMemcpyHostToDevice, b->stream));
    CKB(cudaStreamSynchronize(b->stream));
    b->dirty = false;
    return CCFD_OK;
}

// `steps` batched steps, each variant on its own stream after the fork
// event of the batch stream, joined back into the batch stream
static void launch_steps(ccfd_batch* b, int steps) {
    cudaEventRecord(b->fork, b->stream);
    for (size_t k = 0; k < b->groups.size(); ++k) {
        VariantGroup& g = b->groups[k];
        cudaStream_t gs = b->gstream[k];
        cudaStreamWaitEvent(gs, b->fork, 0);
        for (int i = 0; i < steps; ++i)
            for (int s = 0; s < b->max_nrk; ++s) {
                BatchLaunch B;
                B.recs = g.d_recs;
                B.tmap = g.d_tmap;
                B.ctr = g.d_ctr;
                B.n_tiles = g.n_tiles;
                B.smem_bytes = g.smem_bytes;
                B.rk_mode = 1;
                B.stage = s;
                B.flux_id = g.flux;
                B.order = g.order;
                B.ns = g.ns;
                B.fp32 = g.fp32;
                launch_stage_batch(B, gs);
            }
        cudaEventRecord(b->gdone[k], gs);
        cudaStreamWaitEvent(b->stream, b->gdone[k], 0);
    }
}

// CUDA graphs of one and of kMany batched steps (captured once the
// membership has stayed the same for a call; until then the steps are
// launched directly, which costs less than a capture per change)
static int capture_graphs(ccfd_batch* b) {
    for (int w = 0; w < 2; ++w) {
        const int steps = w ? kMany : 1;
        cudaGraph_t gr;
        CKB(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        launch_steps(b, steps);
        cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
        if (e != cudaSuccess) {
            b->last_cuda_error = (int)e;
            return CCFD_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&b->graph[w], gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) {
            b->last_cuda_error = (int)e;
            return CCFD_ERR_CUDA;
        }
    }
    return CCFD_OK;
}

// copy every member's control block to the host (one gather kernel, one copy)
static int pull_ctrl(ccfd_batch* b) {
    const int n = (int)b->inst.size();
    if (!n) return CCFD_OK;
    k_gather_ctrl<<<n, 64, 0, b->stream>>>(b->d_ctrl_ptr, b->d_ctrl, n);
    CKB(cudaGetLastError());
    CKB(cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, sizeof(Ctrl) * n, cudaMemcpyDeviceToHost, b->stream));
    CKB(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < n; ++i) *b->inst[i]->h_ctrl = b->h_ctrl[i];
    return CCFD_OK;
}

static int find_member(ccfd_batch* b, ccfd_ctx* ctx) {
    for (int i = 0; i < (int)b->inst.size(); ++i)
        if (b->inst[i] == ctx) return i;
    return -1;
}

extern "C" int ccfd_batch_create(int device, ccfd_batch** out) {
    if (!out) return CCFD_ERR_ARG;
    *out = nullptr;
    ccfd_batch* b = new ccfd_batch();
    b->device = device;
    CKB(cudaSetDevice(device));
    CKB(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CKB(cudaEventCreate(&b->ev0));
    CKB(cudaEventCreate(&b->ev1));
    CKB(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    CKB(cudaEventCreateWithFlags(&b->idone, cudaEventDisableTiming));
    CKB(cudaStreamCreateWithFlags(&b->istream, cudaStreamNonBlocking));
    *out = b;
    return CCFD_OK;
}

void ccfd_implicit_batch_release(ccfd_batch* b);

extern "C" void ccfd_batch_destroy(ccfd_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    for (ccfd_ctx* c : b->inst) {
        cudaMemcpy(c->h_ctrl, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost);
        c->cur = c->h_ctrl->par;
        c->batch = nullptr;
    }
    ccfd_implicit_batch_release(b);
    drop_group_memory(b);
    if (b->d_ctrl_ptr) cudaFree((void*)b->d_ctrl_ptr);
    if (b->d_ctrl) cudaFree(b->d_ctrl);
    if (b->h_ctrl) cudaFreeHost(b->h_ctrl);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    for (size_t k = 0; k < b->gstream.size(); ++k) {
        cudaStreamDestroy(b->gstream[k]);
        cudaEventDestroy(b->gdone[k]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->idone) cudaEventDestroy(b->idone);
    if (b->istream) cudaStreamDestroy(b->istream);
    cudaStreamDestroy(b->stream);
    delete b;
}

int ccfd_implicit_batch_join(ccfd_batch* b, ccfd_ctx* ctx);
int ccfd_implicit_batch_leave(ccfd_batch* b, ccfd_ctx* ctx);
void ccfd_implicit_batch_release(ccfd_batch* b);

extern "C" int ccfd_batch_add(ccfd_batch* b, ccfd_ctx* ctx, long nsteps) {
    if (!b || !ctx || !ctx->uploaded || ctx->batch || ctx->device != b->device) return CCFD_ERR_ARG;
    CKB(cudaSetDevice(b->device));
    CKB(cudaStreamSynchronize(ctx->stream));
    Ctrl* h = ctx->h_ctrl;
    CKB(cudaMemcpy(h, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    h->stop_at = nsteps > 0 ? h->iter + nsteps : (1LL << 62);
    h->par = ctx->cur;
    CKB(cudaMemcpy(ctx->ctrl, h, sizeof(Ctrl), cudaMemcpyHostToDevice));
    if (ctx->params.implicit) {
        int st = ccfd_implicit_batch_join(b, ctx);
        if (st) return st;
    } else {
        // time step of the current state for the member's first step; later
        // steps take theirs from the last stage of the step before
        launch_dt(ctx->mesh, ctx->phys, ctx->ctrl, ctx->sp, ctx->prim_buf[ctx->cur], ctx->dt_partial,
                  ctx->dt_bad, b->stream);
        launch_step_begin(ctx->ctrl, ctx->sp, ctx->dt_partial, ctx->dt_bad, ctx->nb_cells, b->stream);
        CKB(cudaGetLastError());
        CKB(cudaStreamSynchronize(b->stream));
    }
    ctx->batch = b;
    b->inst.push_back(ctx);
    b->dirty = true;
    return CCFD_OK;
}

extern "C" int ccfd_batch_remove(ccfd_batch* b, ccfd_ctx* ctx) {
    if (!b || !ctx) return CCFD_ERR_ARG;
    int i = find_member(b, ctx);
    if (i < 0) return CCFD_ERR_ARG;
    CKB(cudaSetDevice(b->device));
    CKB(cudaStreamSynchronize(b->stream));
    CKB(cudaMemcpy(ctx->h_ctrl, ctx->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    if (ctx->params.implicit) {
        int st = ccfd_implicit_batch_leave(b, ctx);
        if (st) return st;
    } else {
        ctx->cur = ctx->h_ctrl->par;
    }
    ctx->batch = nullptr;
    b->inst.erase(b->inst.begin() + i);
    b->dirty = true;
    return CCFD_OK;
}

int ccfd_implicit_batch_steps(ccfd_batch* b, const std::vector<ccfd_ctx*>& members, int steps);

// Advance every running member by up to `steps` time steps.  Members stop
// on their own criteria (tEnd, convergence, maxIter, step budget, errors).
extern "C" int ccfd_batch_step(ccfd_batch* b, int steps, int* n_running) {
    if (!b || steps <= 0) return CCFD_ERR_ARG;
    // a member's history ring must hold the rows of one call
    for (ccfd_ctx* c : b->inst)
        if (c->sp.hist && steps > c->sp.hist_cap) return CCFD_ERR_ARG;
    CKB(cudaSetDevice(b->device));
    int st;
    bool direct = false;
    if (b->dirty) {
        if ((st = rebuild(b))) return st;
        direct = true;
    } else if (!b->groups.empty() && !b->graph[0] && (st = capture_graphs(b))) {
        return st;
    }
    CKB(cudaEventRecord(b->ev0, b->stream));
    std::vector<ccfd_ctx*> imp;
    for (ccfd_ctx* c : b->inst)
        if (c->params.implicit) imp.push_back(c);
    // explicit members: queued asynchronously first ...
    bool any_explicit = !b->groups.empty();
    if (any_explicit && direct) {
        launch_steps(b, steps);
    } else if (any_explicit) {
        for (int left = steps; left > 0;) {
            int w = left >= kMany ? 1 : 0;
            CKB(cudaGraphLaunch(b->graph[w], b->stream));
            left -= w ? kMany : 1;
        }
    }
    CKB(cudaGetLastError());
    // ... then the implicit members are driven on their own stream while the
    // explicit launches run
    if (!imp.empty()) {
        CKB(cudaStreamWaitEvent(b->istream, b->ev0, 0));
        if ((st = ccfd_implicit_batch_steps(b, imp, steps))) return st;
        CKB(cudaEventRecord(b->idone, b->istream));
        CKB(cudaStreamWaitEvent(b->stream, b->idone, 0));
    }
    CKB(cudaEventRecord(b->ev1, b->stream));
    if ((st = pull_ctrl(b))) return st;
    for (ccfd_ctx* c : b->inst)
        if (c->sp.hist && (st = ccfd_history_drain(c))) return st;
    float ms = 0.0f;
    CKB(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->device_ms += ms;
    int running = 0;
    for (ccfd_ctx* c : b->inst) {
        const Ctrl& h = *c->h_ctrl;
        if (!h.done && h.iter < h.stop_at) ++running;
    }
    if (n_running) *n_running = running;
    return CCFD_OK;
}

extern "C" int ccfd_batch_report(ccfd_batch* b, ccfd_ctx* ctx, ccfd_report* r) {
    if (!b || !ctx || !r || find_member(b, ctx) < 0) return CCFD_ERR_ARG;
    ccfd_fill_report(ctx, r);
    r->device_ms = b->device_ms;
    return CCFD_OK;
}

extern "C" int ccfd_batch_size(ccfd_batch* b, int* n) {
    if (!b || !n) return CCFD_ERR_ARG;
    *n = (int)b->inst.size();
    return CCFD_OK;
}

cudaStream_t ccfd_batch_stream(ccfd_batch* b) { return b->stream; }
cudaStream_t ccfd_batch_implicit_stream(ccfd_batch* b) { return b->istream; }
