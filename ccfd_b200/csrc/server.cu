// Request loop with continuous batching on one GPU.
//
// Requests (a case with a step budget) queue in arrival order.  Each call of
// ccfd_server_poll admits queued requests, first come first served, while
// their estimated device memory fits the budget and a slot is free; an
// admitted request is uploaded into its own context and joins the running
// batch at the next step boundary, so it overlaps on the device with the
// requests already running.  The batch then advances every running request;
// requests that stop (end time, convergence, step budget, error) leave the
// batch, their final state is copied to the host and their device memory is
// released for the next admissions.  No counterpart in the reference, which
// runs one case per process.
#include <cuda_runtime.h>
#include <string.h>

#include <chrono>
#include <deque>
#include <map>
#include <vector>

#include "ccfd_ctx.cuh"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

enum ReqState { QUEUED = 0, RUNNING = 1, DONE = 2 };

struct Request {
    long id = 0;
    const ccfd_case* c = nullptr;
    long nsteps = 0;
    size_t est = 0, bytes = 0;
    ccfd_ctx* ctx = nullptr;
    int state = QUEUED;
    int status = CCFD_OK;
    double t_submit = 0, t_admit = 0, t_done = 0;
    ccfd_report rep;
    std::vector<double> prim;  // final primitive state (reference cell order)
};

}  // namespace

struct ccfd_server {
    int device = 0;
    size_t budget = 0, used = 0;
    int max_running = 0;
    ccfd_batch* batch = nullptr;
    std::deque<long> queue;
    std::map<long, Request> reqs;
    long next_id = 1;
    int running = 0;
};

static size_t round_up(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int ccfd_estimate_device_bytes(const ccfd_params* p, const ccfd_mesh* m, size_t* bytes) {
    if (!p || !m || !bytes) return CCFD_ERR_ARG;
    const double N = (double)m->n_cells, H = (double)m->n_half_sides, F = (double)m->n_faces,
                 B = (double)m->n_bc;
    // mesh, state, tiles and per-tile scratch of the explicit path
    double b = 340.0 * N + 52.0 * H + 80.0 * F + 120.0 * B + (1 << 20);
    if (p->implicit) {
        const double K = (double)(p->n_kdim > 0 ? p->n_kdim : 1);
        // Krylov bases V (K+1) and Z (K), eight work vectors, D / D^-1 per
        // cell, off-diagonal blocks per half-side, colouring and level lists
        b += (64.0 * K + 32.0 + 8.0 * 32.0 + 256.0) * N + 144.0 * H + 16.0 * N;
    }
    *bytes = round_up((size_t)(1.2 * b));
    return CCFD_OK;
}

extern "C" int ccfd_device_bytes(ccfd_ctx* ctx, size_t* bytes) {
    if (!ctx || !bytes) return CCFD_ERR_ARG;
    *bytes = ctx->device_bytes;
    return CCFD_OK;
}

extern "C" int ccfd_server_create(int device, size_t hbm_budget_bytes, int max_running, ccfd_server** out) {
    if (!out || hbm_budget_bytes == 0 || max_running <= 0) return CCFD_ERR_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return CCFD_ERR_CUDA;
    ccfd_server* s = new ccfd_server();
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->max_running = max_running;
    int st = ccfd_batch_create(device, &s->batch);
    if (st) {
        delete s;
        return st;
    }
    *out = s;
    return CCFD_OK;
}

extern "C" void ccfd_server_destroy(ccfd_server* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    for (auto& kv : s->reqs)
        if (kv.second.ctx) ccfd_destroy(kv.second.ctx);
    ccfd_batch_destroy(s->batch);
    delete s;
}

// Queue a case (kept by the caller until its result is fetched) with a
// budget of nsteps time steps (<= 0: until the case stops by itself).
extern "C" int ccfd_server_submit(ccfd_server* s, const ccfd_case* c, long nsteps, long* id) {
    if (!s || !c || !id) return CCFD_ERR_ARG;
    Request r;
    r.id = s->next_id++;
    r.c = c;
    r.nsteps = nsteps;
    r.t_submit = now_s();
    int st = ccfd_estimate_device_bytes(&c->params, &c->mesh, &r.est);
    if (st) return st;
    if (r.est > s->budget) return CCFD_ERR_BUDGET;
    *id = r.id;
    s->reqs[r.id] = std::move(r);
    s->queue.push_back(*id);
    return CCFD_OK;
}

static void finish(ccfd_server* s, Request& r, int status) {
    r.status = status;
    r.state = DONE;
    r.t_done = now_s();
    if (r.ctx) {
        r.prim.resize(4 * (size_t)r.c->mesh.n_cells);
        int gs = r.ctx->uploaded ? ccfd_get_state(r.ctx, r.prim.data(), CCFD_PRIMITIVE) : CCFD_ERR_ARG;
        if (gs) r.prim.clear();
        if (!r.status) r.status = gs;
        ccfd_destroy(r.ctx);
        r.ctx = nullptr;
        s->used -= r.bytes;
        s->running--;
    }
}

static int admit(ccfd_server* s, Request& r) {
    const ccfd_case* c = r.c;
    r.t_admit = now_s();
    r.state = RUNNING;
    int st = ccfd_create(&c->params, &r.ctx);
    if (st) {
        r.ctx = nullptr;
        return st;
    }
    s->running++;
    st = ccfd_upload_case(r.ctx, &c->mesh, c->bc_table, c->n_bc_table, &c->exact, 1);
    if (!st) st = ccfd_set_state(r.ctx, c->prim0, CCFD_PRIMITIVE);
    if (!st) st = ccfd_batch_add(s->batch, r.ctx, r.nsteps);
    r.bytes = r.ctx->device_bytes;
    s->used += r.bytes;
    return st;
}

// Admit what fits, advance the running requests by up to `steps` steps,
// retire the ones that stopped.  Counts of queued / running / finished
// (not yet fetched) requests are returned.
extern "C" int ccfd_server_poll(ccfd_server* s, int steps, int* n_queued, int* n_running, int* n_done) {
    if (!s || steps <= 0) return CCFD_ERR_ARG;
    if (cudaSetDevice(s->device) != cudaSuccess) return CCFD_ERR_CUDA;
    while (!s->queue.empty() && s->running < s->max_running) {
        Request& r = s->reqs[s->queue.front()];
        if (s->used + r.est > s->budget) break;  // first come, first served
        s->queue.pop_front();
        int st = admit(s, r);
        if (st) finish(s, r, st);
    }
    int n_batch = 0;
    int st = ccfd_batch_size(s->batch, &n_batch);
    if (st) return st;
    if (n_batch > 0) {
        int left = 0;
        if ((st = ccfd_batch_step(s->batch, steps, &left))) return st;
        for (auto& kv : s->reqs) {
            Request& r = kv.second;
            if (r.state != RUNNING) continue;
            const ccfd::Ctrl& h = *r.ctx->h_ctrl;
            if (!h.done && h.iter < h.stop_at) continue;
            if ((st = ccfd_batch_report(s->batch, r.ctx, &r.rep))) return st;
            if ((st = ccfd_batch_remove(s->batch, r.ctx))) return st;
            finish(s, r, r.rep.status);
        }
    }
    int q = (int)s->queue.size(), d = 0;
    for (auto& kv : s->reqs) d += kv.second.state == DONE;
    if (n_queued) *n_queued = q;
    if (n_running) *n_running = s->running;
    if (n_done) *n_done = d;
    return CCFD_OK;
}

// Result of a finished request: report, final primitive state (n_cells x 4,
// reference order; may be NULL) and host timestamps in seconds of a
// monotonic clock (submit, admit, done; may be NULL).  The request is
// forgotten afterwards.  CCFD_ERR_BUSY while it is queued or running.
extern "C" int ccfd_server_result(ccfd_server* s, long id, ccfd_report* rep, double* prim,
                                  double times[3]) {
    if (!s) return CCFD_ERR_ARG;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return CCFD_ERR_ARG;
    Request& r = it->second;
    if (r.state != DONE) return CCFD_ERR_BUSY;
    if (rep) {
        *rep = r.rep;
        rep->status = r.status;
    }
    if (prim && !r.prim.empty()) memcpy(prim, r.prim.data(), sizeof(double) * r.prim.size());
    if (times) {
        times[0] = r.t_submit;
        times[1] = r.t_admit;
        times[2] = r.t_done;
    }
    int st = r.status;
    s->reqs.erase(it);
    return st;
}

extern "C" int ccfd_server_memory(ccfd_server* s, size_t* used, size_t* budget) {
    if (!s) return CCFD_ERR_ARG;
    if (used) *used = s->used;
    if (budget) *budget = s->budget;
    return CCFD_OK;
}
