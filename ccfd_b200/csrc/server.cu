// Request loop with continuous batching on one GPU.
//
// Requests (a case with a step budget) queue in arrival order.  Worker
// threads admit them, first come first served, while their estimated device
// memory fits the budget and a slot is free: it uploads each admitted case
// into its own context (host-side mesh preparation and host-to-device copies
// on the context's stream) while the GPU keeps stepping the running
// requests.  Each call of ccfd_server_poll moves the uploaded requests into
// the running batch at the step boundary, so they overlap on the device with
// the requests already running, advances the batch, and retires the
// requests that stopped (end time, convergence, step budget, error): the
// workers copy their final state to the host and release their device
// memory for the next admissions, again while the GPU keeps stepping.  No counterpart in the reference, which runs one case
// per process.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "ccfd_ctx.cuh"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

enum ReqState { QUEUED = 0, UPLOADING, READY, RUNNING, RETIRING, DONE };

struct Request {
    long id = 0;
    const ccfd_case* c = nullptr;
    long nsteps = 0;
    size_t est = 0, bytes = 0;  // reserved estimate, then the context's actual bytes
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
    size_t budget = 0, used = 0;  // used: reserved / held device bytes
    int max_running = 0;
    int slots = 0;                // requests uploading, ready or running
    ccfd_batch* batch = nullptr;
    std::deque<long> queue;
    std::map<long, Request> reqs;
    std::vector<long> ready;      // uploaded, waiting for the next step boundary
    std::deque<long> retiring;    // left the batch, state to copy back and memory to release
    long next_id = 1;
    double t_admit = 0, t_step = 0, t_retire = 0;  // host seconds per phase
    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    std::vector<std::thread> workers;  // uploads run in parallel, one request each
};

static size_t round_up(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int ccfd_estimate_device_bytes(const ccfd_params* p, const ccfd_mesh* m, size_t* bytes) {
    if (!p || !m || !bytes) return CCFD_ERR_ARG;
    const double N = (double)m->n_cells, H = (double)m->n_half_sides, F = (double)m->n_faces,
                 B = (double)m->n_bc;
    // mesh, state, tiles and per-tile scratch of the explicit path
    double b = 412.0 * N + 52.0 * H + 80.0 * F + 120.0 * B + (1 << 20);
    if (p->source_func) b += 32.0 * N;
    if (p->implicit) {
        const double K = (double)(p->n_kdim > 0 ? p->n_kdim : 1);
        // Krylov bases V (K+1) and Z (K), eight work vectors, D / D^-1 per
        // cell, off-diagonal blocks per half-side, colouring and sweep lists
        b += (64.0 * K + 32.0 + 8.0 * 32.0 + 256.0 + 96.0) * N + 144.0 * H;
    }
    *bytes = round_up((size_t)(1.2 * b));
    return CCFD_OK;
}

extern "C" int ccfd_device_bytes(ccfd_ctx* ctx, size_t* bytes) {
    if (!ctx || !bytes) return CCFD_ERR_ARG;
    *bytes = ctx->device_bytes;
    return CCFD_OK;
}

// upload one admitted request (worker thread, server lock not held)
static int upload(Request& r) {
    const ccfd_case* c = r.c;
    int st = ccfd_create(&c->params, &r.ctx);
    if (st) {
        r.ctx = nullptr;
        return st;
    }
    st = ccfd_upload_case(r.ctx, &c->mesh, c->bc_table, c->n_bc_table, &c->exact, 1);
    if (!st) st = ccfd_set_state(r.ctx, c->prim0, CCFD_PRIMITIVE);
    return st;
}

static void worker_main(ccfd_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv.wait(lk, [s] {
            if (s->stop || !s->retiring.empty()) return true;
            if (s->queue.empty() || s->slots >= s->max_running) return false;
            return s->used + s->reqs[s->queue.front()].est <= s->budget;
        });
        if (s->stop) return;
        if (!s->retiring.empty()) {
            // retire first: it frees memory for the next admissions
            long rid = s->retiring.front();
            s->retiring.pop_front();
            Request& q = s->reqs[rid];
            lk.unlock();
            double t0 = now_s();
            q.prim.resize(4 * (size_t)q.c->mesh.n_cells);
            int gs = ccfd_get_state(q.ctx, q.prim.data(), CCFD_PRIMITIVE);
            if (gs) q.prim.clear();
            ccfd_destroy(q.ctx);
            double t1 = now_s();
            lk.lock();
            s->t_retire += t1 - t0;
            if (!q.status) q.status = gs;
            q.ctx = nullptr;
            s->used -= q.bytes;
            s->slots--;
            q.state = DONE;
            q.t_done = now_s();
            s->cv.notify_all();
            continue;
        }
        long id = s->queue.front();
        s->queue.pop_front();
        Request& r = s->reqs[id];  // std::map references stay valid
        r.state = UPLOADING;
        r.t_admit = now_s();
        s->used += r.est;
        s->slots++;
        lk.unlock();
        double t0 = now_s();
        int st = upload(r);
        double t1 = now_s();
        lk.lock();
        s->t_admit += t1 - t0;
        if (st) {
            if (r.ctx) ccfd_destroy(r.ctx);
            r.ctx = nullptr;
            s->used -= r.est;
            s->slots--;
            r.status = st;
            r.state = DONE;
            r.t_done = now_s();
        } else {
            // hold the actual bytes from now on (never more than the estimate)
            r.bytes = r.ctx->device_bytes;
            s->used -= r.est;
            s->used += r.bytes;
            r.state = READY;
            s->ready.push_back(id);
        }
        s->cv.notify_all();
    }
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
    unsigned hw = std::thread::hardware_concurrency();
    int nw = (int)std::max(1u, std::min(4u, hw / 2));
    for (int k = 0; k < nw; ++k) s->workers.emplace_back(worker_main, s);
    *out = s;
    return CCFD_OK;
}

extern "C" void ccfd_server_destroy(ccfd_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (auto& w : s->workers) w.join();
    cudaSetDevice(s->device);
    ccfd_batch_destroy(s->batch);
    for (auto& kv : s->reqs)
        if (kv.second.ctx) ccfd_destroy(kv.second.ctx);
    delete s;
}

// Queue a case (kept by the caller until its result is fetched) with a
// budget of nsteps time steps (<= 0: until the case stops by itself).
extern "C" int ccfd_server_submit(ccfd_server* s, const ccfd_case* c, long nsteps, long* id) {
    if (!s || !c || !id) return CCFD_ERR_ARG;
    Request r;
    r.c = c;
    r.nsteps = nsteps;
    r.t_submit = now_s();
    int st = ccfd_estimate_device_bytes(&c->params, &c->mesh, &r.est);
    if (st) return st;
    if (r.est > s->budget) return CCFD_ERR_BUDGET;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r.id = s->next_id++;
        *id = r.id;
        s->reqs[r.id] = std::move(r);
        s->queue.push_back(*id);
    }
    s->cv.notify_all();
    return CCFD_OK;
}

// hand a request that left the batch to the workers, which copy its state
// back and release its context while the GPU keeps stepping (lock held)
static void retire(ccfd_server* s, Request& r, int status) {
    r.status = status;
    r.state = RETIRING;
    s->retiring.push_back(r.id);
    s->cv.notify_all();
}

// Move uploaded requests into the batch, advance the running requests by up
// to `steps` steps, retire the ones that stopped.  Counts of queued (incl.
// uploading) / running / finished-not-fetched requests are returned.
extern "C" int ccfd_server_poll(ccfd_server* s, int steps, int* n_queued, int* n_running, int* n_done) {
    if (!s || steps <= 0) return CCFD_ERR_ARG;
    if (cudaSetDevice(s->device) != cudaSuccess) return CCFD_ERR_CUDA;
    std::vector<long> joining;
    int n_batch = 0, st;
    if ((st = ccfd_batch_size(s->batch, &n_batch))) return st;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        // nothing to step yet: wait briefly for an upload to complete
        if (n_batch == 0 && s->ready.empty() && s->slots > 0)
            s->cv.wait_for(lk, std::chrono::milliseconds(20), [s] { return !s->ready.empty(); });
        joining.swap(s->ready);
    }
    for (long id : joining) {
        Request* r;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r = &s->reqs[id];
        }
        st = ccfd_batch_add(s->batch, r->ctx, r->nsteps);
        std::lock_guard<std::mutex> lk(s->mu);
        if (st) {
            retire(s, *r, st);
            s->cv.notify_all();
        } else {
            r->state = RUNNING;
        }
    }
    if ((st = ccfd_batch_size(s->batch, &n_batch))) return st;
    if (n_batch > 0) {
        double t1 = now_s();
        int left = 0;
        if ((st = ccfd_batch_step(s->batch, steps, &left))) return st;
        double t2 = now_s();
        std::vector<Request*> stopped;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->t_step += t2 - t1;
            for (auto& kv : s->reqs) {
                Request& r = kv.second;
                if (r.state != RUNNING) continue;
                const ccfd::Ctrl& h = *r.ctx->h_ctrl;
                if (h.done || h.iter >= h.stop_at) stopped.push_back(&r);
            }
        }
        for (Request* r : stopped) {
            if ((st = ccfd_batch_report(s->batch, r->ctx, &r->rep))) return st;
            if ((st = ccfd_batch_remove(s->batch, r->ctx))) return st;
            std::lock_guard<std::mutex> lk(s->mu);
            retire(s, *r, r->rep.status);
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->cv.notify_all();
    }
    std::lock_guard<std::mutex> lk(s->mu);
    int q = 0, run = 0, d = 0;
    for (auto& kv : s->reqs) {
        int stt = kv.second.state;
        q += stt == QUEUED || stt == UPLOADING || stt == READY;
        run += stt == RUNNING || stt == RETIRING;
        d += stt == DONE;
    }
    if (n_queued) *n_queued = q;
    if (n_running) *n_running = run;
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
    std::lock_guard<std::mutex> lk(s->mu);
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

// host seconds spent so far uploading (worker thread), stepping and retiring
extern "C" int ccfd_server_times(ccfd_server* s, double out[3]) {
    if (!s || !out) return CCFD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    out[0] = s->t_admit;
    out[1] = s->t_step;
    out[2] = s->t_retire;
    return CCFD_OK;
}

extern "C" int ccfd_server_memory(ccfd_server* s, size_t* used, size_t* budget) {
    if (!s) return CCFD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (used) *used = s->used;
    if (budget) *budget = s->budget;
    return CCFD_OK;
}
