// Request loop with continuous batching (fx_server_*; no reference counterpart:
// FerriX solves one deck per process, src/main.rs:49-64).
//
// A server owns `slots` worker threads on one GPU, each with its own context
// (CUDA stream, PCG / multigrid workspaces). Submitted models (parsed on the
// host, not bound to a context) wait in a FIFO queue. A free slot admits the
// head request once the summed footprint estimate of the running requests plus
// the head's stays within the HBM budget (a request larger than the whole
// budget runs alone). The admitted model is bound to the slot's context,
// uploaded, solved (first *STATIC step, StaticStep::solve semantics) and its
// displacements copied to host memory; then all of its device memory is
// released and it is unbound again. Requests on different slots run
// concurrently on the device, on separate streams; each request's arithmetic is
// the same as alone (no shared reductions, fixed launch shapes), so its result
// does not depend on the mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.hpp"

using namespace fx;

namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
    int64_t ticket = 0;
    fx_model* model = nullptr;
    double bytes = 0.0;
    Clock::time_point t_submit, t_admit, t_done;
    double setup_ms = 0.0, solve_ms = 0.0, finish_ms = 0.0;
    bool done = false;
    int slot = -1;
    int status = FX_OK;
    std::string error;
    fx_step_stats stats{};
    std::vector<double> u;
};

}  // namespace

struct fx_server {
    int device = 0;
    int n_slots = 4;
    double budget = 0.0;
    fx_solve_opts opts{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<int64_t, Request*> reqs;
    double in_use = 0.0;
    int running = 0;
    int started = 0;  // workers whose context creation has finished (or failed)
    int preloaded = -2;  // kernels the slot contexts found loaded on the device (min over slots; -2: none yet)
    int reservation = 0;  // reserve_pool result for the budget
    double pool_bytes = 0.0;  // device pool reservation after the budget was reserved
    int64_t next_ticket = 1;
    bool stop = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> workers;
    std::string last_error;
};

namespace {

void release_device(fx_model* m) {
    if (!m->ctx) return;
    cudaStream_t s = m->ctx->stream;
    m->dev = ModelDev();  // every buffer is freed on the slot's stream
    m->state_ready = false;
    cudaStreamSynchronize(s);
    m->ctx = nullptr;
}

void worker(fx_server* srv, int slot) {
    fx_ctx* ctx = nullptr;
    const int rc = fx_ctx_create(srv->device, &ctx);
    {
        std::lock_guard<std::mutex> g(srv->mu);
        ++srv->started;
        if (rc == FX_OK) {
            const int pre = fx_ctx_preloaded_kernels(ctx);
            srv->preloaded = srv->preloaded == -2 ? pre : std::min(srv->preloaded, pre);
        }
        if (rc != FX_OK) {
            srv->last_error = "slot context creation failed";
            --srv->n_slots;
        }
    }
    srv->cv_done.notify_all();
    if (rc != FX_OK) {
        srv->cv_work.notify_all();
        return;
    }
    while (true) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            srv->cv_work.wait(lk, [&] {
                if (srv->stop) return true;
                if (srv->queue.empty()) return false;
                const double b = srv->queue.front()->bytes;
                return srv->running == 0 || srv->in_use + b <= srv->budget;
            });
            if (srv->stop) break;
            r = srv->queue.front();
            srv->queue.pop_front();
            srv->in_use += r->bytes;
            ++srv->running;
            r->slot = slot;
            r->t_admit = Clock::now();
        }
        fx_model* m = r->model;
        int st = FX_OK;
        std::string err;
        m->ctx = ctx;
        const Clock::time_point a = Clock::now();
        st = fx_state_initialize(m);
        const Clock::time_point b = Clock::now();
        if (st == FX_OK) st = fx_step_solve(m, 0, &srv->opts, &r->stats);
        const Clock::time_point c = Clock::now();
        if (st == FX_OK) {
            r->u.resize(3 * (size_t)m->dense.n_nodes);
            st = fx_state_get_displacements(m, r->u.data());
        }
        if (st != FX_OK) err = fx_ctx_last_error(ctx);
        release_device(m);
        r->setup_ms = ms_since(a, b);
        r->solve_ms = ms_since(b, c);
        r->finish_ms = ms_since(c, Clock::now());
        {
            std::lock_guard<std::mutex> g(srv->mu);
            r->status = st;
            r->error = err;
            r->t_done = Clock::now();
            r->done = true;
            srv->in_use -= r->bytes;
            --srv->running;
        }
        srv->cv_done.notify_all();
        srv->cv_work.notify_all();
    }
    fx_ctx_destroy(ctx);
}

}  // namespace

extern "C" {

void fx_default_server_opts(fx_server_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->device = 0;
    o->slots = 4;
    o->hbm_budget_bytes = 0.0;
    fx_default_solve_opts(&o->opts);
}

int fx_server_create(const fx_server_opts* opts, fx_server** out) {
    if (!out) return FX_INVALID_ARGUMENT;
    *out = nullptr;
    fx_server_opts o;
    if (opts) o = *opts;
    else fx_default_server_opts(&o);
    if (o.slots <= 0 || o.slots > 64) return FX_INVALID_ARGUMENT;
    if (cudaSetDevice(o.device) != cudaSuccess) return FX_CUDA;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return FX_CUDA;
    fx_server* s = new (std::nothrow) fx_server();
    if (!s) return FX_GENERIC;
    s->device = o.device;
    s->n_slots = o.slots;
    s->budget = o.hbm_budget_bytes > 0.0 ? o.hbm_budget_bytes : 0.7 * (double)free_b;
    s->opts = o.opts;
    // the budget is held in the device's memory pool from now on, so that requests
    // never grow the pool while other requests' kernels run
    cudaStream_t rs = nullptr;
    if (cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking) == cudaSuccess) {
        s->reservation = reserve_pool(o.device, rs, std::min(s->budget, 0.9 * (double)free_b));
        cudaStreamSynchronize(rs);
        cudaStreamDestroy(rs);
    } else {
        cudaGetLastError();
        s->reservation = -1;
    }
    s->pool_bytes = pool_reserved_bytes(o.device);
    for (int i = 0; i < o.slots; ++i) s->workers.emplace_back(worker, s, i);
    {  // every slot has its context (stream, workspaces) before the first request
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait_for(lk, std::chrono::seconds(60), [&] { return s->started == o.slots; });
    }
    *out = s;
    return FX_OK;
}

int fx_server_get_info(fx_server* s, fx_server_info* out) {
    if (!s || !out) return FX_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(s->mu);
    out->slots = s->n_slots;
    out->preloaded_kernels = s->preloaded == -2 ? -1 : s->preloaded;
    out->budget_bytes = s->budget;
    out->pool_reserved_bytes = s->pool_bytes;
    out->reservation = s->reservation;
    return FX_OK;
}

int fx_server_submit(fx_server* s, fx_model* m, int64_t* ticket) {
    if (!s || !m || !ticket) return FX_INVALID_ARGUMENT;
    if (m->ctx) return FX_INVALID_ARGUMENT;  // must be a host-only model (fx_model_from_inp with ctx NULL)
    Request* r = new (std::nothrow) Request();
    if (!r) return FX_GENERIC;
    try {
        ensure_dense(m);
    } catch (const Error& e) {
        delete r;
        std::lock_guard<std::mutex> g(s->mu);
        s->last_error = e.what();
        return e.status;
    }
    r->model = m;
    r->bytes = model_footprint(m->dense);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) {
            delete r;
            return FX_CANCELLED;
        }
        r->ticket = s->next_ticket++;
        s->reqs[r->ticket] = r;
        s->queue.push_back(r);
        *ticket = r->ticket;
    }
    s->cv_work.notify_all();
    return FX_OK;
}

int fx_server_wait(fx_server* s, int64_t ticket, double timeout_s, double* u, fx_request_result* res) {
    if (!s) return FX_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return FX_INVALID_ARGUMENT;
    Request* r = it->second;
    const auto pred = [&] { return r->done; };
    if (timeout_s < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return FX_TIMEOUT;
    s->reqs.erase(it);
    lk.unlock();
    if (u && r->status == FX_OK) std::memcpy(u, r->u.data(), r->u.size() * sizeof(double));
    if (res) {
        res->status = r->status;
        res->queue_ms = ms_since(r->t_submit, r->t_admit);
        res->service_ms = ms_since(r->t_admit, r->t_done);
        res->latency_ms = ms_since(r->t_submit, r->t_done);
        res->footprint_bytes = r->bytes;
        res->admit_at_ms = ms_since(s->t0, r->t_admit);
        res->done_at_ms = ms_since(s->t0, r->t_done);
        res->slot = r->slot;
        res->stats = r->stats;
        res->setup_ms = r->setup_ms;
        res->solve_ms = r->solve_ms;
        res->finish_ms = r->finish_ms;
        std::strncpy(res->error, r->error.c_str(), sizeof(res->error) - 1);
        res->error[sizeof(res->error) - 1] = 0;
    }
    const int st = r->status;
    delete r;
    return st;
}

void fx_server_destroy(fx_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& kv : s->reqs) {  // requests never admitted, or never collected
        Request* r = kv.second;
        if (!r->done && r->model) r->model->ctx = nullptr;
        delete r;
    }
    delete s;
}

}  // extern "C"
