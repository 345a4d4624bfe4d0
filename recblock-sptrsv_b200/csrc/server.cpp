// server.cpp -- request loop over device-resident factors (no counterpart in
// the reference, which runs one solve per process).
//
// Factors: each admitted factor keeps its plan (permutation, blocks, kernel
// plan, captured block walks) on the device, with work vectors reserved at
// admission for the server's batch width, so no solve allocates or frees
// device memory while requests are served.  Admission is charged against the
// HBM budget: the plan, its work vectors and, once the factor receives its
// first host-array request, the staging buffers for host arrays.
//
// Requests: host arrays (rbs_server_submit) or device arrays
// (rbs_server_submit_device), n x k column-major, one precision each.  They
// queue per factor.
//
// Dispatch: ONE dispatcher thread issues every CUDA call of the server.  Each
// factor has its own stream and completion event and moves through
//   idle -> (batch started) -> refinement step in flight -> ... -> final
//   copies in flight -> idle.
// A factor that is idle and has queued requests takes all queued requests
// of the first request's precision that fit the batch width (FIFO) and runs
// them as ONE multi-RHS solve: the requests' columns are read in place
// through a device table of column pointers, with no staging copy for device
// requests.  The dispatcher then polls the events of all busy factors and
// advances whichever finished: mixed-precision refinement decides on the
// host, per factor, whether another correction is needed, without holding up
// the other factors.  So requests that arrive while a batch runs join that
// factor's next batch (continuous batching within a factor) and the batches
// of all factors overlap on the device (batching across factors).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "rbs.h"
#include "rbs_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    const double *b = nullptr;
    double *x = nullptr;
    bool device = false;
    int k = 0, prec = 0;
    Clock::time_point t_submit;
    int status = -1;  // -1 pending
    double latency_ms = 0;
    int batch_k = 0;
    std::string error;
};

struct Factor {
    rbs_plan *plan = nullptr;
    int n = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    // column tables (b columns, then x columns): pinned host copy and device copy
    const double **h_tab = nullptr;
    double **d_tab = nullptr;
    // staging for host-array requests (allocated with the first such request)
    double *db = nullptr, *dx = nullptr, *hb = nullptr, *hx = nullptr;
    long long stage_bytes = 0;
    std::deque<std::shared_ptr<Request>> queue;   // guarded by the server mutex
    std::vector<std::shared_ptr<Request>> batch;  // dispatcher thread only
    int state = 0;                                // 0 idle, 1 refinement step in flight, 2 final copies in flight
    int batch_k = 0;
    bool batch_host = false;
    long long bytes = 0;
};

int fail(int rc, const std::string &msg) {
    rbs::set_error(msg);
    return rc;
}

}  // namespace

struct rbs_server {
    long long budget = 0, used = 0;
    int max_k = 16;
    int device = 0;
    std::mutex mu;                       // guards factors, queues, requests, stats, stop
    std::condition_variable work_cv, done_cv;
    std::vector<std::unique_ptr<Factor>> factors;
    std::unordered_map<long long, std::shared_ptr<Request>> requests;
    long long next_id = 1, queued = 0;
    bool stop = false;
    std::thread dispatcher;
    std::vector<double> latencies;       // completed requests
    long long batches = 0, batched_rhs = 0, solves = 0;
    Clock::time_point t_first{}, t_last{};
    bool any_done = false;
};

namespace {

// Requests of one batch are finished with status rc (the same for all).
void complete(rbs_server *s, Factor &f, int rc, const std::string &err) {
    const auto now = Clock::now();
    if ((rc == RBS_OK || rc == RBS_ERR_NOCONV) && f.batch_host) {
        int off = 0;
        for (auto &r : f.batch) {
            if (!r->device) std::memcpy(r->x, f.hx + (size_t)off * f.n, sizeof(double) * (size_t)f.n * r->k);
            off += r->k;
        }
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto &r : f.batch) {
            r->status = rc;
            r->error = err;
            r->batch_k = f.batch_k;
            r->latency_ms = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
            s->latencies.push_back(r->latency_ms);
            s->solves += r->k;
        }
        s->batches += 1;
        s->batched_rhs += f.batch_k;
        s->t_last = now;
        s->any_done = true;
    }
    s->done_cv.notify_all();
    f.batch.clear();
    f.state = 0;
}

// Host staging of a factor (n x max_k, device and pinned host), charged
// against the budget.
int ensure_staging(rbs_server *s, Factor &f, std::string &err) {
    if (f.db) return RBS_OK;
    const long long bytes = (long long)sizeof(double) * f.n * s->max_k;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->used + 2 * bytes > s->budget) {
            err = "rbs_server: host-array staging for this factor (" + std::to_string(2 * bytes) +
                  " B) exceeds the remaining HBM budget";
            return RBS_ERR_BUDGET;
        }
        s->used += 2 * bytes;
        f.bytes += 2 * bytes;
    }
    f.stage_bytes = 2 * bytes;
    cudaError_t e = cudaMalloc(&f.db, (size_t)bytes);
    if (e == cudaSuccess) e = cudaMalloc(&f.dx, (size_t)bytes);
    if (e == cudaSuccess) e = cudaMallocHost(&f.hb, (size_t)bytes);
    if (e == cudaSuccess) e = cudaMallocHost(&f.hx, (size_t)bytes);
    if (e != cudaSuccess) {
        err = std::string("rbs_server: staging: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? RBS_ERR_NOMEM : RBS_ERR_CUDA;
    }
    return RBS_OK;
}

// Start the factor's batch (f.batch set): column tables, host staging copies,
// the solve's first phase, the completion event.
void start(rbs_server *s, Factor &f) {
    std::string err;
    int rc = RBS_OK;
    f.batch_host = false;
    f.batch_k = 0;
    for (auto &r : f.batch) {
        f.batch_host = f.batch_host || !r->device;
        f.batch_k += r->k;
    }
    if (f.batch_host && (rc = ensure_staging(s, f, err)) != RBS_OK) {
        f.batch_host = false;  // nothing to copy back
        return complete(s, f, rc, err);
    }
    const int mk = s->max_k;
    int k = 0;
    for (auto &r : f.batch) {
        for (int c = 0; c < r->k; ++c) {
            const size_t o = (size_t)(k + c) * f.n;
            if (r->device) {
                f.h_tab[k + c] = r->b + (size_t)c * f.n;
                f.h_tab[mk + k + c] = r->x + (size_t)c * f.n;
            } else {
                std::memcpy(f.hb + o, r->b + (size_t)c * f.n, sizeof(double) * f.n);
                f.h_tab[k + c] = f.db + o;
                f.h_tab[mk + k + c] = f.dx + o;
            }
        }
        k += r->k;
    }
    f.batch_k = k;
    cudaError_t e = cudaSuccess;
    if (f.batch_host) e = cudaMemcpyAsync(f.db, f.hb, sizeof(double) * (size_t)f.n * k, cudaMemcpyHostToDevice, f.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(f.d_tab, f.h_tab, sizeof(double *) * 2 * mk, cudaMemcpyHostToDevice, f.stream);
    if (e != cudaSuccess) return complete(s, f, RBS_ERR_CUDA, std::string("rbs_server: ") + cudaGetErrorString(e));
    int more = 0;
    rc = rbs::device_batch_start(f.plan->p, f.d_tab, f.d_tab + mk, k, f.batch.front()->prec, &more, err);
    if (rc != RBS_OK) return complete(s, f, rc, err);
    if (!more && f.batch_host)
        e = cudaMemcpyAsync(f.hx, f.dx, sizeof(double) * (size_t)f.n * k, cudaMemcpyDeviceToHost, f.stream);
    if (e == cudaSuccess) e = cudaEventRecord(f.ev, f.stream);
    if (e != cudaSuccess) return complete(s, f, RBS_ERR_CUDA, std::string("rbs_server: ") + cudaGetErrorString(e));
    f.state = more ? 1 : 2;
}

// The factor's event has completed: next refinement step, final copies, or done.
void advance(rbs_server *s, Factor &f) {
    std::string err;
    if (f.state == 1) {
        int more = 0;
        int rc = rbs::device_batch_next(f.plan->p, &more, err);
        if (rc != RBS_OK) return complete(s, f, rc, err);
        cudaError_t e = cudaSuccess;
        if (!more && f.batch_host)
            e = cudaMemcpyAsync(f.hx, f.dx, sizeof(double) * (size_t)f.n * f.batch_k, cudaMemcpyDeviceToHost,
                                f.stream);
        if (e == cudaSuccess) e = cudaEventRecord(f.ev, f.stream);
        if (e != cudaSuccess) return complete(s, f, RBS_ERR_CUDA, std::string("rbs_server: ") + cudaGetErrorString(e));
        f.state = more ? 1 : 2;
        return;
    }
    int iters = 0;
    double corr = 0;
    const int rc = rbs::device_batch_finish(f.plan->p, &iters, &corr, err);
    complete(s, f, rc, err);
}

void dispatch(rbs_server *s) {
    cudaSetDevice(s->device);
    std::vector<Factor *> fs, starting;
    for (;;) {
        bool busy = false, progressed = false;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            fs.clear();
            for (auto &f : s->factors) fs.push_back(f.get());
        }
        for (Factor *f : fs) {
            if (f->state == 0) continue;
            busy = true;
            const cudaError_t q = cudaEventQuery(f->ev);
            if (q == cudaErrorNotReady) continue;
            progressed = true;
            if (q != cudaSuccess) {
                complete(s, *f, RBS_ERR_CUDA, std::string("rbs_server: ") + cudaGetErrorString(q));
                continue;
            }
            advance(s, *f);
        }
        starting.clear();
        bool exit_now = false;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (Factor *f : fs) {
                if (f->state != 0 || f->queue.empty()) continue;
                int k = 0;
                const int prec = f->queue.front()->prec;
                while (!f->queue.empty() && f->queue.front()->prec == prec &&
                       (f->batch.empty() || k + f->queue.front()->k <= s->max_k)) {
                    k += f->queue.front()->k;
                    f->batch.push_back(f->queue.front());
                    f->queue.pop_front();
                    --s->queued;
                }
                starting.push_back(f);
            }
            if (s->stop && s->queued == 0 && starting.empty() && !busy) exit_now = true;
        }
        if (exit_now) return;
        for (Factor *f : starting) {
            start(s, *f);
            progressed = true;
            busy = true;
        }
        if (progressed) continue;
        std::unique_lock<std::mutex> lk(s->mu);
        if (busy)  // work in flight: poll again shortly, or at once on a new request
            s->work_cv.wait_for(lk, std::chrono::microseconds(20), [&] { return s->queued > 0 || s->stop; });
        else
            s->work_cv.wait(lk, [&] { return s->queued > 0 || s->stop; });
    }
}

void release(Factor &f) {
    if (f.stream) cudaStreamSynchronize(f.stream);
    // the plan runs on this stream: free it before the stream goes away
    if (f.plan) rbs_plan_free(f.plan);
    if (f.db) cudaFree(f.db);
    if (f.dx) cudaFree(f.dx);
    if (f.hb) cudaFreeHost(f.hb);
    if (f.hx) cudaFreeHost(f.hx);
    if (f.d_tab) cudaFree(f.d_tab);
    if (f.h_tab) cudaFreeHost(f.h_tab);
    if (f.ev) cudaEventDestroy(f.ev);
    if (f.stream) cudaStreamDestroy(f.stream);
    f = Factor();
}

int submit(rbs_server *s, int factor_id, const double *b, double *x, int k, int prec, bool device, long long *ticket) {
    if (!s || !b || !x || !ticket || k < 1) return fail(RBS_ERR_ARG, "rbs_server_submit: bad arguments");
    if (prec != RBS_PREC_FP64 && prec != RBS_PREC_MIXED && prec != RBS_PREC_FP32)
        return fail(RBS_ERR_ARG, "rbs_server_submit: unknown precision");
    auto r = std::make_shared<Request>();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (factor_id < 0 || factor_id >= (int)s->factors.size())
            return fail(RBS_ERR_ARG, "rbs_server_submit: unknown factor");
        if (k > s->max_k) return fail(RBS_ERR_ARG, "rbs_server_submit: k exceeds the server's batch width");
        if (s->stop) return fail(RBS_ERR_ARG, "rbs_server_submit: server is shutting down");
        r->id = s->next_id++;
        r->b = b;
        r->x = x;
        r->device = device;
        r->k = k;
        r->prec = prec;
        r->t_submit = Clock::now();
        if (!s->any_done && s->requests.empty()) s->t_first = r->t_submit;
        s->requests[r->id] = r;
        s->factors[factor_id]->queue.push_back(r);
        ++s->queued;
    }
    s->work_cv.notify_one();
    *ticket = r->id;
    return RBS_OK;
}

}  // namespace

extern "C" {

int rbs_server_create(long long hbm_budget_bytes, int max_batch_rhs, rbs_server **out) {
    if (!out || hbm_budget_bytes <= 0 || max_batch_rhs < 1 || max_batch_rhs > 128)
        return fail(RBS_ERR_ARG, "rbs_server_create: need a positive budget and 1 <= max_batch_rhs <= 128");
    rbs_server *s = new (std::nothrow) rbs_server();
    if (!s) return fail(RBS_ERR_NOMEM, "rbs_server_create: out of host memory");
    s->budget = hbm_budget_bytes;
    s->max_k = max_batch_rhs;
    cudaGetDevice(&s->device);
    try {
        s->dispatcher = std::thread(dispatch, s);
    } catch (...) {
        delete s;
        return fail(RBS_ERR_NOMEM, "rbs_server_create: cannot start the dispatcher thread");
    }
    *out = s;
    return RBS_OK;
}

int rbs_server_add_factor(rbs_server *s, rbs_plan *plan, int *factor_id) {
    if (!s || !plan || !factor_id) return fail(RBS_ERR_ARG, "rbs_server_add_factor: NULL argument");
    if (!plan->p.dev) return fail(RBS_ERR_ARG, "rbs_server_add_factor: plan has no device state");
    auto f = std::make_unique<Factor>();
    f->n = plan->p.n;
    std::string err;
    cudaError_t e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&f->h_tab, sizeof(double *) * 2 * s->max_k);
    if (e == cudaSuccess) e = cudaMalloc(&f->d_tab, sizeof(double *) * 2 * s->max_k);
    if (e != cudaSuccess) {
        release(*f);
        return fail(e == cudaErrorMemoryAllocation ? RBS_ERR_NOMEM : RBS_ERR_CUDA,
                    std::string("rbs_server_add_factor: ") + cudaGetErrorString(e));
    }
    // work vectors for the batch width now: no solve of this factor grows them later
    int rc = rbs_plan_set_stream(plan, f->stream);
    if (rc == RBS_OK && (rc = rbs::device_reserve(plan->p, s->max_k, err)) != RBS_OK) rbs::set_error(err);
    if (rc != RBS_OK) {
        const std::string msg = rbs_last_error();
        rbs_plan_set_stream(plan, nullptr);  // the caller keeps the plan, on a stream of its own again
        release(*f);
        return fail(rc, "rbs_server_add_factor: " + msg);
    }
    const long long bytes = rbs::device_bytes(plan->p) + (long long)sizeof(double *) * 2 * s->max_k;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->used + bytes > s->budget) {
        rbs_plan_set_stream(plan, nullptr);
        release(*f);
        return fail(RBS_ERR_BUDGET, "rbs_server_add_factor: plan with work vectors (" + std::to_string(bytes) +
                                        " B) exceeds the remaining budget (" + std::to_string(s->budget - s->used) +
                                        " B)");
    }
    f->plan = plan;
    f->bytes = bytes;
    s->used += bytes;
    *factor_id = (int)s->factors.size();
    s->factors.push_back(std::move(f));
    return RBS_OK;
}

int rbs_server_submit(rbs_server *s, int factor_id, const double *b, double *x, int k, int prec, long long *ticket) {
    return submit(s, factor_id, b, x, k, prec, false, ticket);
}

int rbs_server_submit_device(rbs_server *s, int factor_id, const double *d_b, double *d_x, int k, int prec,
                             long long *ticket) {
    return submit(s, factor_id, d_b, d_x, k, prec, true, ticket);
}

int rbs_server_wait(rbs_server *s, long long ticket, double *latency_ms, int *batch_k) {
    if (!s) return fail(RBS_ERR_ARG, "rbs_server_wait: NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return fail(RBS_ERR_ARG, "rbs_server_wait: unknown ticket");
    auto r = it->second;
    s->done_cv.wait(lk, [&] { return r->status >= 0; });
    s->requests.erase(ticket);
    if (latency_ms) *latency_ms = r->latency_ms;
    if (batch_k) *batch_k = r->batch_k;
    if (r->status != RBS_OK) rbs::set_error(r->error);
    return r->status;
}

int rbs_server_stats_get(rbs_server *s, rbs_server_stats *st) {
    if (!s || !st) return fail(RBS_ERR_ARG, "rbs_server_stats_get: NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(st, 0, sizeof(*st));
    std::vector<double> l = s->latencies;
    st->completed = (long long)l.size();
    st->solves = s->solves;
    st->batches = s->batches;
    st->mean_batch_rhs = s->batches ? (double)s->batched_rhs / s->batches : 0;
    st->factors = (int)s->factors.size();
    st->hbm_used = s->used;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) { return l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
        st->p50_ms = pct(0.50);
        st->p99_ms = pct(0.99);
        const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
        st->solves_per_s = span > 0 ? s->solves / span : 0;
    }
    return RBS_OK;
}

int rbs_server_reset_stats(rbs_server *s) {
    if (!s) return RBS_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->latencies.clear();
    s->batches = s->batched_rhs = s->solves = 0;
    s->any_done = false;
    return RBS_OK;
}

int rbs_server_destroy(rbs_server *s) {
    if (!s) return RBS_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->work_cv.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();  // queued requests are served first
    for (auto &f : s->factors) release(*f);
    delete s;
    return RBS_OK;
}

}  // extern "C"
