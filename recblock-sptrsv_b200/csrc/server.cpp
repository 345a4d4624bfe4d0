// server.cpp -- request loop over device-resident factors (no counterpart in
// the reference, which runs one solve per process).
//
// Each admitted factor keeps its plan (permutation, blocks, kernel plan) on
// the device and gets a worker thread with its own CUDA stream.  Requests
// (host b and x, k right-hand sides, a precision) queue per factor; a worker
// that finds requests waiting takes as many as fit in its batch width (same
// precision, FIFO), packs their columns into one pinned staging buffer and
// runs ONE multi-RHS solve for all of them, so requests that arrive while a
// batch is on the GPU join the next one (continuous batching within a
// factor) while other factors' workers run on their own streams at the same
// time (batching across factors is concurrency on the device).  Admission:
// a factor is accepted only if its plan plus its workspace fit in the
// remaining HBM budget.
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
    long long id;
    const double *b;
    double *x;
    int k, prec;
    Clock::time_point t_submit;
    int status = -1;  // -1 pending
    double latency_ms = 0;
    int batch_k = 0;
    std::string error;
};

struct Factor;

}  // namespace

struct rbs_server {
    long long budget = 0, used = 0;
    int max_k = 16;
    std::mutex mu;                       // guards factors, requests, stats
    std::condition_variable done_cv;
    std::vector<std::unique_ptr<Factor>> factors;
    std::unordered_map<long long, std::shared_ptr<Request>> requests;
    long long next_id = 1;
    std::vector<double> latencies;       // completed requests
    long long batches = 0, batched_rhs = 0, solves = 0;
    Clock::time_point t_first{}, t_last{};
    bool any_done = false;
};

namespace {

struct Factor {
    rbs_server *srv = nullptr;
    rbs_plan *plan = nullptr;
    int n = 0;
    cudaStream_t stream = nullptr;
    double *db = nullptr, *dx = nullptr;     // device batch buffers (n x max_k)
    double *hb = nullptr, *hx = nullptr;     // pinned staging
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::shared_ptr<Request>> queue;
    bool stop = false;
    std::thread worker;
    long long bytes = 0;

    void run() {
        const int max_k = srv->max_k;
        for (;;) {
            std::vector<std::shared_ptr<Request>> batch;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (stop && queue.empty()) return;
                int k = 0;
                const int prec = queue.front()->prec;
                while (!queue.empty() && queue.front()->prec == prec &&
                       (batch.empty() || k + queue.front()->k <= max_k)) {
                    k += queue.front()->k;
                    batch.push_back(queue.front());
                    queue.pop_front();
                }
            }
            int k = 0;
            for (auto &r : batch) {
                std::memcpy(hb + (size_t)k * n, r->b, sizeof(double) * (size_t)n * r->k);
                k += r->k;
            }
            std::string err;
            int rc = RBS_OK;
            cudaError_t e = cudaMemcpyAsync(db, hb, sizeof(double) * (size_t)n * k, cudaMemcpyHostToDevice, stream);
            if (e != cudaSuccess) {
                rc = RBS_ERR_CUDA;
                err = cudaGetErrorString(e);
            }
            if (rc == RBS_OK) {
                rc = rbs_solve(plan, db, dx, k, n, batch.front()->prec, nullptr);
                if (rc != RBS_OK && rc != RBS_ERR_NOCONV) err = rbs_last_error();
            }
            if (rc == RBS_OK || rc == RBS_ERR_NOCONV) {
                e = cudaMemcpyAsync(hx, dx, sizeof(double) * (size_t)n * k, cudaMemcpyDeviceToHost, stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
                if (e != cudaSuccess) {
                    rc = RBS_ERR_CUDA;
                    err = cudaGetErrorString(e);
                }
            }
            // results out of the staging buffer before the server lock: the
            // copies (tens of MB) must not hold up the other factors' workers
            if (rc == RBS_OK || rc == RBS_ERR_NOCONV) {
                int off = 0;
                for (auto &r : batch) {
                    std::memcpy(r->x, hx + (size_t)off * n, sizeof(double) * (size_t)n * r->k);
                    off += r->k;
                }
            }
            const auto now = Clock::now();
            {
                std::lock_guard<std::mutex> lk(srv->mu);
                for (auto &r : batch) {
                    r->status = rc;
                    r->error = err;
                    r->batch_k = k;
                    r->latency_ms = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
                    srv->latencies.push_back(r->latency_ms);
                    srv->solves += r->k;
                }
                srv->batches += 1;
                srv->batched_rhs += k;
                srv->t_last = now;
                srv->any_done = true;
            }
            srv->done_cv.notify_all();
        }
    }

    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
        if (stream) cudaStreamSynchronize(stream);
        // the plan runs on this stream: free it before the stream goes away
        if (plan) rbs_plan_free(plan);
        if (db) cudaFree(db);
        if (dx) cudaFree(dx);
        if (hb) cudaFreeHost(hb);
        if (hx) cudaFreeHost(hx);
        if (stream) cudaStreamDestroy(stream);
        db = dx = hb = hx = nullptr;
        stream = nullptr;
        plan = nullptr;
    }
};

int fail(int rc, const std::string &msg) {
    rbs::set_error(msg);
    return rc;
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
    *out = s;
    return RBS_OK;
}

int rbs_server_add_factor(rbs_server *s, rbs_plan *plan, int *factor_id) {
    if (!s || !plan || !factor_id) return fail(RBS_ERR_ARG, "rbs_server_add_factor: NULL argument");
    rbs_plan_info info;
    if (rbs_plan_info_get(plan, &info) != RBS_OK) return RBS_ERR_ARG;
    if (info.device_bytes == 0) return fail(RBS_ERR_ARG, "rbs_server_add_factor: plan has no device state");
    // workspace: batch buffers plus the plan's work vectors at the batch width
    const long long n = info.n;
    const long long work = n * s->max_k * (8LL * 2 + 40LL);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->used + info.device_bytes + work > s->budget)
        return fail(RBS_ERR_BUDGET, "rbs_server_add_factor: plan (" + std::to_string(info.device_bytes) +
                                        " B) + workspace (" + std::to_string(work) + " B) exceed the remaining budget (" +
                                        std::to_string(s->budget - s->used) + " B)");
    auto f = std::make_unique<Factor>();
    f->srv = s;
    f->plan = plan;
    f->n = (int)n;
    f->bytes = info.device_bytes + work;
    const size_t bytes = sizeof(double) * (size_t)n * s->max_k;
    cudaError_t e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&f->db, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&f->dx, bytes);
    if (e == cudaSuccess) e = cudaMallocHost(&f->hb, bytes);
    if (e == cudaSuccess) e = cudaMallocHost(&f->hx, bytes);
    if (e != cudaSuccess) {
        f->plan = nullptr;  // the caller keeps the plan on failure
        f->shutdown();
        return fail(e == cudaErrorMemoryAllocation ? RBS_ERR_NOMEM : RBS_ERR_CUDA,
                    std::string("rbs_server_add_factor: ") + cudaGetErrorString(e));
    }
    if (rbs_plan_set_stream(plan, f->stream) != RBS_OK) {
        f->plan = nullptr;
        f->shutdown();
        return RBS_ERR_CUDA;
    }
    s->used += f->bytes;
    Factor *raw = f.get();
    raw->worker = std::thread([raw] { raw->run(); });
    *factor_id = (int)s->factors.size();
    s->factors.push_back(std::move(f));
    return RBS_OK;
}

int rbs_server_submit(rbs_server *s, int factor_id, const double *b, double *x, int k, int prec, long long *ticket) {
    if (!s || !b || !x || !ticket || k < 1) return fail(RBS_ERR_ARG, "rbs_server_submit: bad arguments");
    Factor *f;
    auto r = std::make_shared<Request>();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (factor_id < 0 || factor_id >= (int)s->factors.size())
            return fail(RBS_ERR_ARG, "rbs_server_submit: unknown factor");
        f = s->factors[factor_id].get();
        if (k > s->max_k) return fail(RBS_ERR_ARG, "rbs_server_submit: k exceeds the server's batch width");
        r->id = s->next_id++;
        r->b = b;
        r->x = x;
        r->k = k;
        r->prec = prec;
        r->t_submit = Clock::now();
        if (!s->any_done && s->requests.empty()) s->t_first = r->t_submit;
        s->requests[r->id] = r;
    }
    {
        std::lock_guard<std::mutex> lk(f->mu);
        f->queue.push_back(r);
    }
    f->cv.notify_one();
    *ticket = r->id;
    return RBS_OK;
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
    for (auto &f : s->factors) f->shutdown();
    delete s;
    return RBS_OK;
}

}  // extern "C"
