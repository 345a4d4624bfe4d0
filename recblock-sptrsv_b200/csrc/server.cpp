// server.cpp -- request loop over device-resident factors (no counterpart in
// the reference, which runs one solve per process).
//
// Factors: each admitted factor keeps its plan (permutation, blocks, kernel
// plan, captured block walks) on the device, with work vectors reserved at
// admission for the server's batch width, so no solve allocates or frees
// device memory while requests are served.  Small factors can be admitted
// together as a group: one block-diagonal plan (rbs_batch_analyse) whose
// systems are the group's members.  Admission is charged against the HBM
// budget: the plan, its work vectors and, once the unit receives its first
// host-array request, the staging buffers for host arrays.
//
// Requests: host arrays (rbs_server_submit) or device arrays
// (rbs_server_submit_device), n x k column-major, one precision each.  They
// queue per factor (per member of a group).
//
// Dispatch: ONE dispatcher thread issues every CUDA call of the server.  The
// unit of scheduling is a plan -- a single factor, or a group -- with its own
// stream and completion event, moving through
//   idle -> (batch started) -> refinement step in flight -> ... -> final
//   copies in flight -> idle.
// An idle unit with queued requests takes, for every member, the queued
// requests of one precision (that of its oldest request) that fit the batch
// width (FIFO), and runs them as ONE multi-RHS solve: column c of the solve
// carries the c-th queued column of every member, so a group's launch serves
// requests of many factors at once (their rows never interact).  Columns
// are read and written in place through device tables of column pointers,
// with no staging copy for device requests.  The dispatcher polls the events
// of all busy units and advances whichever finished: mixed-precision
// refinement decides on the host, per unit, whether another correction is
// needed, without holding up the others.  So requests that arrive while a
// batch runs join their unit's next batch (continuous batching within a
// factor), a group's launch carries requests of all its members, and the
// batches of all units overlap on the device (batching across factors).
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

struct Unit;

// A factor as requests see it: a whole plan, or member `member` of a group
// (its rows [row0, row0 + n) of the group's block-diagonal system).
struct Factor {
    Unit *unit = nullptr;
    int member = 0, n = 0, row0 = 0;
    std::deque<std::shared_ptr<Request>> queue;   // guarded by the server mutex
    std::vector<std::shared_ptr<Request>> batch;  // dispatcher thread only
    int batch_cols = 0;
};

struct Unit {
    rbs_plan *plan = nullptr;
    int n = 0;      // rows of the plan
    int count = 1;  // members (1: a single factor)
    std::vector<Factor *> members;
    int *d_seg = nullptr, *d_off = nullptr;  // groups: system of every row, first row of every system
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    // column tables (b, then x; a group's entry for column c, member f at
    // c*count + f): pinned host copy and device copy
    const double **h_tab = nullptr;
    double **d_tab = nullptr;
    // staging for host-array requests (n x max_k, allocated with the first such request)
    double *db = nullptr, *dx = nullptr, *hb = nullptr, *hx = nullptr;
    int state = 0;  // 0 idle, 1 refinement step in flight, 2 final copies in flight
    int batch_k = 0, batch_prec = 0;
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
    std::mutex mu;                       // guards factors, units, queues, requests, stats, stop
    std::condition_variable work_cv, done_cv;
    std::vector<std::unique_ptr<Unit>> units;
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

// Requests of the unit's batch are finished with status rc (the same for all).
void complete(rbs_server *s, Unit &u, int rc, const std::string &err) {
    const auto now = Clock::now();
    if ((rc == RBS_OK || rc == RBS_ERR_NOCONV) && u.batch_host) {
        for (Factor *f : u.members) {
            int c = 0;
            for (auto &r : f->batch) {
                if (!r->device)
                    for (int q = 0; q < r->k; ++q)
                        std::memcpy(r->x + (size_t)q * f->n, u.hx + (size_t)(c + q) * u.n + f->row0,
                                    sizeof(double) * (size_t)f->n);
                c += r->k;
            }
        }
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        long long cols = 0;
        for (Factor *f : u.members) {
            for (auto &r : f->batch) {
                r->status = rc;
                r->error = err;
                r->batch_k = u.batch_k;
                r->latency_ms = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
                s->latencies.push_back(r->latency_ms);
                s->solves += r->k;
            }
            cols += f->batch_cols;
        }
        s->batches += 1;
        s->batched_rhs += cols;
        s->t_last = now;
        s->any_done = true;
    }
    s->done_cv.notify_all();
    for (Factor *f : u.members) {
        f->batch.clear();
        f->batch_cols = 0;
    }
    u.state = 0;
}

// Host staging of a unit (n x max_k, device and pinned host), charged
// against the budget.
int ensure_staging(rbs_server *s, Unit &u, std::string &err) {
    if (u.db) return RBS_OK;
    const long long bytes = (long long)sizeof(double) * u.n * s->max_k;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->used + 2 * bytes > s->budget) {
            err = "rbs_server: host-array staging for this factor (" + std::to_string(2 * bytes) +
                  " B) exceeds the remaining HBM budget";
            return RBS_ERR_BUDGET;
        }
        s->used += 2 * bytes;
        u.bytes += 2 * bytes;
    }
    cudaError_t e = cudaMalloc(&u.db, (size_t)bytes);
    if (e == cudaSuccess) e = cudaMalloc(&u.dx, (size_t)bytes);
    if (e == cudaSuccess) e = cudaMallocHost(&u.hb, (size_t)bytes);
    if (e == cudaSuccess) e = cudaMallocHost(&u.hx, (size_t)bytes);
    if (e != cudaSuccess) {
        err = std::string("rbs_server: staging: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? RBS_ERR_NOMEM : RBS_ERR_CUDA;
    }
    return RBS_OK;
}

// Start the unit's batch (members' batches set): column tables, host staging
// copies, the solve's first phase, the completion event.
void start(rbs_server *s, Unit &u) {
    std::string err;
    int rc = RBS_OK;
    const int mk = s->max_k, F = u.count;
    u.batch_host = false;
    u.batch_k = 0;
    for (Factor *f : u.members) {
        f->batch_cols = 0;
        for (auto &r : f->batch) {
            u.batch_host = u.batch_host || !r->device;
            f->batch_cols += r->k;
        }
        u.batch_k = std::max(u.batch_k, f->batch_cols);
    }
    if (u.batch_host && (rc = ensure_staging(s, u, err)) != RBS_OK) {
        u.batch_host = false;  // nothing to copy back
        return complete(s, u, rc, err);
    }
    const double **btab = u.h_tab, **xtab = u.h_tab + (size_t)mk * F;
    std::fill(u.h_tab, u.h_tab + 2 * (size_t)mk * F, nullptr);
    for (Factor *f : u.members) {
        int c = 0;
        for (auto &r : f->batch) {
            for (int q = 0; q < r->k; ++q, ++c) {
                const size_t slot = F == 1 ? (size_t)c : (size_t)c * F + f->member;
                if (r->device) {
                    btab[slot] = r->b + (size_t)q * f->n;
                    xtab[slot] = r->x + (size_t)q * f->n;
                } else {
                    const size_t o = (size_t)c * u.n + f->row0;
                    std::memcpy(u.hb + o, r->b + (size_t)q * f->n, sizeof(double) * f->n);
                    btab[slot] = u.db + o;
                    xtab[slot] = u.dx + o;
                }
            }
        }
    }
    const int k = u.batch_k;
    cudaError_t e = cudaSuccess;
    if (u.batch_host)
        e = cudaMemcpyAsync(u.db, u.hb, sizeof(double) * (size_t)u.n * k, cudaMemcpyHostToDevice, u.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(u.d_tab, u.h_tab, sizeof(double *) * 2 * (size_t)mk * F, cudaMemcpyHostToDevice, u.stream);
    if (e != cudaSuccess) return complete(s, u, RBS_ERR_CUDA, std::string("rbs_server: ") + cudaGetErrorString(e));
    int more = 0;
    if (F == 1) {
        rc = rbs::device_batch_start(u.plan->p, u.d_tab, u.d_tab + mk, k, u.batch_prec, &more, err);
    } else {
        const rbs::BatchGroup g{u.d_tab, u.d_tab + (size_t)mk * F, u.d_seg, u.d_off, F};
        rc = rbs::device_batch_start(u.plan->p, nullptr, nullptr, k, u.batch_prec, &more, err, &g);
    }
    if (rc != RBS_OK) return complete(s, u, rc, err);
    if (!more && u.batch_host)
        e = cudaMemcpyAsync(u.hx, u.dx, sizeof(double) * (size_t)u.n * k, cudaMemcpyDeviceToHost, u.stream);
    if (e == cudaSuccess) e = cudaEventRecord(u.ev, u.stream);
    if (e != cudaSuccess) return complete(s, u, RBS_ERR_CUDA, std::string("rbs_server: ") + cudaGetErrorString(e));
    u.state = more ? 1 : 2;
}

// The unit's event has completed: next refinement step, final copies, or done.
void advance(rbs_server *s, Unit &u) {
    std::string err;
    if (u.state == 1) {
        int more = 0;
        int rc = rbs::device_batch_next(u.plan->p, &more, err);
        if (rc != RBS_OK) return complete(s, u, rc, err);
        cudaError_t e = cudaSuccess;
        if (!more && u.batch_host)
            e = cudaMemcpyAsync(u.hx, u.dx, sizeof(double) * (size_t)u.n * u.batch_k, cudaMemcpyDeviceToHost,
                                u.stream);
        if (e == cudaSuccess) e = cudaEventRecord(u.ev, u.stream);
        if (e != cudaSuccess) return complete(s, u, RBS_ERR_CUDA, std::string("rbs_server: ") + cudaGetErrorString(e));
        u.state = more ? 1 : 2;
        return;
    }
    int iters = 0;
    double corr = 0;
    const int rc = rbs::device_batch_finish(u.plan->p, &iters, &corr, err);
    complete(s, u, rc, err);
}

// Under the server lock: the batch of an idle unit, if any member has
// requests.  Precision: that of the unit's oldest queued request.
bool take_batch(rbs_server *s, Unit &u) {
    const Request *oldest = nullptr;
    for (Factor *f : u.members)
        if (!f->queue.empty() && (!oldest || f->queue.front()->t_submit < oldest->t_submit))
            oldest = f->queue.front().get();
    if (!oldest) return false;
    u.batch_prec = oldest->prec;
    for (Factor *f : u.members) {
        int k = 0;
        // FIFO per member: stop at the first request of another precision
        while (!f->queue.empty() && f->queue.front()->prec == u.batch_prec &&
               (f->batch.empty() || k + f->queue.front()->k <= s->max_k)) {
            k += f->queue.front()->k;
            f->batch.push_back(f->queue.front());
            f->queue.pop_front();
            --s->queued;
        }
    }
    return true;
}

void dispatch(rbs_server *s) {
    cudaSetDevice(s->device);
    std::vector<Unit *> us, starting;
    for (;;) {
        bool busy = false, progressed = false;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            us.clear();
            for (auto &u : s->units) us.push_back(u.get());
        }
        for (Unit *u : us) {
            if (u->state == 0) continue;
            busy = true;
            const cudaError_t q = cudaEventQuery(u->ev);
            if (q == cudaErrorNotReady) continue;
            progressed = true;
            if (q != cudaSuccess) {
                complete(s, *u, RBS_ERR_CUDA, std::string("rbs_server: ") + cudaGetErrorString(q));
                continue;
            }
            advance(s, *u);
        }
        starting.clear();
        bool exit_now = false;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (Unit *u : us)
                if (u->state == 0 && take_batch(s, *u)) starting.push_back(u);
            if (s->stop && s->queued == 0 && starting.empty() && !busy) exit_now = true;
        }
        if (exit_now) return;
        for (Unit *u : starting) {
            start(s, *u);
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

void release(Unit &u) {
    if (u.stream) cudaStreamSynchronize(u.stream);
    // the plan runs on this stream: free it before the stream goes away
    if (u.plan) rbs_plan_free(u.plan);
    for (void *p : {(void *)u.db, (void *)u.dx, (void *)u.d_tab, (void *)u.d_seg, (void *)u.d_off})
        if (p) cudaFree(p);
    if (u.hb) cudaFreeHost(u.hb);
    if (u.hx) cudaFreeHost(u.hx);
    if (u.h_tab) cudaFreeHost(u.h_tab);
    if (u.ev) cudaEventDestroy(u.ev);
    if (u.stream) cudaStreamDestroy(u.stream);
    u = Unit();
}

// A new unit for `plan` (members' row ranges in offs, count + 1 entries, or
// NULL for a single factor): stream, tables, work vectors reserved for the
// batch width, budget charge.  On failure the caller keeps the plan.
int add_unit(rbs_server *s, rbs_plan *plan, int count, const int *offs, int *factor_ids) {
    if (!s || !plan || !factor_ids || count < 1) return fail(RBS_ERR_ARG, "rbs_server_add: NULL argument");
    if (!plan->p.dev) return fail(RBS_ERR_ARG, "rbs_server_add: plan has no device state");
    const int n = plan->p.n;
    if (offs) {
        if (offs[0] != 0 || offs[count] != n)
            return fail(RBS_ERR_ARG, "rbs_server_add_group: row offsets must run from 0 to the plan's n");
        for (int f = 0; f < count; ++f)
            if (offs[f + 1] <= offs[f]) return fail(RBS_ERR_ARG, "rbs_server_add_group: empty or decreasing system");
    }
    auto u = std::make_unique<Unit>();
    u->n = n;
    u->count = count;
    const size_t tab = sizeof(double *) * 2 * (size_t)s->max_k * count;
    cudaError_t e = cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&u->ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&u->h_tab, tab);
    if (e == cudaSuccess) e = cudaMalloc(&u->d_tab, tab);
    if (e == cudaSuccess && offs) {
        std::vector<int> seg((size_t)n);
        for (int f = 0; f < count; ++f) std::fill(seg.begin() + offs[f], seg.begin() + offs[f + 1], f);
        e = cudaMalloc(&u->d_seg, sizeof(int) * (size_t)n);
        if (e == cudaSuccess) e = cudaMalloc(&u->d_off, sizeof(int) * ((size_t)count + 1));
        if (e == cudaSuccess) e = cudaMemcpy(u->d_seg, seg.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(u->d_off, offs, sizeof(int) * ((size_t)count + 1), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        release(*u);
        return fail(e == cudaErrorMemoryAllocation ? RBS_ERR_NOMEM : RBS_ERR_CUDA,
                    std::string("rbs_server_add: ") + cudaGetErrorString(e));
    }
    // work vectors for the batch width now: no solve of this unit grows them later
    std::string err;
    int rc = rbs_plan_set_stream(plan, u->stream);
    if (rc == RBS_OK && (rc = rbs::device_reserve(plan->p, s->max_k, err)) != RBS_OK) rbs::set_error(err);
    if (rc != RBS_OK) {
        const std::string msg = rbs_last_error();
        rbs_plan_set_stream(plan, nullptr);  // the caller keeps the plan, on a stream of its own again
        release(*u);
        return fail(rc, "rbs_server_add: " + msg);
    }
    const long long bytes = rbs::device_bytes(plan->p) + (long long)tab + (offs ? 4LL * (n + count + 1) : 0);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->used + bytes > s->budget) {
        rbs_plan_set_stream(plan, nullptr);
        release(*u);
        return fail(RBS_ERR_BUDGET, "rbs_server_add: plan with work vectors (" + std::to_string(bytes) +
                                        " B) exceeds the remaining budget (" + std::to_string(s->budget - s->used) +
                                        " B)");
    }
    u->plan = plan;
    u->bytes = bytes;
    s->used += bytes;
    for (int f = 0; f < count; ++f) {
        auto fac = std::make_unique<Factor>();
        fac->unit = u.get();
        fac->member = f;
        fac->row0 = offs ? offs[f] : 0;
        fac->n = offs ? offs[f + 1] - offs[f] : n;
        u->members.push_back(fac.get());
        factor_ids[f] = (int)s->factors.size();
        s->factors.push_back(std::move(fac));
    }
    s->units.push_back(std::move(u));
    return RBS_OK;
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
    return add_unit(s, plan, 1, nullptr, factor_id);
}

int rbs_server_add_group(rbs_server *s, rbs_plan *batch_plan, int count, const int *row_offsets, int *factor_ids) {
    if (!row_offsets) return fail(RBS_ERR_ARG, "rbs_server_add_group: NULL row offsets");
    return add_unit(s, batch_plan, count, row_offsets, factor_ids);
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
    for (auto &u : s->units) release(*u);
    delete s;
    return RBS_OK;
}

}  // extern "C"
