// api.cu -- the extern "C" boundary declared in include/rbs.h.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "rbs.h"
#include "rbs_internal.h"

namespace rbs {
namespace {
thread_local std::string g_error;
}
void set_error(const std::string &msg) { g_error = msg; }
}  // namespace rbs

using rbs::set_error;

static int fail(int rc, const std::string &msg) {
    set_error(msg);
    return rc;
}

extern "C" {

const char *rbs_last_error(void) { return rbs::g_error.c_str(); }

void rbs_options_default(rbs_options *opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->select = RBS_SELECT_AUTO;
    opt->device = -1;
    opt->lv_device_id = 0;
    opt->host_only = 0;
    opt->max_rhs = 1;
    opt->mixed = 1;
    opt->ir_tol = 1e-13;
    opt->ir_max_iter = 8;
    opt->spin_limit = 1LL << 22;
}

int rbs_auto_lv(int m, int device_id) { return rbs::auto_lv(m, device_id); }

}  // extern "C"

// rbs_analyse, optionally with the original-row offsets of independent
// systems (a batch), which the level-chunk layout solves one CTA each.
static int analyse_impl(const int *ptr, const int *idx, const double *val, int n, int nnz, int fmt, int substitution,
                        int lv, const rbs_options *opt, rbs_plan **plan, const std::vector<int> *segs) {
    if (!plan) return fail(RBS_ERR_ARG, "rbs_analyse: plan is NULL");
    *plan = nullptr;
    rbs_options o;
    rbs_options_default(&o);
    if (opt) o = *opt;
    if (o.max_rhs < 1) o.max_rhs = 1;
    if (o.spin_limit <= 0) o.spin_limit = 1LL << 22;
    if (o.ir_max_iter <= 0) o.ir_max_iter = 8;
    if (!(o.ir_tol > 0)) o.ir_tol = 1e-13;
    if (o.select < RBS_SELECT_REFERENCE || o.select > RBS_SELECT_TUNE)
        return fail(RBS_ERR_ARG, "rbs_analyse: unknown select mode");
    rbs_plan *P = new (std::nothrow) rbs_plan();
    if (!P) return fail(RBS_ERR_NOMEM, "rbs_analyse: out of host memory");
    std::string err;
    int rc;
    try {
        rc = rbs::analyse_host(P->p, ptr, idx, val, n, nnz, fmt, substitution, lv, o, err, segs);
        if (rc == RBS_OK && !o.host_only) rc = rbs::device_build(P->p, err);
        if (rc == RBS_OK && !o.host_only && o.select == RBS_SELECT_TUNE) rc = rbs::device_tune(P->p, err);
    } catch (const std::bad_alloc &) {
        rc = RBS_ERR_NOMEM;
        err = "rbs_analyse: out of host memory";
    }
    if (rc != RBS_OK) {
        rbs::device_free(P->p);
        delete P;
        return fail(rc, err);
    }
    *plan = P;
    set_error("");
    return RBS_OK;
}

extern "C" {

int rbs_analyse(const int *ptr, const int *idx, const double *val, int n, int nnz, int fmt, int substitution, int lv,
                const rbs_options *opt, rbs_plan **plan) {
    return analyse_impl(ptr, idx, val, n, nnz, fmt, substitution, lv, opt, plan, nullptr);
}

int rbs_analyse_device(const int *d_ptr, const int *d_idx, const double *d_val, int n, int nnz, int fmt,
                       int substitution, int lv, const rbs_options *opt, rbs_plan **plan) {
    if (!plan) return fail(RBS_ERR_ARG, "rbs_analyse_device: plan is NULL");
    *plan = nullptr;
    if (!d_ptr || !d_idx || !d_val || n <= 0 || nnz < n)
        return fail(RBS_ERR_ARG, "rbs_analyse_device: need n > 0, nnz >= n and non-null arrays");
    if (substitution != RBS_FORWARD && substitution != RBS_BACKWARD)
        return fail(RBS_ERR_ARG, "rbs_analyse: substitution must be RBS_FORWARD or RBS_BACKWARD");
    if (fmt != RBS_FMT_CSC && fmt != RBS_FMT_CSR) return fail(RBS_ERR_ARG, "rbs_analyse: fmt must be RBS_FMT_CSC or RBS_FMT_CSR");
    rbs_options o;
    rbs_options_default(&o);
    if (opt) o = *opt;
    if (o.max_rhs < 1) o.max_rhs = 1;
    if (o.spin_limit <= 0) o.spin_limit = 1LL << 22;
    if (o.ir_max_iter <= 0) o.ir_max_iter = 8;
    if (!(o.ir_tol > 0)) o.ir_tol = 1e-13;
    if (o.select < RBS_SELECT_REFERENCE || o.select > RBS_SELECT_TUNE)
        return fail(RBS_ERR_ARG, "rbs_analyse: unknown select mode");
    if (o.device >= 0) {
        cudaError_t e = cudaSetDevice(o.device);
        if (e != cudaSuccess) return fail(RBS_ERR_CUDA, std::string("rbs_analyse_device: ") + cudaGetErrorString(e));
    }
    rbs_plan *P = new (std::nothrow) rbs_plan();
    if (!P) return fail(RBS_ERR_NOMEM, "rbs_analyse: out of host memory");
    std::string err;
    int rc;
    try {
        // validation, level sets, reordering and the processing-order CSR on
        // the device; then the block extraction and packing on the device
        // (counts, local levels, entry pools) and the O(rows) layout steps
        // on the host
        auto t0 = std::chrono::steady_clock::now();
        rbs::DevRows rows;
        rc = rbs::device_analyse(P->p, d_ptr, d_idx, d_val, n, nnz, fmt, substitution, err, &rows);
        P->p.analyse_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        P->p.device_analyse_ms = P->p.analyse_ms;
        if (rc == RBS_OK) rc = rbs::analyse_after_levels(P->p, n, nnz, substitution, lv, o, err, nullptr, &rows);
        if (rc == RBS_OK && !o.host_only) rc = rbs::device_build(P->p, err);
        if (rc == RBS_OK && !o.host_only && o.select == RBS_SELECT_TUNE) rc = rbs::device_tune(P->p, err);
    } catch (const std::bad_alloc &) {
        rc = RBS_ERR_NOMEM;
        err = "rbs_analyse: out of host memory";
    }
    if (rc != RBS_OK) {
        rbs::device_free(P->p);
        delete P;
        return fail(rc, err);
    }
    *plan = P;
    set_error("");
    return RBS_OK;
}

int rbs_batch_analyse(int count, const int *const *ptr, const int *const *idx, const double *const *val,
                      const int *n, const int *nnz, int fmt, int substitution, int lv, const rbs_options *opt,
                      rbs_plan **plan, int *row_offsets) {
    if (!plan || count <= 0 || !ptr || !idx || !val || !n || !nnz || !row_offsets)
        return fail(RBS_ERR_ARG, "rbs_batch_analyse: bad arguments");
    long long N = 0, Z = 0;
    for (int i = 0; i < count; ++i) {
        if (n[i] <= 0 || nnz[i] < n[i] || !ptr[i] || !idx[i] || !val[i])
            return fail(RBS_ERR_ARG, "rbs_batch_analyse: system " + std::to_string(i) + " is malformed");
        N += n[i];
        Z += nnz[i];
    }
    if (N > 0x7fffffffLL || Z > 0x7fffffffLL) return fail(RBS_ERR_ARG, "rbs_batch_analyse: batch exceeds 2^31 rows or entries");
    for (int i = 0; i < count; ++i)
        if (ptr[i][0] != 0 || ptr[i][n[i]] != nnz[i])
            return fail(RBS_ERR_STRUCTURE, "rbs_batch_analyse: pointer array of system " + std::to_string(i) +
                                               " must run from 0 to nnz");
    std::vector<long long> z0((size_t)count + 1, 0);
    row_offsets[0] = 0;
    for (int i = 0; i < count; ++i) {
        row_offsets[i + 1] = row_offsets[i] + n[i];
        z0[(size_t)i + 1] = z0[(size_t)i] + nnz[i];
    }
    // the block-diagonal matrix, system by system on host threads
    std::vector<int> bp((size_t)N + 1);
    rbs::bulk_vector<int> bi((size_t)Z);
    rbs::bulk_vector<double> bv((size_t)Z);
    rbs::parallel_for((size_t)count, [&](size_t i) {
        const int r0 = row_offsets[i];
        for (int c = 0; c < n[i]; ++c) bp[(size_t)(r0 + c)] = (int)(z0[i] + ptr[i][c]);
        for (int k = 0; k < nnz[i]; ++k) {
            const int v = idx[i][k];
            bi[(size_t)(z0[i] + k)] = (v >= 0 && v < n[i]) ? v + r0 : -1;  // -1 is rejected by the analysis
            bv[(size_t)(z0[i] + k)] = val[i][k];
        }
    });
    bp[(size_t)N] = (int)Z;
    const std::vector<int> segs(row_offsets, row_offsets + count);
    return analyse_impl(bp.data(), bi.data(), bv.data(), (int)N, (int)Z, fmt, substitution, lv < 0 ? 0 : lv, opt, plan,
                        &segs);
}

static int check_solve_args(rbs_plan *plan, const double *b, const double *x, int k, int ld, int prec) {
    if (!plan) return fail(RBS_ERR_ARG, "solve: plan is NULL");
    if (!b || !x) return fail(RBS_ERR_ARG, "solve: b or x is NULL");
    if (k < 1) return fail(RBS_ERR_ARG, "solve: k must be >= 1");
    if (ld < plan->p.n) return fail(RBS_ERR_ARG, "solve: ld must be >= n");
    if (prec != RBS_PREC_FP64 && prec != RBS_PREC_MIXED && prec != RBS_PREC_FP32)
        return fail(RBS_ERR_ARG, "solve: unknown precision");
    return RBS_OK;
}

int rbs_solve(rbs_plan *plan, const double *d_b, double *d_x, int k, int ld, int prec, rbs_stats *stats) {
    int rc = check_solve_args(plan, d_b, d_x, k, ld, prec);
    if (rc) return rc;
    std::string err;
    rc = rbs::device_solve(plan->p, d_b, d_x, k, ld, prec, true, stats, err);
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_solve_async(rbs_plan *plan, const double *d_b, double *d_x, int k, int ld, int prec) {
    int rc = check_solve_args(plan, d_b, d_x, k, ld, prec);
    if (rc) return rc;
    if (prec == RBS_PREC_MIXED) return rbs_solve(plan, d_b, d_x, k, ld, prec, nullptr);
    std::string err;
    rc = rbs::device_solve(plan->p, d_b, d_x, k, ld, prec, false, nullptr, err);
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_plan_sync(rbs_plan *plan) {
    if (!plan || !plan->p.dev) return fail(RBS_ERR_ARG, "rbs_plan_sync: no device plan");
    std::string err;
    int rc = rbs::device_sync(plan->p, err);
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_solve_host(rbs_plan *plan, const double *b, double *x, int k, int ld, int prec, rbs_stats *stats) {
    int rc = check_solve_args(plan, b, x, k, ld, prec);
    if (rc) return rc;
    if (!plan->p.dev) return fail(RBS_ERR_ARG, "rbs_solve_host: plan has no device state");
    // plan-owned staging buffers (kept between calls); the copies run on the
    // plan's stream, so pinned host arrays overlap nothing else but avoid a
    // bounce through pageable staging in the driver
    size_t bytes = sizeof(double) * (size_t)ld * (size_t)k;
    double *db = nullptr, *dx = nullptr;
    std::string err;
    rc = rbs::device_staging(plan->p, bytes, db, dx, err);
    if (rc) return fail(rc, err);
    void *st = rbs::device_stream(plan->p);
    size_t nbytes = sizeof(double) * (size_t)plan->p.n;
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < k && e == cudaSuccess; ++c)
        e = cudaMemcpyAsync(db + (size_t)c * ld, b + (size_t)c * ld, nbytes, cudaMemcpyHostToDevice,
                            (cudaStream_t)st);
    if (e != cudaSuccess) return fail(RBS_ERR_CUDA, std::string("rbs_solve_host: ") + cudaGetErrorString(e));
    rc = rbs::device_solve(plan->p, db, dx, k, ld, prec, false, nullptr, err);
    if (rc == RBS_OK || rc == RBS_ERR_NOCONV) {
        for (int c = 0; c < k && e == cudaSuccess; ++c)
            e = cudaMemcpyAsync(x + (size_t)c * ld, dx + (size_t)c * ld, nbytes, cudaMemcpyDeviceToHost,
                                (cudaStream_t)st);
        if (e != cudaSuccess && rc == RBS_OK) {
            rc = RBS_ERR_CUDA;
            err = std::string("rbs_solve_host: ") + cudaGetErrorString(e);
        }
    }
    int rc2 = rbs::device_finish(plan->p, stats, k, prec, err);
    if (rc == RBS_OK) rc = rc2;
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_solve_host_async(rbs_plan *plan, const double *b, double *x, int k, int ld, int prec) {
    int rc = check_solve_args(plan, b, x, k, ld, prec);
    if (rc) return rc;
    if (!plan->p.dev) return fail(RBS_ERR_ARG, "rbs_solve_host_async: plan has no device state");
    if (prec == RBS_PREC_MIXED) return rbs_solve_host(plan, b, x, k, ld, prec, nullptr);  // refinement waits per step
    std::string err;
    rc = rbs::device_host_async(plan->p, b, x, k, ld, prec, err);
    if (rc) return fail(rc, "rbs_solve_host_async: " + err);
    return RBS_OK;
}

int rbs_plan_set_stream(rbs_plan *plan, void *stream) {
    if (!plan) return fail(RBS_ERR_ARG, "rbs_plan_set_stream: plan is NULL");
    std::string err;
    int rc = rbs::device_set_stream(plan->p, stream, err);
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_plan_reserve(rbs_plan *plan, int k) {
    if (!plan) return fail(RBS_ERR_ARG, "rbs_plan_reserve: plan is NULL");
    std::string err;
    int rc = rbs::device_reserve(plan->p, k, err);
    if (rc) return fail(rc, "rbs_plan_reserve: " + err);
    return RBS_OK;
}

int rbs_plan_info_get(const rbs_plan *plan, rbs_plan_info *info) {
    if (!plan || !info) return fail(RBS_ERR_ARG, "rbs_plan_info_get: NULL argument");
    const rbs::Plan &P = plan->p;
    std::memset(info, 0, sizeof(*info));
    info->n = P.n;
    info->nnz = P.nnz;
    info->lv = P.lv;
    info->substitution = P.sub;
    info->nlevel = P.nlevel;
    info->sum_block = P.sum_block;
    for (const rbs::ExecBlock &B : P.blocks)
        if (B.kernel >= 0 && B.kernel < 8) info->kernels[B.kernel]++;
    info->device_bytes = rbs::device_bytes(P);
    info->analyse_ms = P.analyse_ms;
    return RBS_OK;
}

int rbs_plan_export(const rbs_plan *plan, const char *name, void *dst, long long cap, long long *count) {
    if (!plan || !name || !count) return fail(RBS_ERR_ARG, "rbs_plan_export: NULL argument");
    std::vector<int> iv;
    std::vector<double> dv;
    bool is_double = false;
    std::string err;
    int rc;
    try {
        rc = rbs::export_reference(plan->p, name, iv, dv, is_double, err);
    } catch (const std::bad_alloc &) {
        return fail(RBS_ERR_NOMEM, "rbs_plan_export: out of host memory");
    }
    if (rc) return fail(rc, err);
    *count = is_double ? (long long)dv.size() : (long long)iv.size();
    if (!dst) return RBS_OK;
    if (cap < *count) return fail(RBS_ERR_ARG, "rbs_plan_export: destination too small");
    if (is_double)
        std::memcpy(dst, dv.data(), dv.size() * sizeof(double));
    else
        std::memcpy(dst, iv.data(), iv.size() * sizeof(int));
    return RBS_OK;
}

int rbs_plan_profile(rbs_plan *plan, int enable) {
    if (!plan) return fail(RBS_ERR_ARG, "rbs_plan_profile: plan is NULL");
    std::string err;
    int rc = rbs::device_profile(plan->p, enable, err);
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_plan_block_times(const rbs_plan *plan, double *ms, double *bytes, long long *solves, int cap) {
    if (!plan || cap < plan->p.sum_block) return fail(RBS_ERR_ARG, "rbs_plan_block_times: bad arguments");
    std::vector<double> v;
    long long s = 0;
    if (rbs::device_block_times(plan->p, v, s)) return fail(RBS_ERR_ARG, "rbs_plan_block_times: no device state");
    for (int b = 0; b < plan->p.sum_block; ++b) {
        if (ms) ms[b] = v[b];
        if (bytes) bytes[b] = rbs::block_bytes(plan->p, plan->p.blocks[b]);
    }
    if (solves) *solves = s;
    return RBS_OK;
}

int rbs_ilu0_device(const int *d_rowptr, const int *d_colidx, const double *d_val, int n, int nnz, double *d_lu,
                    const rbs_options *opt) {
    if (!d_rowptr || !d_colidx || !d_val || !d_lu || n <= 0 || nnz < n)
        return fail(RBS_ERR_ARG, "rbs_ilu0_device: need n > 0, nnz >= n and non-null arrays");
    rbs_options o;
    rbs_options_default(&o);
    if (opt) o = *opt;
    if (o.spin_limit <= 0) o.spin_limit = 1LL << 22;
    std::string err;
    const int rc = rbs::device_ilu0(d_rowptr, d_colidx, d_val, n, nnz, d_lu, o, err);
    if (rc) return fail(rc, err);
    set_error("");
    return RBS_OK;
}

struct rbs_mtx {
    rbs::DeviceMtx m;
};

static int mtx_open(const char *path, const void *bytes, long long len, const rbs_options *opt, rbs_mtx **mtx) {
    if (!mtx) return fail(RBS_ERR_ARG, "rbs_mtx_read: mtx is NULL");
    *mtx = nullptr;
    rbs_options o;
    rbs_options_default(&o);
    if (opt) o = *opt;
    rbs_mtx *h = new (std::nothrow) rbs_mtx;
    if (!h) return fail(RBS_ERR_NOMEM, "rbs_mtx_read: out of host memory");
    std::string err;
    const int rc = rbs::mtx_read(path, bytes, len, o, h->m, err);
    if (rc) {
        delete h;
        return fail(rc, err);
    }
    *mtx = h;
    set_error("");
    return RBS_OK;
}

int rbs_mtx_read(const char *path, const rbs_options *opt, rbs_mtx **mtx) {
    if (!path) return fail(RBS_ERR_ARG, "rbs_mtx_read: path is NULL");
    return mtx_open(path, nullptr, 0, opt, mtx);
}

int rbs_mtx_read_buffer(const void *bytes, long long len, const rbs_options *opt, rbs_mtx **mtx) {
    if ((!bytes && len) || len < 0) return fail(RBS_ERR_ARG, "rbs_mtx_read_buffer: bad buffer");
    return mtx_open(nullptr, bytes, len, opt, mtx);
}

int rbs_mtx_info_get(const rbs_mtx *mtx, rbs_mtx_info *info) {
    if (!mtx || !info) return fail(RBS_ERR_ARG, "rbs_mtx_info_get: NULL argument");
    const rbs::DeviceMtx &M = mtx->m;
    info->m = M.m;
    info->n = M.n;
    info->nnz_file = M.nnz_file;
    info->nnz = M.nnz;
    info->nnz_lower = M.nnz_lower;
    info->nnz_upper = M.nnz_upper;
    info->field = M.field;
    info->symmetric = M.symmetric;
    info->host_values = M.host_values;
    info->read_ms = M.read_ms;
    info->parse_ms = M.parse_ms;
    return RBS_OK;
}

int rbs_mtx_csr(const rbs_mtx *mtx, int *d_rowptr, int *d_colidx, double *d_val) {
    if (!mtx || !d_rowptr || ((!d_colidx || !d_val) && mtx->m.nnz))
        return fail(RBS_ERR_ARG, "rbs_mtx_csr: NULL argument");
    std::string err;
    const int rc = rbs::mtx_csr(mtx->m, d_rowptr, d_colidx, d_val, err);
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_mtx_triangle(const rbs_mtx *mtx, int substitution, int fmt, const double *d_strict_val, int *d_ptr,
                     int *d_idx, double *d_val) {
    if (!mtx || !d_ptr || !d_idx || !d_val) return fail(RBS_ERR_ARG, "rbs_mtx_triangle: NULL argument");
    if (substitution != RBS_FORWARD && substitution != RBS_BACKWARD)
        return fail(RBS_ERR_ARG, "rbs_mtx_triangle: substitution must be RBS_FORWARD or RBS_BACKWARD");
    if (fmt != RBS_FMT_CSC && fmt != RBS_FMT_CSR)
        return fail(RBS_ERR_ARG, "rbs_mtx_triangle: fmt must be RBS_FMT_CSC or RBS_FMT_CSR");
    std::string err;
    const int rc = rbs::mtx_triangle(mtx->m, substitution, fmt, d_strict_val, d_ptr, d_idx, d_val, err);
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_mtx_write(const char *path, int m, int n, const int *rowptr, const int *colidx, const double *val,
                  int symmetric) {
    if (!path || !rowptr || (!colidx && m > 0 && rowptr[m] > 0) || m < 0 || n < 0)
        return fail(RBS_ERR_ARG, "rbs_mtx_write: bad arguments");
    std::string err;
    const int rc = rbs::mtx_write(path, m, n, rowptr, colidx, val, symmetric, err);
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_mtx_free(rbs_mtx *mtx) {
    if (!mtx) return RBS_OK;
    rbs::mtx_free(mtx->m);
    delete mtx;
    return RBS_OK;
}

int rbs_ic0_device(const int *d_rowptr, const int *d_colidx, const double *d_val, int n, int nnz, double *d_l,
                   const rbs_options *opt) {
    if (!d_rowptr || !d_colidx || !d_val || !d_l || n <= 0 || nnz < n)
        return fail(RBS_ERR_ARG, "rbs_ic0_device: need n > 0, nnz >= n and non-null arrays");
    rbs_options o;
    rbs_options_default(&o);
    if (opt) o = *opt;
    if (o.spin_limit <= 0) o.spin_limit = 1LL << 22;
    std::string err;
    const int rc = rbs::device_ic0(d_rowptr, d_colidx, d_val, n, nnz, d_l, o, err);
    if (rc) return fail(rc, err);
    set_error("");
    return RBS_OK;
}

int rbs_plan_save(const rbs_plan *plan, const char *path) {
    if (!plan || !path) return fail(RBS_ERR_ARG, "rbs_plan_save: NULL argument");
    std::string err;
    int rc = rbs::plan_save(plan->p, path, err);
    if (rc) return fail(rc, err);
    return RBS_OK;
}

int rbs_plan_load(const char *path, const rbs_options *opt, rbs_plan **plan) {
    if (!plan || !path) return fail(RBS_ERR_ARG, "rbs_plan_load: NULL argument");
    *plan = nullptr;
    rbs_plan *P = new (std::nothrow) rbs_plan();
    if (!P) return fail(RBS_ERR_NOMEM, "rbs_plan_load: out of host memory");
    std::string err;
    int rc;
    try {
        rc = rbs::plan_load(P->p, path, err);
        if (rc == RBS_OK) {
            // run-time options from the caller; the analysis from the file
            rbs_options o = P->p.opt;
            if (opt) {
                o.device = opt->device;
                o.host_only = opt->host_only;
                o.max_rhs = opt->max_rhs < 1 ? 1 : opt->max_rhs;
                o.mixed = opt->mixed;
                if (opt->ir_tol > 0) o.ir_tol = opt->ir_tol;
                if (opt->ir_max_iter > 0) o.ir_max_iter = opt->ir_max_iter;
                if (opt->spin_limit > 0) o.spin_limit = opt->spin_limit;
            } else {
                o.host_only = 0;
            }
            P->p.opt = o;
            if (!o.host_only) rc = rbs::device_build(P->p, err);
        }
    } catch (const std::bad_alloc &) {
        rc = RBS_ERR_NOMEM;
        err = "rbs_plan_load: out of host memory";
    }
    if (rc != RBS_OK) {
        rbs::device_free(P->p);
        delete P;
        return fail(rc, err);
    }
    *plan = P;
    set_error("");
    return RBS_OK;
}

int rbs_plan_free(rbs_plan *plan) {
    if (!plan) return RBS_OK;
    rbs::device_free(plan->p);
    delete plan;
    return RBS_OK;
}

// ---- reference-signature shims ------------------------------------------

static int bench_repeat() {
    const char *s = std::getenv("RBS_BENCH_REPEAT");  // common.h:13-15 BENCH_REPEAT
    int r = s ? std::atoi(s) : 200;
    return r > 0 ? r : 200;
}

void recblocking_solver_cuda(int *d_cscColPtrTR, int *d_cscRowIdxTR, double *d_cscValTR, int m, int n, int nnzTR,
                             double *d_x, double *d_b, int substitution, int lv, double *cal_time,
                             double *preprocess_time) {
    if (m != n) {
        set_error("recblocking_solver_cuda: matrix must be square");
        return;
    }
    auto t0 = std::chrono::steady_clock::now();
    rbs_plan *plan = nullptr;
    int rc = rbs_analyse_device(d_cscColPtrTR, d_cscRowIdxTR, d_cscValTR, m, nnzTR, RBS_FMT_CSC, substitution, lv,
                                nullptr, &plan);
    auto t1 = std::chrono::steady_clock::now();
    if (rc) return;
    if (preprocess_time) *preprocess_time = std::chrono::duration<double, std::milli>(t1 - t0).count();
    // recblocking_calculate.h:37-167: mean over BENCH_REPEAT solves
    int reps = bench_repeat();
    double total = 0;
    for (int r = 0; r < reps && rc == RBS_OK; ++r) {
        rbs_stats st;
        rc = rbs_solve(plan, d_b, d_x, 1, m, RBS_PREC_FP64, &st);
        total += st.ms;
    }
    if (rc == RBS_OK && cal_time) *cal_time += total / reps;
    rbs_plan_free(plan);
}

void recblocking_solver(int *cscColPtr, int *cscRowIdx, double *cscVal, int m, int n, int nnz, double *b, double *x,
                        double *x_ref, int rhs, int lv, int substitution, double *cal_time) {
    (void)x_ref;
    if (m != n) {
        set_error("recblocking_solver: matrix must be square");
        return;
    }
    rbs_options o;
    rbs_options_default(&o);
    o.max_rhs = rhs > 0 ? rhs : 1;
    rbs_plan *plan = nullptr;
    if (rbs_analyse(cscColPtr, cscRowIdx, cscVal, m, nnz, RBS_FMT_CSC, substitution, lv, &o, &plan)) return;
    rbs_stats st;
    int k = rhs > 0 ? rhs : 1;
    if (rbs_solve_host(plan, b, x, k, m, RBS_PREC_FP64, &st) == RBS_OK && cal_time) *cal_time += st.ms;
    rbs_plan_free(plan);
}

}  // extern "C"
