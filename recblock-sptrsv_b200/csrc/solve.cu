// solve.cu -- executor: device copy of a plan and the solve walk
// (recblocking_calculate.h:15-168 L_calculate / :170-325 U_calculate) with
// no host synchronisation between blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "kernels.cuh"
#include "rbs_internal.h"

namespace rbs {

struct DeviceState {
    int device = 0, num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // plan pools
    int *rp = nullptr, *col = nullptr, *lvl = nullptr, *map = nullptr, *rows = nullptr, *perm = nullptr;
    double *val = nullptr, *inv = nullptr;
    float *val32 = nullptr, *inv32 = nullptr;
    int *full_rp = nullptr, *full_col = nullptr;
    double *full_val = nullptr;
    int *tickets = nullptr, *status = nullptr, *h_status = nullptr;
    int ntri = 0;
    // work vectors for kcap right-hand sides
    int kcap = 0;
    double *bw64 = nullptr, *xw64 = nullptr, *b64keep = nullptr, *x64acc = nullptr;
    float *bw32 = nullptr, *xw32 = nullptr;
    double *norms = nullptr, *h_norms = nullptr;
    std::map<long long, LevelDesc *> desc_cache;
    long long bytes = 0, work_bytes = 0;
    bool mixed = false;
    // per-block timing (rbs_plan_profile)
    bool profile = false;
    std::vector<cudaEvent_t> bev;
    std::vector<double> bms;
    long long bsolves = 0;
    // staging for the host-array API
    double *stage_b = nullptr, *stage_x = nullptr;
    size_t stage_bytes = 0;
    int last_iters = 0;
    double last_corr = 0;
};

namespace {

#define CK(call)                                                                     \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                \
            return RBS_ERR_CUDA;                                                     \
        }                                                                            \
    } while (0)

template <typename T>
int upload(DeviceState &D, T *&dst, const std::vector<T> &src, std::string &err) {
    size_t bytes = std::max<size_t>(src.size(), 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&dst, bytes);
    if (e != cudaSuccess) {
        err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? RBS_ERR_NOMEM : RBS_ERR_CUDA;
    }
    D.bytes += (long long)bytes;
    if (!src.empty()) CK(cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return RBS_OK;
}

template <typename T>
int alloc(DeviceState &D, T *&dst, size_t count, std::string &err) {
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&dst, bytes);
    if (e != cudaSuccess) {
        err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? RBS_ERR_NOMEM : RBS_ERR_CUDA;
    }
    D.bytes += (long long)bytes;
    return RBS_OK;
}

int grid_for(long long work, int threads, int num_sms) {
    long long g = (work + threads - 1) / threads;
    long long cap = (long long)num_sms * 16;
    return (int)std::max(1LL, std::min(g, cap));
}

double sent64_host() {
    unsigned long long bits = RBS_SENT64;
    double v;
    std::memcpy(&v, &bits, 8);
    return v;
}

int pow2_at_least(int k) {
    int K = 1;
    while (K < k) K <<= 1;
    return K;
}

void free_work(DeviceState &D) {
    cudaFree(D.bw64);
    cudaFree(D.xw64);
    cudaFree(D.b64keep);
    cudaFree(D.x64acc);
    cudaFree(D.bw32);
    cudaFree(D.xw32);
    D.bw64 = D.xw64 = D.b64keep = D.x64acc = nullptr;
    D.bw32 = D.xw32 = nullptr;
    for (auto &kv : D.desc_cache) cudaFree(kv.second);
    D.desc_cache.clear();
}

// Work vectors sized for K right-hand sides; solution vectors start filled
// with the sentinel and every solve leaves them that way.
int ensure_work(Plan &P, int K, std::string &err) {
    DeviceState &D = *P.dev;
    if (K <= D.kcap) return RBS_OK;
    free_work(D);
    D.bytes -= D.work_bytes;
    const long long before = D.bytes;
    size_t cnt = (size_t)P.n * K;
    int rc;
    if ((rc = alloc(D, D.bw64, cnt, err))) return rc;
    if ((rc = alloc(D, D.xw64, cnt, err))) return rc;
    k_fill<double><<<grid_for((long long)cnt, 256, D.num_sms), 256, 0, D.stream>>>(
        D.xw64, (long long)cnt, sent64_host());
    if (D.mixed) {
        if ((rc = alloc(D, D.b64keep, cnt, err))) return rc;
        if ((rc = alloc(D, D.x64acc, cnt, err))) return rc;
        if ((rc = alloc(D, D.bw32, cnt, err))) return rc;
        if ((rc = alloc(D, D.xw32, cnt, err))) return rc;
        unsigned s32 = RBS_SENT32;
        float f32;
        std::memcpy(&f32, &s32, 4);
        k_fill<float><<<grid_for((long long)cnt, 256, D.num_sms), 256, 0, D.stream>>>(D.xw32, (long long)cnt, f32);
    }
    CK(cudaGetLastError());
    D.kcap = K;
    D.work_bytes = D.bytes - before;
    return RBS_OK;
}

template <typename VT> struct Pools;
template <> struct Pools<double> {
    static const double *val(const DeviceState &D) { return D.val; }
    static const double *inv(const DeviceState &D) { return D.inv; }
    static double *bw(const DeviceState &D) { return D.bw64; }
    static double *xw(const DeviceState &D) { return D.xw64; }
};
template <> struct Pools<float> {
    static const float *val(const DeviceState &D) { return D.val32; }
    static const float *inv(const DeviceState &D) { return D.inv32; }
    static float *bw(const DeviceState &D) { return D.bw32; }
    static float *xw(const DeviceState &D) { return D.xw32; }
};

template <typename VT, int K>
int level_descs(Plan &P, LevelDesc *&out, std::string &err) {
    DeviceState &D = *P.dev;
    long long key = (long long)K * 4 + (sizeof(VT) == 8 ? 0 : 1);
    auto it = D.desc_cache.find(key);
    if (it != D.desc_cache.end()) {
        out = it->second;
        return RBS_OK;
    }
    std::vector<LevelDesc> h;
    for (const ExecBlock &B : P.blocks) {
        if (!B.tri || B.kernel != RBS_K_LEVEL) continue;
        LevelDesc d{};
        d.rp = D.rp + B.rp_off;
        d.col = D.col;
        d.lvl = D.lvl + B.lvl_off;
        d.map = B.map_off >= 0 ? D.map + B.map_off : nullptr;
        d.val = Pools<VT>::val(D);
        d.inv = Pools<VT>::inv(D) + B.r0;
        d.b = Pools<VT>::bw(D) + (long long)B.r0 * K;
        d.x = Pools<VT>::xw(D) + (long long)B.r0 * K;
        d.m = B.m;
        d.nlv = B.nlv;
        d.G = B.group;
        h.push_back(d);
    }
    LevelDesc *dd = nullptr;
    CK(cudaMalloc(&dd, std::max<size_t>(h.size(), 1) * sizeof(LevelDesc)));
    if (!h.empty()) CK(cudaMemcpy(dd, h.data(), h.size() * sizeof(LevelDesc), cudaMemcpyHostToDevice));
    D.desc_cache[key] = dd;
    out = dd;
    return RBS_OK;
}

template <typename VT, int K>
int syncfree_grid(const DeviceState &D) {
    static int per_sm = -1;
    if (per_sm < 0) {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_tri_syncfree<VT, K>, 256, 0) != cudaSuccess ||
            nb < 1)
            nb = 1;
        per_sm = nb;
    }
    return per_sm * D.num_sms;
}

// One pass over all blocks: triangles solve into xw, squares update bw.
template <typename VT, int K>
int run_blocks(Plan &P, std::string &err) {
    DeviceState &D = *P.dev;
    cudaStream_t st = D.stream;
    const VT *val = Pools<VT>::val(D);
    const VT *inv = Pools<VT>::inv(D);
    VT *bw = Pools<VT>::bw(D);
    VT *xw = Pools<VT>::xw(D);
    LevelDesc *descs = nullptr;
    int rc = level_descs<VT, K>(P, descs, err);
    if (rc) return rc;
    if (D.ntri) CK(cudaMemsetAsync(D.tickets, 0, sizeof(int) * D.ntri, st));
    const long long limit = P.opt.spin_limit;
    int ti = 0, li = 0;
    for (const ExecBlock &B : P.blocks) {
        if (D.profile) CK(cudaEventRecord(D.bev[2 * B.index], st));
        if (B.tri) {
            const VT *bb = bw + (long long)B.r0 * K;
            VT *xx = xw + (long long)B.r0 * K;
            switch (B.kernel) {
            case RBS_K_DIAG:
                k_tri_diag<VT, K><<<grid_for((long long)B.m * K, 256, D.num_sms), 256, 0, st>>>(inv + B.r0, bb, xx,
                                                                                               B.m);
                break;
            case RBS_K_LEVEL:
                k_tri_level<VT, K><<<1, 1024, 0, st>>>(descs + li);
                ++li;
                break;
            case RBS_K_SEQ:
            case RBS_K_BANDSCAN:
                k_tri_seq<VT, K><<<1, 32, 0, st>>>(D.rp + B.rp_off, D.col, val, inv + B.r0, bb, xx, B.m);
                break;
            default: {
                const int g = K == 1 ? B.group : (K < 32 ? K : 32);
                const long long warps = ((long long)B.m * g + 31) / 32;
                int grid = (int)std::min<long long>(syncfree_grid<VT, K>(D), (warps + 7) / 8);
                k_tri_syncfree<VT, K><<<std::max(grid, 1), 256, 0, st>>>(D.rp + B.rp_off, D.col, val, inv + B.r0, bb,
                                                                        xx, B.m, B.group, D.tickets + ti, D.status,
                                                                        limit);
                break;
            }
            }
            ++ti;
        } else if (B.kernel == RBS_K_SPMV) {
            const int g = K == 1 ? B.group : (K < 32 ? K : 32);
            const int *rows = B.rows_off >= 0 ? D.rows + B.rows_off : nullptr;
            k_spmv_sub<VT, K><<<grid_for((long long)B.nrows * g, 256, D.num_sms), 256, 0, st>>>(
                D.rp + B.rp_off, D.col, val, rows, B.nrows, B.group, xw + (long long)B.c0 * K,
                bw + (long long)B.r0 * K, B.longrows > 0);
            if (B.longrows > 0)
                k_spmv_long<VT, K><<<D.num_sms * 2, 256, 0, st>>>(D.rp + B.rp_off, D.col, val, rows,
                                                                  D.rows + B.long_off, B.longrows,
                                                                  xw + (long long)B.c0 * K, bw + (long long)B.r0 * K);
        }
        if (D.profile) CK(cudaEventRecord(D.bev[2 * B.index + 1], st));
    }
    CK(cudaGetLastError());
    return RBS_OK;
}

template <int K>
int solve_fp64(Plan &P, const double *b, double *x, int k, int ld, std::string &err) {
    DeviceState &D = *P.dev;
    const int n = P.n;
    const int grid = grid_for((long long)n * K, 256, D.num_sms);
    k_gather<double, K><<<grid, 256, 0, D.stream>>>(b, ld, k, D.perm, n, D.bw64);
    int rc = run_blocks<double, K>(P, err);
    if (rc) return rc;
    k_scatter_reset<double, K><<<grid, 256, 0, D.stream>>>(D.xw64, D.perm, n, k, x, ld);
    CK(cudaGetLastError());
    return RBS_OK;
}

template <int K>
int solve_fp32(Plan &P, const double *b, double *x, int k, int ld, std::string &err) {
    DeviceState &D = *P.dev;
    const int n = P.n;
    const int grid = grid_for((long long)n * K, 256, D.num_sms);
    k_gather<float, K><<<grid, 256, 0, D.stream>>>(b, ld, k, D.perm, n, D.bw32);
    int rc = run_blocks<float, K>(P, err);
    if (rc) return rc;
    k_scatter_reset<float, K><<<grid, 256, 0, D.stream>>>(D.xw32, D.perm, n, k, x, ld);
    CK(cudaGetLastError());
    return RBS_OK;
}

// FP32 sweeps with FP64 residuals and FP64 accumulation:
//   x0 = L32^-1 b;  repeat  r = b - L x (FP64),  d = L32^-1 r,  x += d
// until ||d||/||x|| <= ir_tol for every right-hand side.
template <int K>
int solve_mixed(Plan &P, const double *b, double *x, int k, int ld, int &iters, double &corr, std::string &err) {
    DeviceState &D = *P.dev;
    const int n = P.n;
    const int grid = grid_for((long long)n * K, 256, D.num_sms);
    k_gather<double, K><<<grid, 256, 0, D.stream>>>(b, ld, k, D.perm, n, D.b64keep);
    k_gather<float, K><<<grid, 256, 0, D.stream>>>(b, ld, k, D.perm, n, D.bw32);
    int rc = run_blocks<float, K>(P, err);
    if (rc) return rc;
    CK(cudaMemsetAsync(D.norms, 0, sizeof(double) * 2 * K, D.stream));
    k_update<K><<<grid_for((long long)n * K, 256, D.num_sms), 256, 0, D.stream>>>(D.x64acc, D.xw32, n, 1, D.norms);
    const int G = P.nnz / std::max(1, n) < 6 ? 4 : 8;
    iters = 0;
    corr = 1.0;
    for (int it = 0; it < P.opt.ir_max_iter; ++it) {
        k_residual<K><<<grid_for((long long)n * (K == 1 ? G : std::min(K, 32)), 256, D.num_sms), 256, 0, D.stream>>>(
            D.full_rp, D.full_col, D.full_val, D.x64acc, D.b64keep, D.bw32, n, G);
        rc = run_blocks<float, K>(P, err);
        if (rc) return rc;
        CK(cudaMemsetAsync(D.norms, 0, sizeof(double) * 2 * K, D.stream));
        k_update<K><<<grid_for((long long)n * K, 256, D.num_sms), 256, 0, D.stream>>>(D.x64acc, D.xw32, n, 0,
                                                                                        D.norms);
        CK(cudaMemcpyAsync(D.h_norms, D.norms, sizeof(double) * 2 * K, cudaMemcpyDeviceToHost, D.stream));
        CK(cudaStreamSynchronize(D.stream));
        ++iters;
        corr = 0;
        for (int c = 0; c < k; ++c) {
            double dn = std::sqrt(D.h_norms[c]), xn = std::sqrt(D.h_norms[K + c]);
            double r = xn > 0 ? dn / xn : dn;
            if (!(r <= corr)) corr = r;  // NaN-propagating max
        }
        if (corr <= P.opt.ir_tol) break;
    }
    k_scatter64<K><<<grid, 256, 0, D.stream>>>(D.x64acc, D.perm, n, k, x, ld);
    CK(cudaGetLastError());
    if (!(corr <= P.opt.ir_tol)) {
        err = "mixed-precision refinement stopped at ||dx||/||x|| = " + std::to_string(corr);
        return RBS_ERR_NOCONV;
    }
    return RBS_OK;
}

template <int K>
int solve_k(Plan &P, const double *b, double *x, int k, int ld, int prec, int &iters, double &corr,
            std::string &err) {
    if (prec == RBS_PREC_FP64) return solve_fp64<K>(P, b, x, k, ld, err);
    if (prec == RBS_PREC_FP32) return solve_fp32<K>(P, b, x, k, ld, err);
    return solve_mixed<K>(P, b, x, k, ld, iters, corr, err);
}

}  // namespace

int device_build(Plan &P, std::string &err) {
    if (P.dev) device_free(P);
    P.dev = new DeviceState();
    DeviceState &D = *P.dev;
    if (P.opt.device >= 0) CK(cudaSetDevice(P.opt.device));
    CK(cudaGetDevice(&D.device));
    CK(cudaDeviceGetAttribute(&D.num_sms, cudaDevAttrMultiProcessorCount, D.device));
    CK(cudaStreamCreateWithFlags(&D.stream, cudaStreamNonBlocking));
    D.own_stream = true;
    CK(cudaEventCreate(&D.ev0));
    CK(cudaEventCreate(&D.ev1));
    int rc;
    if ((rc = upload(D, D.rp, P.rp_pool, err))) return rc;
    if ((rc = upload(D, D.col, P.col_pool, err))) return rc;
    if ((rc = upload(D, D.val, P.val_pool, err))) return rc;
    if ((rc = upload(D, D.lvl, P.lvl_pool, err))) return rc;
    if ((rc = upload(D, D.map, P.map_pool, err))) return rc;
    if ((rc = upload(D, D.rows, P.rows_pool, err))) return rc;
    if ((rc = upload(D, D.perm, P.perm, err))) return rc;
    if ((rc = upload(D, D.inv, P.inv_diag, err))) return rc;
    D.mixed = P.opt.mixed != 0;
    if (D.mixed) {
        std::vector<float> v32(P.val_pool.size()), i32(P.inv_diag.size());
        for (size_t i = 0; i < v32.size(); ++i) v32[i] = (float)P.val_pool[i];
        for (size_t i = 0; i < i32.size(); ++i) i32[i] = (float)P.inv_diag[i];
        if ((rc = upload(D, D.val32, v32, err))) return rc;
        if ((rc = upload(D, D.inv32, i32, err))) return rc;
        if ((rc = upload(D, D.full_rp, P.full_rp, err))) return rc;
        if ((rc = upload(D, D.full_col, P.full_col, err))) return rc;
        if ((rc = upload(D, D.full_val, P.full_val, err))) return rc;
    }
    D.ntri = 1 << P.lv;
    if ((rc = alloc(D, D.tickets, (size_t)D.ntri, err))) return rc;
    if ((rc = alloc(D, D.status, 1, err))) return rc;
    if ((rc = alloc(D, D.norms, 2 * 128, err))) return rc;
    CK(cudaMallocHost(&D.h_status, sizeof(int)));
    CK(cudaMallocHost(&D.h_norms, sizeof(double) * 2 * 128));
    CK(cudaMemsetAsync(D.status, 0, sizeof(int), D.stream));
    if ((rc = ensure_work(P, pow2_at_least(std::max(1, std::min(P.opt.max_rhs, 128))), err))) return rc;
    CK(cudaStreamSynchronize(D.stream));
    return RBS_OK;
}

int device_profile(Plan &P, int enable, std::string &err) {
    if (!P.dev) {
        err = "plan has no device state";
        return RBS_ERR_ARG;
    }
    DeviceState &D = *P.dev;
    CK(cudaStreamSynchronize(D.stream));
    if (enable && D.bev.empty()) {
        D.bev.resize(2 * P.blocks.size());
        for (auto &e : D.bev) CK(cudaEventCreate(&e));
    }
    D.profile = enable != 0;
    D.bms.assign(P.blocks.size(), 0.0);
    D.bsolves = 0;
    return RBS_OK;
}

int device_block_times(const Plan &P, std::vector<double> &ms, long long &solves) {
    if (!P.dev) return RBS_ERR_ARG;
    ms = P.dev->bms;
    ms.resize(P.blocks.size(), 0.0);
    solves = P.dev->bsolves;
    return RBS_OK;
}

int device_staging(Plan &P, size_t bytes, double *&db, double *&dx, std::string &err) {
    DeviceState &D = *P.dev;
    if (bytes > D.stage_bytes) {
        cudaFree(D.stage_b);
        cudaFree(D.stage_x);
        D.stage_b = D.stage_x = nullptr;
        D.bytes -= 2 * (long long)D.stage_bytes;
        D.stage_bytes = 0;
        int rc;
        if ((rc = alloc(D, D.stage_b, bytes / sizeof(double), err))) return rc;
        if ((rc = alloc(D, D.stage_x, bytes / sizeof(double), err))) return rc;
        D.stage_bytes = bytes;
    }
    db = D.stage_b;
    dx = D.stage_x;
    return RBS_OK;
}

void device_free(Plan &P) {
    if (!P.dev) return;
    DeviceState &D = *P.dev;
    if (D.stream) cudaStreamSynchronize(D.stream);
    free_work(D);
    for (auto &e : D.bev) cudaEventDestroy(e);
    cudaFree(D.stage_b);
    cudaFree(D.stage_x);
    void *ptrs[] = {D.rp, D.col, D.lvl, D.map, D.rows, D.perm, D.val, D.inv, D.val32, D.inv32,
                    D.full_rp, D.full_col, D.full_val, D.tickets, D.status, D.norms};
    for (void *p : ptrs) cudaFree(p);
    if (D.h_status) cudaFreeHost(D.h_status);
    if (D.h_norms) cudaFreeHost(D.h_norms);
    if (D.ev0) cudaEventDestroy(D.ev0);
    if (D.ev1) cudaEventDestroy(D.ev1);
    if (D.own_stream && D.stream) cudaStreamDestroy(D.stream);
    delete P.dev;
    P.dev = nullptr;
}

long long device_bytes(const Plan &P) { return P.dev ? P.dev->bytes : 0; }

int device_set_stream(Plan &P, void *stream, std::string &err) {
    if (!P.dev) {
        err = "plan has no device state";
        return RBS_ERR_ARG;
    }
    DeviceState &D = *P.dev;
    CK(cudaStreamSynchronize(D.stream));
    if (D.own_stream) CK(cudaStreamDestroy(D.stream));
    if (stream) {
        D.stream = (cudaStream_t)stream;
        D.own_stream = false;
    } else {
        CK(cudaStreamCreateWithFlags(&D.stream, cudaStreamNonBlocking));
        D.own_stream = true;
    }
    return RBS_OK;
}

int device_sync(Plan &P, std::string &err) {
    DeviceState &D = *P.dev;
    CK(cudaMemcpyAsync(D.h_status, D.status, sizeof(int), cudaMemcpyDeviceToHost, D.stream));
    CK(cudaStreamSynchronize(D.stream));
    if (*D.h_status & RBS_STATUS_TIMEOUT) {
        CK(cudaMemsetAsync(D.status, 0, sizeof(int), D.stream));
        // the solution work vector may hold leftovers of the aborted solve
        size_t cnt = (size_t)P.n * D.kcap;
        k_fill<double><<<grid_for((long long)cnt, 256, D.num_sms), 256, 0, D.stream>>>(
            D.xw64, (long long)cnt, sent64_host());
        CK(cudaStreamSynchronize(D.stream));
        err = "a device wait exceeded its poll budget (dependency never produced)";
        return RBS_ERR_TIMEOUT;
    }
    return RBS_OK;
}

void *device_stream(Plan &P) { return P.dev ? (void *)P.dev->stream : nullptr; }

int device_solve(Plan &P, const double *d_b, double *d_x, int k, int ld, int prec, bool sync, rbs_stats *stats,
                 std::string &err) {
    if (!P.dev) {
        err = "plan was analysed with host_only; it has no device state";
        return RBS_ERR_ARG;
    }
    if (prec != RBS_PREC_FP64 && !P.dev->mixed) {
        err = "plan was built without FP32 copies (options.mixed = 0)";
        return RBS_ERR_UNSUPPORTED;
    }
    DeviceState &D = *P.dev;
    int iters = 0;
    double corr = 0;
    int rc = RBS_OK;
    CK(cudaEventRecord(D.ev0, D.stream));
    for (int c0 = 0; c0 < k && rc == RBS_OK; c0 += 128) {
        int kk = std::min(128, k - c0);
        int K = pow2_at_least(kk);
        if ((rc = ensure_work(P, K, err))) break;
        const double *b = d_b + (long long)c0 * ld;
        double *x = d_x + (long long)c0 * ld;
        int it = 0;
        double cr = 0;
        switch (K) {
        case 1: rc = solve_k<1>(P, b, x, kk, ld, prec, it, cr, err); break;
        case 2: rc = solve_k<2>(P, b, x, kk, ld, prec, it, cr, err); break;
        case 4: rc = solve_k<4>(P, b, x, kk, ld, prec, it, cr, err); break;
        case 8: rc = solve_k<8>(P, b, x, kk, ld, prec, it, cr, err); break;
        case 16: rc = solve_k<16>(P, b, x, kk, ld, prec, it, cr, err); break;
        case 32: rc = solve_k<32>(P, b, x, kk, ld, prec, it, cr, err); break;
        case 64: rc = solve_k<64>(P, b, x, kk, ld, prec, it, cr, err); break;
        default: rc = solve_k<128>(P, b, x, kk, ld, prec, it, cr, err); break;
        }
        iters = std::max(iters, it);
        corr = std::max(corr, cr);
    }
    CK(cudaEventRecord(D.ev1, D.stream));
    D.last_iters = iters;
    D.last_corr = corr;
    if (!sync) return rc;
    int rc2 = device_finish(P, stats, k, prec, err);
    return rc != RBS_OK ? rc : rc2;
}

int device_finish(Plan &P, rbs_stats *stats, int k, int prec, std::string &err) {
    DeviceState &D = *P.dev;
    int rc = device_sync(P, err);
    if (rc == RBS_OK && D.profile && prec != RBS_PREC_MIXED && k <= 128) {
        for (size_t b = 0; b < P.blocks.size(); ++b) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, D.bev[2 * b], D.bev[2 * b + 1]) == cudaSuccess) D.bms[b] += ms;
        }
        ++D.bsolves;
    }
    if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, D.ev0, D.ev1);
        const int iters = D.last_iters;
        stats->ms = ms;
        stats->iterations = iters;
        stats->correction = D.last_corr;
        double n = P.n, nnz = P.nnz;
        stats->useful_bytes = nnz * 12.0 + 4.0 * (n + 1) + 16.0 * n * k;
        if (prec == RBS_PREC_FP64)
            stats->moved_bytes = stats->useful_bytes;
        else if (prec == RBS_PREC_FP32)
            stats->moved_bytes = nnz * 8.0 + 4.0 * (n + 1) + 8.0 * n * k * 2;
        else
            stats->moved_bytes = (iters + 1) * (nnz * 8.0 + 4.0 * (n + 1) + 8.0 * n * k * 2) +
                                 iters * (nnz * 12.0 + 4.0 * (n + 1) + 8.0 * n * k * 3);
    }
    return rc;
}

}  // namespace rbs
