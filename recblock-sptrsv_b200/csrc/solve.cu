// solve.cu -- executor: device copy of a plan and the solve walk
// (recblocking_calculate.h:15-168 L_calculate / :170-325 U_calculate) with
// no host synchronisation between blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <type_traits>
#include <vector>

#include "band.cuh"
#include "kernels.cuh"
#include "cta_syncfree.cuh"
#include "level_ca.cuh"
#include "level_lc.cuh"
#include "rbs_internal.h"

namespace rbs {

// Kernel attributes (the dynamic shared-memory limit) belong to a device
// context: set them once per device, tracked by one bit per device.
inline bool attr_done(const std::atomic<unsigned long long> &seen) {
    int dev = 0;
    cudaGetDevice(&dev);
    return (seen.load() >> (dev & 63)) & 1ULL;
}
inline void attr_mark(std::atomic<unsigned long long> &seen) {
    int dev = 0;
    cudaGetDevice(&dev);
    seen.fetch_or(1ULL << (dev & 63));
}

static_assert(RBS_MEDROW == SQ_MEDROW && RBS_LONGROW == SQ_LONGROW, "the squares' row classes of analysis and kernels");

struct DeviceState {
    int device = 0, num_sms = 148;
    int smem_sm = 233472, smem_reserved = 1024;  // shared memory per SM, reserved per CTA
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // plan pools
    int *rp = nullptr, *col = nullptr, *lvl = nullptr, *map = nullptr, *rows = nullptr, *perm = nullptr;
    int *ipos = nullptr;  // original row -> processing position (inverse of perm)
    double *val = nullptr, *inv = nullptr;
    float *val32 = nullptr, *inv32 = nullptr;
    int *full_rp = nullptr, *full_col = nullptr;
    double *full_val = nullptr;
    double *band_coef = nullptr, *band_inv = nullptr;   // band-scan layout (f64)
    float *band_coef32 = nullptr, *band_inv32 = nullptr;
    double *band_maps = nullptr, *band_states = nullptr; // scratch of the band scan (f64 or f32), kcap columns
    size_t band_maps1 = 1, band_states1 = 1;             // ... elements per column
    int *ell_col = nullptr;
    double *ell_val = nullptr;
    float *ell_val32 = nullptr;
    EllChunk *ell_chunks = nullptr;
    std::map<long long, CsfDesc *> ell_cache;
    int *ca_tab = nullptr, *ca_col = nullptr;
    short *ca_col16 = nullptr;  // window-slot columns of WIN blocks with W >= 2 (16-bit copy of ca_col)
    double *ca_val = nullptr;
    float *ca_val32 = nullptr;
    std::map<long long, CaDesc *> ca_cache;
    uint32_t *lc_rec64 = nullptr, *lc_rec32 = nullptr;  // level-chunk records (16-byte aligned words)
    LcChunk *lc_tab = nullptr;
    LcSeg *lc_segs = nullptr;
    int *lc_queue = nullptr;                              // one segment counter per triangle
    cudaStream_t side = nullptr;                         // L2 prefetch stream; moves of the overlapped walk
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    double **iotab = nullptr;                            // caller's columns for the overlapped walk (k_set_io)
    int *io_rows = nullptr;                              // per triangle, its original rows ascending (n entries)
    // x work vector left without its sentinel by an overlapped walk (which
    // polls nothing); refilled before the next walk of that precision
    bool xw_dirty64 = false, xw_dirty32 = false;
    std::vector<cudaEvent_t> ov_ev;                      // per-triangle events of the overlapped walk
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
    // asynchronous host-array solves (device_host_async): two staging slots
    // used in turn, uploads on `cin`, downloads on `cout`, so one call's
    // copies overlap the neighbouring calls' solves
    struct HostPipe {
        cudaStream_t cin = nullptr, cout = nullptr;
        cudaEvent_t in_done[2] = {nullptr, nullptr}, solved[2] = {nullptr, nullptr}, out_done[2] = {nullptr, nullptr};
        double *db[2] = {nullptr, nullptr}, *dx[2] = {nullptr, nullptr};
        size_t bytes = 0;
        int next = 0;
        bool used[2] = {false, false};
    } pipe;
    int last_iters = 0;
    double last_corr = 0;
    // the asynchronous batch in flight (device_batch_*)
    int bat_K = 0, bat_k = 0, bat_prec = 0, bat_iters = 0;
    double bat_corr = 0;
    double *const *bat_xcols = nullptr;
    GroupCols bat_gx{};  // the batch's solution tables when it spans the systems of a block-diagonal plan
    // captured block walks per (precision, K, profiling)
    bool use_graphs = true;
    std::map<long long, cudaGraphExec_t> graphs;
    std::set<long long> graph_seen;
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

template <typename T, typename A>
int upload(DeviceState &D, T *&dst, const std::vector<T, A> &src, std::string &err) {
    // 256 bytes of padding: staged bulk copies round their end up to 16 bytes
    size_t bytes = std::max<size_t>(src.size(), 1) * sizeof(T) + 256;
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
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T) + 256;
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
    cudaFree(D.band_maps);
    cudaFree(D.band_states);
    D.band_maps = D.band_states = nullptr;
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
    for (auto &kv : D.ell_cache) cudaFree(kv.second);
    D.ell_cache.clear();
    for (auto &kv : D.ca_cache) cudaFree(kv.second);
    D.ca_cache.clear();
}

void drop_graphs_fwd(DeviceState &D);

float sent32_host() {
    unsigned bits = RBS_SENT32;
    float v;
    std::memcpy(&v, &bits, 4);
    return v;
}

// Work vectors sized for K right-hand sides; solution vectors start filled
// with the sentinel and every solve leaves them that way.  Growing frees the
// old vectors and every captured block walk that points into them; if an
// allocation fails, the plan is left with no work vectors at all (kcap 0),
// so the next solve allocates again instead of running on freed memory.
int ensure_work(Plan &P, int K, std::string &err) {
    DeviceState &D = *P.dev;
    if (K <= D.kcap) return RBS_OK;
    // the old vectors may still be read by work queued on the stream
    CK(cudaStreamSynchronize(D.stream));
    drop_graphs_fwd(D);
    free_work(D);
    D.bytes -= D.work_bytes;
    D.work_bytes = 0;
    D.kcap = 0;
    const long long before = D.bytes;
    const size_t cnt = (size_t)P.n * K;
    auto undo = [&](int rc) {
        free_work(D);
        D.bytes = before;
        return rc;
    };
    int rc;
    if ((rc = alloc(D, D.bw64, cnt, err))) return undo(rc);
    if ((rc = alloc(D, D.xw64, cnt, err))) return undo(rc);
    if (D.mixed) {
        if ((rc = alloc(D, D.b64keep, cnt, err))) return undo(rc);
        if ((rc = alloc(D, D.x64acc, cnt, err))) return undo(rc);
        if ((rc = alloc(D, D.bw32, cnt, err))) return undo(rc);
        if ((rc = alloc(D, D.xw32, cnt, err))) return undo(rc);
    }
    if ((rc = alloc(D, D.band_maps, D.band_maps1 * K, err))) return undo(rc);
    if ((rc = alloc(D, D.band_states, D.band_states1 * K, err))) return undo(rc);
    k_fill<double><<<grid_for((long long)cnt, 256, D.num_sms), 256, 0, D.stream>>>(D.xw64, (long long)cnt,
                                                                                    sent64_host());
    if (D.mixed)
        k_fill<float><<<grid_for((long long)cnt, 256, D.num_sms), 256, 0, D.stream>>>(D.xw32, (long long)cnt,
                                                                                       sent32_host());
    D.xw_dirty64 = D.xw_dirty32 = false;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("ensure_work: ") + cudaGetErrorString(e);
        return undo(RBS_ERR_CUDA);
    }
    D.kcap = K;
    D.work_bytes = D.bytes - before;
    return RBS_OK;
}

template <typename VT> struct Pools;
template <> struct Pools<double> {
    static const double *val(const DeviceState &D) { return D.val; }
    static const double *inv(const DeviceState &D) { return D.inv; }
    static const double *bcoef(const DeviceState &D) { return D.band_coef; }
    static const double *binv(const DeviceState &D) { return D.band_inv; }
    static const double *ellv(const DeviceState &D) { return D.ell_val; }
    static const double *cav(const DeviceState &D) { return D.ca_val; }
    static const unsigned char *lcrec(const DeviceState &D) { return reinterpret_cast<const unsigned char *>(D.lc_rec64); }
    static double *bw(const DeviceState &D) { return D.bw64; }
    static double *xw(const DeviceState &D) { return D.xw64; }
    static bool &dirty(DeviceState &D) { return D.xw_dirty64; }
    static double sent() { return sent64_host(); }
};
template <> struct Pools<float> {
    static const float *val(const DeviceState &D) { return D.val32; }
    static const float *inv(const DeviceState &D) { return D.inv32; }
    static const float *bcoef(const DeviceState &D) { return D.band_coef32; }
    static const float *binv(const DeviceState &D) { return D.band_inv32; }
    static const float *ellv(const DeviceState &D) { return D.ell_val32; }
    static const float *cav(const DeviceState &D) { return D.ca_val32; }
    static const unsigned char *lcrec(const DeviceState &D) { return reinterpret_cast<const unsigned char *>(D.lc_rec32); }
    static float *bw(const DeviceState &D) { return D.bw32; }
    static float *xw(const DeviceState &D) { return D.xw32; }
    static bool &dirty(DeviceState &D) { return D.xw_dirty32; }
    static float sent() { return sent32_host(); }
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

template <typename VT>
int ell_descs(Plan &P, CsfDesc *&out, std::string &err) {
    DeviceState &D = *P.dev;
    long long key = sizeof(VT) == 8 ? 0 : 1;
    auto it = D.ell_cache.find(key);
    if (it != D.ell_cache.end()) {
        out = it->second;
        return RBS_OK;
    }
    std::vector<CsfDesc> h;
    for (const ExecBlock &B : P.blocks) {
        if (!B.tri || B.kernel != RBS_K_LEVEL || !B.ell_ok) continue;
        CsfDesc d{};
        d.col = D.ell_col;
        d.val = Pools<VT>::ellv(D);
        d.inv = Pools<VT>::inv(D) + B.r0;
        d.b = Pools<VT>::bw(D) + B.r0;
        d.x = Pools<VT>::xw(D) + B.r0;
        d.chunks = D.ell_chunks + B.ell_chunk_off;
        d.m = B.m;
        d.nchunks = B.ell_nchunks;
        d.G = B.group;
        h.push_back(d);
    }
    CsfDesc *dd = nullptr;
    CK(cudaMalloc(&dd, std::max<size_t>(h.size(), 1) * sizeof(CsfDesc)));
    if (!h.empty()) CK(cudaMemcpy(dd, h.data(), h.size() * sizeof(CsfDesc), cudaMemcpyHostToDevice));
    D.ell_cache[key] = dd;
    out = dd;
    if (!h.empty()) {
        static std::atomic<unsigned long long> attr{0};
        if (!attr_done(attr)) {
            CK(cudaFuncSetAttribute(k_tri_cta_syncfree<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)CsfLayout<VT>::total));
            attr_mark(attr);
        }
    }
    return RBS_OK;
}

template <typename VT, int W, int S, int G = 1, bool MC = false>
int ca_attr(std::string &err) {
    static std::atomic<unsigned long long> done{0};
    if (!attr_done(done)) {
        CK(cudaFuncSetAttribute(k_tri_level_ca<VT, W, S, false, G, MC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)ca_smem_total<VT, W, S, false, G>()));
        CK(cudaFuncSetAttribute(k_tri_level_ca<VT, W, S, true, G, MC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)ca_smem_total<VT, W, S, true, G>()));
        if constexpr (S == 4) {
            CK(cudaFuncSetAttribute(k_tri_level_ca<VT, W, S, false, G, MC, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ca_smem_total<VT, W, S, false, G>()));
            CK(cudaFuncSetAttribute(k_tri_level_ca<VT, W, S, true, G, MC, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ca_smem_total<VT, W, S, true, G>()));
        }
        attr_mark(done);
    }
    return RBS_OK;
}

// Stage counts of the staged level kernel per (value type, ELL width W,
// right-hand sides per CTA G): the deepest staging that fits the 227 KB of
// shared memory next to the x window of G values per slot.
template <typename VT> constexpr int ca_stages(int W, int G) {
    if (G == 1) return W == 4 ? 2 : 4;
    if (sizeof(VT) == 8) return W == 4 ? 0 : 2;  // 0: no such kernel
    return W == 4 ? 2 : 4;
}

// Right-hand sides per CTA of a staged level triangle solved for K columns.
// One column per CTA walks a level fastest (half the shared-memory traffic
// per row), but every CTA reads the same level's rows at the same moment,
// so the L2 lines holding them serve one request per CTA: past about 32
// CTAs a solve's time grows with their number.  On the 2D Laplacian
// (n = 1M, FP64), one column per CTA against two: k = 16 14.7k against
// 11.1k solves/s, k = 32 25.9k against 20.6k, k = 48 23.7k against 28.4k,
// k = 64 28.1k against 36.2k, k = 128 29.7k against 55.8k.  RBS_CA_GROUP
// (1 or 2) overrides the choice.
template <typename VT> int ca_group(const ExecBlock &B, int K) {
    if (K == 1) return 1;
    static const int forced = [] {
        const char *e = std::getenv("RBS_CA_GROUP");
        return e ? std::atoi(e) : 0;
    }();
    int G = forced == 1 || forced == 2 ? forced : K <= 32 ? 1 : 2;
    if (G == 2 && ca_stages<VT>(B.ca_w, 2) == 0) G = 1;
    return G;
}

// Layout of a K-column solve's work vectors: 0 = row-interleaved (entry
// (p, c) at p*K + c), G > 0 = grouped by column groups of G (group c/G's
// rows contiguous, G values each), taken when every triangle is a staged
// level triangle or diagonal-only, so that each CTA's copies coalesce; G is
// then the plan's columns per CTA.
template <typename VT> int plan_group(const Plan &P, int K) {
    if (K == 1) return 0;
    int G = 2;
    for (const ExecBlock &B : P.blocks) {
        if (!B.tri || B.nnz == B.m) continue;
        if (B.kernel != RBS_K_LEVEL || !B.ca_ok) return 0;
        G = std::min(G, ca_group<VT>(B, K));
    }
    return G;
}

template <typename VT>
int ca_descs(Plan &P, CaDesc *&out, int K, int GL, std::string &err) {
    DeviceState &D = *P.dev;
    const long long key = ((long long)K * 2 + (sizeof(VT) == 8 ? 0 : 1)) * 4 + GL;
    auto it = D.ca_cache.find(key);
    if (it != D.ca_cache.end()) {
        out = it->second;
        return RBS_OK;
    }
    std::vector<CaDesc> h;
    for (const ExecBlock &B : P.blocks) {
        if (!B.tri || B.kernel != RBS_K_LEVEL || !B.ca_ok) continue;
        CaDesc d{};
        d.col = B.ca_win && B.ca_w >= 2 ? static_cast<const void *>(D.ca_col16 + B.ca_lo)
                                        : static_cast<const void *>(D.ca_col + B.ca_lo);
        d.val = Pools<VT>::cav(D) + B.ca_lo;
        d.inv = Pools<VT>::inv(D) + B.r0;
        const long long rowlen = GL ? GL : K;  // values per row within a column group's rows
        d.b = Pools<VT>::bw(D) + (long long)B.r0 * rowlen;
        d.x = Pools<VT>::xw(D) + (long long)B.r0 * rowlen;
        d.lvl = D.ca_tab + B.ca_tab_off;
        d.m = B.m;
        d.nlv = B.nlv;
        d.ld = (int)rowlen;
        d.gstride = GL ? (long long)P.n * GL : ca_group<VT>(B, K);
        h.push_back(d);
    }
    CaDesc *dd = nullptr;
    CK(cudaMalloc(&dd, std::max<size_t>(h.size(), 1) * sizeof(CaDesc)));
    if (!h.empty()) CK(cudaMemcpy(dd, h.data(), h.size() * sizeof(CaDesc), cudaMemcpyHostToDevice));
    D.ca_cache[key] = dd;
    out = dd;
    int rc;
    if ((rc = ca_attr<VT, 1, 4>(err)) || (rc = ca_attr<VT, 2, 4>(err)) || (rc = ca_attr<VT, 4, 2>(err))) return rc;
    if (K > 1) {
        if ((rc = ca_attr<VT, 1, 4, 1, true>(err)) || (rc = ca_attr<VT, 2, 4, 1, true>(err)) ||
            (rc = ca_attr<VT, 4, 2, 1, true>(err)))
            return rc;
        if constexpr (sizeof(VT) == 8) {
            if ((rc = ca_attr<VT, 1, 2, 2, true>(err)) || (rc = ca_attr<VT, 2, 2, 2, true>(err))) return rc;
        } else {
            if ((rc = ca_attr<VT, 1, 4, 2, true>(err)) || (rc = ca_attr<VT, 2, 4, 2, true>(err)) ||
                (rc = ca_attr<VT, 4, 2, 2, true>(err)))
                return rc;
        }
    }
    return RBS_OK;
}

// One staged level triangle: one thread per row of the widest level, one
// CTA per group of G right-hand sides.
template <typename VT, int W, int S, int G, bool MC>
void launch_ca(const ExecBlock &B, const CaDesc *desc, int K, cudaStream_t st) {
    const int nt = std::min(1024, std::max(32, (B.maxwidth + 31) / 32 * 32));
    const dim3 grid(1, K / G);
    if constexpr (S == 4) {
        // triangles of wide levels (a mean of 384 rows or more) take the late
        // copies and the register read-ahead
        if (B.m >= 384LL * std::max(1, B.nlv)) {
            if (B.ca_win)
                k_tri_level_ca<VT, W, S, true, G, MC, true><<<grid, nt, ca_smem_total<VT, W, S, true, G>(), st>>>(desc);
            else
                k_tri_level_ca<VT, W, S, false, G, MC, true><<<grid, nt, ca_smem_total<VT, W, S, false, G>(), st>>>(
                    desc);
            return;
        }
    }
    if (B.ca_win)
        k_tri_level_ca<VT, W, S, true, G, MC><<<grid, nt, ca_smem_total<VT, W, S, true, G>(), st>>>(desc);
    else
        k_tri_level_ca<VT, W, S, false, G, MC><<<grid, nt, ca_smem_total<VT, W, S, false, G>(), st>>>(desc);
}

template <typename VT>
void launch_ca_any(const ExecBlock &B, const CaDesc *desc, int K, int G, cudaStream_t st) {
    if (K == 1) {
        if (B.ca_w == 1) launch_ca<VT, 1, 4, 1, false>(B, desc, K, st);
        else if (B.ca_w == 2) launch_ca<VT, 2, 4, 1, false>(B, desc, K, st);
        else launch_ca<VT, 4, 2, 1, false>(B, desc, K, st);
    } else if (G == 1) {
        if (B.ca_w == 1) launch_ca<VT, 1, 4, 1, true>(B, desc, K, st);
        else if (B.ca_w == 2) launch_ca<VT, 2, 4, 1, true>(B, desc, K, st);
        else launch_ca<VT, 4, 2, 1, true>(B, desc, K, st);
    } else if constexpr (sizeof(VT) == 8) {
        if (B.ca_w == 1) launch_ca<VT, 1, 2, 2, true>(B, desc, K, st);
        else launch_ca<VT, 2, 2, 2, true>(B, desc, K, st);
    } else {
        if (B.ca_w == 1) launch_ca<VT, 1, 4, 2, true>(B, desc, K, st);
        else if (B.ca_w == 2) launch_ca<VT, 2, 4, 2, true>(B, desc, K, st);
        else launch_ca<VT, 4, 2, 2, true>(B, desc, K, st);
    }
}

// Shared memory of the staged level kernel as launch_ca_any picks it
// (window blocks with W >= 2 stage 16-bit columns).
template <typename VT, int W, int S, int G>
size_t ca_total(bool win) {
    return win ? ca_smem_total<VT, W, S, true, G>() : ca_smem_total<VT, W, S, false, G>();
}

template <typename VT>
size_t ca_smem_bytes(int W, bool win, int K, int G) {
    if (K == 1 || G == 1) {
        if (W == 1) return ca_total<VT, 1, 4, 1>(win);
        if (W == 2) return ca_total<VT, 2, 4, 1>(win);
        return ca_total<VT, 4, 2, 1>(win);
    }
    if constexpr (sizeof(VT) == 8) {
        return W == 1 ? ca_total<VT, 1, 2, 2>(win) : ca_total<VT, 2, 2, 2>(win);
    } else {
        if (W == 1) return ca_total<VT, 1, 4, 2>(win);
        if (W == 2) return ca_total<VT, 2, 4, 2>(win);
        return ca_total<VT, 4, 2, 2>(win);
    }
}

template <typename VT>
constexpr int lc_smem() {
    return LC_RING + LC_XW * (int)sizeof(VT) + LC_NB * 8;
}
template <typename VT>
int lc_attr(std::string &err) {
    static std::atomic<unsigned long long> done{0};
    if (!attr_done(done)) {
        CK(cudaFuncSetAttribute(k_tri_lc<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize, lc_smem<VT>()));
        attr_mark(done);
    }
    return RBS_OK;
}

// Prefetch [p, p+bytes) into L2 with bulk prefetches of 16 KB.
__global__ void k_prefetch_l2(const char *p, long long bytes) {
    const long long piece = 16384;
    for (long long off = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * piece; off < bytes;
         off += (long long)gridDim.x * blockDim.x * piece) {
        const unsigned n = (unsigned)(((bytes - off < piece ? bytes - off : piece) + 15) & ~15ll);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p + off), "r"(n) : "memory");
    }
}

void prefetch_range(cudaStream_t st, const void *base, long long bytes) {
    if (bytes <= 0) return;
    const char *a = (const char *)((unsigned long long)base & ~15ull);
    bytes += (const char *)base - a;
    const long long pieces = (bytes + 16383) / 16384;
    const int grid = (int)std::min<long long>((pieces + 127) / 128, 1184);
    k_prefetch_l2<<<std::max(grid, 1), 128, 0, st>>>(a, bytes);
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

// Band-scan triangle: three launches, each over all K right-hand sides (see band.cuh).
template <typename VT, int W>
int run_band(Plan &P, const ExecBlock &B, const VT *bb, VT *xx, int K, std::string &err) {
    DeviceState &D = *P.dev;
    cudaStream_t st = D.stream;
    const VT *coef = Pools<VT>::bcoef(D) + B.band_off;
    const VT *binv = Pools<VT>::binv(D) + B.band_off / W;
    VT *maps = reinterpret_cast<VT *>(D.band_maps);
    VT *states = reinterpret_cast<VT *>(D.band_states);
    constexpr int E = W * W + W;
    const size_t smem = (size_t)BAND_T * E * sizeof(VT);
    static std::atomic<unsigned long long> attr_set{0};
    if (!attr_done(attr_set)) {
        CK(cudaFuncSetAttribute(k_band_onepass<VT, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_mark(attr_set);
    }
    const int nch = B.band_nch, nblk = band_blocks(nch);
    // per column: the CTA totals (nblk maps) in the maps scratch, the ticket
    // and the CTAs' ready flags (nblk + 1 ints) in the states scratch
    int *flags = reinterpret_cast<int *>(states);
    CK(cudaMemsetAsync(flags, 0, sizeof(int) * (size_t)K * (nblk + 1), st));
    k_band_onepass<VT, W><<<dim3(nblk, K), BAND_T, smem, st>>>(coef, binv, bb, K, B.m, B.band_c, nch, maps, flags, xx,
                                                             D.status, P.opt.spin_limit);
    return RBS_OK;
}

// Grouped-layout moves of the processing positions [pa, pb) on stream st
// (the whole vector, or one triangle's rows inside the overlapped walk).
// smem: dynamic shared memory the launch reserves and does not use (0, or
// move_reserve's choice on the overlapped walk's side stream).
//
// The overlapped walk's side-stream moves reserve just more shared memory
// than an SM running one of the plan's staged triangles has left
// (move_reserve), so they cannot share an SM with a triangle's CTA and slow
// its level chain, as long as eight move CTAs of 256 threads still fit on an
// idle SM.  Fewer resident move threads measured slower than the sharing
// costs: 768 per SM took 2.5x as long per launch, 2048 in CTAs of 512 with
// a 42 KB reservation 1.4-1.9x, and the 128-column solve lost 14% with them.
constexpr int MOVE_SMEM_MAX = 64 << 10;

template <typename F>
void move_attr(F *kernel, std::atomic<unsigned long long> &done) {
    if (attr_done(done)) return;
    // a failure here surfaces as the launch error of the move itself
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MOVE_SMEM_MAX) == cudaSuccess)
        attr_mark(done);
}

template <typename VT, typename VT2, int K, int GL>
void launch_gather_grp(cudaStream_t st, int smem, const double *b, int ld, const double *const *cols, int k,
                       const int *perm, int n, int pa, int pb, VT *out, VT2 *out2, GroupCols grp) {
    static std::atomic<unsigned long long> done{0};
    if (smem) move_attr(k_gather_grp<VT, VT2, K, GL>, done);
    const unsigned gx = (unsigned)((pb - pa + 255) / 256);
    k_gather_grp<VT, VT2, K, GL><<<dim3(gx, GroupTile<K, GL>::CHUNKS), 256, smem, st>>>(b, ld, cols, k, perm, n, pa,
                                                                                       pb, out, out2, grp);
}

template <typename VT, typename VT2, int K>
void gather_grp(const DeviceState &D, cudaStream_t st, int n, const double *b, int ld, const double *const *cols,
                int k, VT *out, VT2 *out2, int GL, GroupCols grp, int pa, int pb, int smem = 0) {
    if (pb <= pa) return;
    if (GL == 1)
        launch_gather_grp<VT, VT2, K, 1>(st, smem, b, ld, cols, k, D.perm, n, pa, pb, out, out2, grp);
    else if constexpr (K % 2 == 0)
        launch_gather_grp<VT, VT2, K, 2>(st, smem, b, ld, cols, k, D.perm, n, pa, pb, out, out2, grp);
}

template <typename VT, int K, bool RESET>
void scatter_grp(const DeviceState &D, cudaStream_t st, int n, VT *xw, int k, double *x, int ld,
                 double *const *cols, int GL, GroupCols grp, int pa, int pb) {
    if (pb <= pa) return;
    const unsigned gx = (unsigned)((pb - pa + 255) / 256);
    if (GL == 1) {
        k_scatter_grp<VT, K, 1, RESET><<<dim3(gx, GroupTile<K, 1>::CHUNKS), 256, 0, st>>>(xw, D.perm, n, k, pa, pb, x,
                                                                                          ld, cols, grp);
    } else if constexpr (K % 2 == 0) {
        k_scatter_grp<VT, K, 2, RESET><<<dim3(gx, GroupTile<K, 2>::CHUNKS), 256, 0, st>>>(xw, D.perm, n, k, pa, pb, x,
                                                                                          ld, cols, grp);
    }
}

template <typename VT, int K, int GL>
void launch_scatter_rows(const DeviceState &D, cudaStream_t st, int n, const VT *xw, double *const *cols, int qa,
                         int qb, int smem) {
    using T = GroupTile<K, GL>;
    constexpr int TR = 256 / T::GT;
    static std::atomic<unsigned long long> done{0};
    if (smem) move_attr(k_scatter_rows<VT, K, GL>, done);
    const unsigned gx = (unsigned)((qb - qa + TR - 1) / TR);
    k_scatter_rows<VT, K, GL><<<dim3(gx, T::CHUNKS), 256, smem, st>>>(xw, D.io_rows, D.ipos, n, qa, qb, cols);
}

template <typename VT, int K>
void scatter_rows(const DeviceState &D, cudaStream_t st, int n, const VT *xw, double *const *cols, int GL, int qa,
                  int qb, int smem = 0) {
    if (qb <= qa) return;
    if (GL == 1) launch_scatter_rows<VT, K, 1>(D, st, n, xw, cols, qa, qb, smem);
    else if constexpr (K % 2 == 0) launch_scatter_rows<VT, K, 2>(D, st, n, xw, cols, qa, qb, smem);
}

// The overlapped walk (several columns, grouped layout): the triangles, in
// walk order, partition the rows; the right-hand sides of triangle j are
// moved in before the first block that touches its rows (need: the last
// triangle whose rows a block reads or updates in the b work vector) and its
// solutions moved out after the last block that reads them (last_use).
struct IoSchedule {
    std::vector<int> r0, r1;      // triangle j: processing rows [r0[j], r1[j])
    std::vector<int> need;        // per block
    std::vector<int> last_use;    // per triangle: block index
    bool ok = false;
};

IoSchedule io_schedule(const Plan &P) {
    IoSchedule S;
    const int nb = (int)P.blocks.size();
    for (const ExecBlock &B : P.blocks)
        if (B.tri) {
            if (B.r0 != (S.r1.empty() ? 0 : S.r1.back())) return S;  // not a partition in walk order
            S.r0.push_back(B.r0);
            S.r1.push_back(B.r0 + B.m);
        }
    if (S.r1.empty() || S.r1.back() != P.n) return S;
    auto tri_of = [&](int row) {
        return (int)(std::upper_bound(S.r0.begin(), S.r0.end(), row) - S.r0.begin()) - 1;
    };
    S.need.assign(nb, 0);
    S.last_use.assign(S.r0.size(), 0);
    for (int bi = 0, j = 0; bi < nb; ++bi) {
        const ExecBlock &B = P.blocks[bi];
        S.need[bi] = B.m > 0 ? tri_of(B.r0 + B.m - 1) : 0;
        if (B.tri) {
            S.last_use[j] = std::max(S.last_use[j], bi);
            ++j;
        } else if (B.ncols > 0) {
            for (int t = tri_of(B.c0); t <= tri_of(B.c0 + B.ncols - 1); ++t) S.last_use[t] = std::max(S.last_use[t], bi);
        }
    }
    S.ok = true;
    return S;
}

// The sorted row lists of the overlapped walk's scatter (k_scatter_rows),
// built on the host once per plan, outside any stream capture.  A plan whose
// triangles do not partition the rows in walk order gets none, and its walk
// moves the whole vectors before and after the blocks.
int ensure_io_rows(Plan &P, std::string &err) {
    DeviceState &D = *P.dev;
    if (D.io_rows || (long long)P.perm.size() != (long long)P.n) return RBS_OK;
    const IoSchedule S = io_schedule(P);
    if (!S.ok) return RBS_OK;
    std::vector<int> rows(P.perm.begin(), P.perm.end());
    for (size_t j = 0; j < S.r0.size(); ++j) std::sort(rows.begin() + S.r0[j], rows.begin() + S.r1[j]);
    return upload(D, D.io_rows, rows, err);
}

// Dynamic shared memory of the side-stream moves next to staged triangles
// of at least ca_min bytes: one byte more than such an SM has left, rounded
// up to 1 KB, when eight move CTAs still fit on an idle SM; 0 otherwise (or
// when no triangle is staged).  RBS_MOVE_SMEM (bytes, at most 64 KB)
// overrides the choice.
int move_reserve(const DeviceState &D, size_t ca_min) {
    static const long long forced = [] {
        const char *e = std::getenv("RBS_MOVE_SMEM");
        return e ? std::atoll(e) : -1LL;
    }();
    if (forced >= 0) return (int)std::min<long long>(forced, MOVE_SMEM_MAX);
    if (!ca_min) return 0;
    const long long left = (long long)D.smem_sm - (long long)ca_min - D.smem_reserved;  // beside one triangle
    long long need = left - D.smem_reserved + 1;  // a move CTA needs its own reservation too
    if (need <= 0) return 0;
    need = (need + 1023) / 1024 * 1024;
    if (8 * (need + D.smem_reserved) > D.smem_sm) return 0;
    return (int)need;
}

// One pass over all blocks: triangles solve into xw, squares update bw.
template <typename VT, int K>
int launch_blocks(Plan &P, std::string &err, bool io = false) {
    DeviceState &D = *P.dev;
    cudaStream_t st = D.stream;
    const VT *val = Pools<VT>::val(D);
    const VT *inv = Pools<VT>::inv(D);
    VT *bw = Pools<VT>::bw(D);
    VT *xw = Pools<VT>::xw(D);
    LevelDesc *descs = nullptr;
    int rc = level_descs<VT, K>(P, descs, err);
    if (rc) return rc;
    CsfDesc *edescs = nullptr;
    CaDesc *cdescs = nullptr;
    const int GL = plan_group<VT>(P, K);
    if ((rc = ca_descs<VT>(P, cdescs, K, GL, err))) return rc;
    if (K == 1 && (rc = ell_descs<VT>(P, edescs, err))) return rc;
    if (D.ntri) CK(cudaMemsetAsync(D.tickets, 0, sizeof(int) * D.ntri, st));
    if (K == 1 && D.lc_queue) {
        CK(cudaMemsetAsync(D.lc_queue, 0, sizeof(int) * D.ntri, st));
        if ((rc = lc_attr<VT>(err))) return rc;
    }
    const long long limit = P.opt.spin_limit;
    // The staged level kernel runs on one SM; the others pull the data of
    // the staged triangles into L2 meanwhile (up to 96 MB, in block order).
    bool forked = false;
    if (K == 1 && D.side) {
        long long budget = 96ll << 20;
        for (const ExecBlock &B : P.blocks) {
            if (!B.tri || B.kernel != RBS_K_LEVEL || B.lvl_var == LVL_PLAIN || budget <= 0) continue;
            if (!forked) {
                CK(cudaEventRecord(D.ev_fork, st));
                CK(cudaStreamWaitEvent(D.side, D.ev_fork, 0));
                forked = true;
            }
            if (B.lvl_var == LVL_LC && B.lc_ok) {
                const int *sg = P.lc_segs.data() + 3 * B.lc_seg_off;
                const int c0 = sg[0], c1 = P.lc_segs[(size_t)(3 * (B.lc_seg_off + B.lc_nseg - 1))] +
                                           P.lc_segs[(size_t)(3 * (B.lc_seg_off + B.lc_nseg - 1) + 1)];
                if (c1 > c0) {
                    const bool f64 = sizeof(VT) == 8;
                    const int *t0 = P.lc_tab.data() + LC_TAB_INTS * (size_t)c0,
                              *t1 = P.lc_tab.data() + LC_TAB_INTS * (size_t)(c1 - 1);
                    const long long a = 16LL * (f64 ? t0[0] : t0[2]), e = 16LL * ((f64 ? t1[0] : t1[2]) + (f64 ? t1[1] : t1[3]));
                    prefetch_range(D.side, Pools<VT>::lcrec(D) + a, e - a);
                    budget -= e - a;
                }
                continue;
            }
            if (B.ca_ok && B.lvl_var == LVL_CA) {
                const long long ne = B.ca_hi - B.ca_lo;
                prefetch_range(D.side, Pools<VT>::cav(D) + B.ca_lo, ne * (long long)sizeof(VT));
                if (B.ca_win && B.ca_w >= 2) prefetch_range(D.side, D.ca_col16 + B.ca_lo, ne * 2);
                else prefetch_range(D.side, D.ca_col + B.ca_lo, ne * 4);
                prefetch_range(D.side, inv + B.r0, (long long)B.m * sizeof(VT));
                budget -= ne * ((long long)sizeof(VT) + 4) + (long long)B.m * sizeof(VT);
                continue;
            }
            if (B.ell_ok && B.lvl_var == LVL_CSF) {
                const long long ne = B.ell_hi - B.ell_lo;
                prefetch_range(D.side, Pools<VT>::ellv(D) + B.ell_lo, ne * (long long)sizeof(VT));
                prefetch_range(D.side, D.ell_col + B.ell_lo, ne * 4);
                prefetch_range(D.side, inv + B.r0, (long long)B.m * sizeof(VT));
                budget -= ne * ((long long)sizeof(VT) + 4) + (long long)B.m * sizeof(VT);
                continue;
            }
        }
    }
    // Overlapped walk (io: several columns in the grouped layout, the caller's
    // columns in D.iotab): the first triangle's right-hand sides are moved in
    // on the walk's stream, the other triangles' on the side stream, in walk
    // order, each followed by an event the first block that needs it waits
    // for; solutions go out on the side stream as blocks free them.  The moves
    // run on the SMs the walk leaves idle.
    io = io && K > 1 && GL > 0;
    IoSchedule S;
    std::vector<std::vector<int>> freed;  // per block: triangles whose solutions it is the last to read
    int waited = 0, T = 0, move_smem = 0;
    if (io) {
        S = io_schedule(P);
        if (!D.io_rows) S.ok = false;
        T = (int)S.r0.size();
        if (!S.ok) {
            gather_grp<VT, VT, K>(D, st, P.n, nullptr, P.n, D.iotab, K, bw, (VT *)nullptr, GL, GroupCols{}, 0, P.n);
        } else {
            while ((int)D.ov_ev.size() < 2 * T) {
                cudaEvent_t e = nullptr;
                CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                D.ov_ev.push_back(e);
            }
            size_t ca_min = 0;
            for (const ExecBlock &B : P.blocks)
                if (B.tri && B.kernel == RBS_K_LEVEL && B.ca_ok) {
                    const size_t v = ca_smem_bytes<VT>(B.ca_w, B.ca_win != 0, K, GL);
                    ca_min = ca_min ? std::min(ca_min, v) : v;
                }
            move_smem = move_reserve(D, ca_min);
            CK(cudaEventRecord(D.ev_fork, st));
            CK(cudaStreamWaitEvent(D.side, D.ev_fork, 0));
            gather_grp<VT, VT, K>(D, st, P.n, nullptr, P.n, D.iotab, K, bw, (VT *)nullptr, GL, GroupCols{}, S.r0[0],
                                  S.r1[0]);
            for (int j = 1; j < T; ++j) {
                gather_grp<VT, VT, K>(D, D.side, P.n, nullptr, P.n, D.iotab, K, bw, (VT *)nullptr, GL, GroupCols{},
                                      S.r0[j], S.r1[j], move_smem);
                CK(cudaEventRecord(D.ov_ev[j], D.side));
            }
            freed.assign(P.blocks.size(), {});
            for (int j = 0; j < T; ++j) freed[S.last_use[j]].push_back(j);
        }
    }
    int ti = 0, li = 0, eti = 0, cti = 0;
    for (const ExecBlock &B : P.blocks) {
        const int bi = (int)(&B - P.blocks.data());
        if (io && S.ok && S.need[bi] > waited) {
            CK(cudaStreamWaitEvent(st, D.ov_ev[S.need[bi]], 0));
            waited = S.need[bi];
        }
        if (D.profile) CK(cudaEventRecord(D.bev[2 * B.index], st));
        if (B.tri) {
            const VT *bb = bw + (long long)B.r0 * K;
            VT *xx = xw + (long long)B.r0 * K;
            // Several right-hand sides: a level triangle with a staged
            // level-ELL layout runs one CTA per group of columns; the other
            // single-CTA level kernels have no multi-column form, and one
            // dependency walk of the multi-CTA sync-free kernel serves all K
            // columns, so their triangles take it.
            const bool mc_ca = K > 1 && B.kernel == RBS_K_LEVEL && B.ca_ok;
            const int kernel = (K > 1 && B.kernel == RBS_K_LEVEL && !mc_ca) ? RBS_K_SYNCFREE : B.kernel;
            switch (kernel) {
            case RBS_K_DIAG:
                if (GL) {
                    const int grid = grid_for((long long)B.m * K, 256, D.num_sms);
                    const long long gs = (long long)P.n * GL;
                    if (GL == 1)
                        k_tri_diag_grp<VT, 1><<<grid, 256, 0, st>>>(inv + B.r0, bw + B.r0, xw + B.r0, B.m, K, gs);
                    else
                        k_tri_diag_grp<VT, 2><<<grid, 256, 0, st>>>(inv + B.r0, bw + 2LL * B.r0, xw + 2LL * B.r0, B.m,
                                                                    K / 2, gs);
                    break;
                }
                k_tri_diag<VT, K><<<grid_for((long long)B.m * K, 256, D.num_sms), 256, 0, st>>>(inv + B.r0, bb, xx,
                                                                                               B.m);
                break;
            case RBS_K_LEVEL:
                if (K == 1 && B.lvl_var == LVL_LC && B.lc_ok) {
                    const int grid = std::min(B.lc_nseg, D.num_sms);
                    k_tri_lc<VT><<<grid, LC_T, lc_smem<VT>(), st>>>(D.lc_segs + B.lc_seg_off, B.lc_nseg,
                                                                   Pools<VT>::lcrec(D), sizeof(VT) == 4 ? 1 : 0, bb,
                                                                   xx, D.lc_queue + ti, D.status, limit);
                } else if ((K == 1 && B.lvl_var == LVL_CA && B.ca_ok) || mc_ca) {
                    launch_ca_any<VT>(B, cdescs + cti, K, GL ? GL : ca_group<VT>(B, K), st);
                } else if (K == 1 && B.lvl_var == LVL_CSF && B.ell_ok) {
                    k_tri_cta_syncfree<VT><<<1, 1024, CsfLayout<VT>::total, st>>>(edescs + eti, D.status, limit);
                } else {
                    k_tri_level<VT, K><<<1, 1024, 0, st>>>(descs + li);
                }
                break;
            case RBS_K_SEQ:
                k_tri_seq<VT, K><<<1, 32, 0, st>>>(D.rp + B.rp_off, D.col, val, inv + B.r0, bb, xx, B.m);
                break;
            case RBS_K_BANDSCAN: {
                int rc2 = RBS_OK;
                switch (B.band_w) {
                case 1: rc2 = run_band<VT, 1>(P, B, bb, xx, K, err); break;
                case 2: rc2 = run_band<VT, 2>(P, B, bb, xx, K, err); break;
                case 4: rc2 = run_band<VT, 4>(P, B, bb, xx, K, err); break;
                default: rc2 = run_band<VT, 8>(P, B, bb, xx, K, err); break;
                }
                if (rc2) return rc2;
                break;
            }
            default: {
                const int gs = B.sf_group >= 1 && B.sf_group <= 32 ? B.sf_group : std::max(1, B.group);
                const int g = K == 1 ? gs : (K < 32 ? K : 32);
                const long long warps = ((long long)B.m * g + 31) / 32;
                int grid = (int)std::min<long long>(syncfree_grid<VT, K>(D), (warps + 7) / 8);
                k_tri_syncfree<VT, K><<<std::max(grid, 1), 256, 0, st>>>(D.rp + B.rp_off, D.col, val, inv + B.r0, bb,
                                                                        xx, B.m, gs, D.tickets + ti, D.status, limit);
                break;
            }
            }
            if (B.kernel == RBS_K_LEVEL) {  // descriptor tables list every level triangle
                ++li;
                if (B.ell_ok) ++eti;
                if (B.ca_ok) ++cti;
            }
            ++ti;
        } else if (B.kernel == RBS_K_SPMV && GL) {
            const int *rows = B.rows_off >= 0 ? D.rows + B.rows_off : nullptr;
            const int grid = grid_for((long long)B.nrows * (K / GL), 256, D.num_sms);
            const long long gs = (long long)P.n * GL;
            if (GL == 1)
                k_spmv_sub_grp<VT, 1><<<grid, 256, 0, st>>>(D.rp + B.rp_off, D.col, val, rows, B.nrows, K, gs,
                                                            xw + B.c0, bw + B.r0);
            else
                k_spmv_sub_grp<VT, 2><<<grid, 256, 0, st>>>(D.rp + B.rp_off, D.col, val, rows, B.nrows, K / 2, gs,
                                                            xw + 2LL * B.c0, bw + 2LL * B.r0);
        } else if (B.kernel == RBS_K_SPMV) {
            const int g = K == 1 ? B.group : (K < 32 ? K : 32);
            const int *rows = B.rows_off >= 0 ? D.rows + B.rows_off : nullptr;
            const bool med = K == 1 && B.medrows > 0;
            const int maxlen = med ? RBS_MEDROW : B.longrows > 0 ? RBS_LONGROW : 0x7fffffff;
            // the medium rows' warps lead the launch (their CTAs first), the
            // other rows' groups follow in the same grid
            const int medctas = med ? grid_for((long long)B.medrows * 32, 256, D.num_sms) : 0;
            // single column, a grid at its cap (every warp loops): a lane
            // group takes two rows per iteration
            const long long lanes = (long long)B.nrows * g;
            const int pairs = K == 1 && lanes > (long long)grid_for(lanes, 256, D.num_sms) * 256;
            k_spmv_sub<VT, K><<<medctas + grid_for(pairs ? (lanes + 1) / 2 : lanes, 256, D.num_sms), 256, 0, st>>>(
                D.rp + B.rp_off, D.col, val, rows, B.nrows, B.group, xw + (long long)B.c0 * K,
                bw + (long long)B.r0 * K, maxlen, med ? D.rows + B.med_off : nullptr, med ? B.medrows : 0,
                medctas, pairs);
            if (B.longrows > 0)
                k_spmv_long<VT, K><<<D.num_sms * 2, 256, 0, st>>>(D.rp + B.rp_off, D.col, val, rows,
                                                                  D.rows + B.long_off, B.longrows,
                                                                  xw + (long long)B.c0 * K, bw + (long long)B.r0 * K);
        }
        if (D.profile) CK(cudaEventRecord(D.bev[2 * B.index + 1], st));
        if (!freed.empty())
            for (int j : freed[bi]) CK(cudaEventRecord(D.ov_ev[T + j], st));
    }
    if (io) {
        double *const *xcols = D.iotab + RBS_IO_COLS;
        if (S.ok) {
            for (const auto &fj : freed)
                for (int j : fj) {
                    CK(cudaStreamWaitEvent(D.side, D.ov_ev[T + j], 0));
                    scatter_rows<VT, K>(D, D.side, P.n, xw, xcols, GL, S.r0[j], S.r1[j], move_smem);
                }
            CK(cudaEventRecord(D.ev_join, D.side));
            CK(cudaStreamWaitEvent(st, D.ev_join, 0));
        } else {
            scatter_grp<VT, K, true>(D, st, P.n, xw, K, nullptr, P.n, xcols, GL, GroupCols{}, 0, P.n);
        }
    }
    if (forked) {
        CK(cudaEventRecord(D.ev_join, D.side));
        CK(cudaStreamWaitEvent(st, D.ev_join, 0));
    }
    CK(cudaGetLastError());
    return RBS_OK;
}

// The block walk of a (precision, K) pair is captured into a CUDA graph on
// its second use (the first runs eagerly and performs the one-time set-up
// that capture does not allow) and replayed afterwards: one launch per
// solve pass instead of one per block.
// Whether the block walk for K columns runs a kernel that polls the x work
// vector for its sentinel (the sync-free kernels), with the kernel choice
// of launch_blocks.
bool walk_polls(const Plan &P, int K) {
    for (const ExecBlock &B : P.blocks) {
        if (!B.tri) continue;
        if (B.kernel == RBS_K_SYNCFREE) return true;
        if (B.kernel != RBS_K_LEVEL) continue;
        if (K > 1 && !B.ca_ok) return true;  // multi-column level triangles without the staged layout
        if (K == 1 && B.lvl_var == LVL_CSF && B.ell_ok) return true;
    }
    return false;
}

template <typename VT, int K>
int run_blocks(Plan &P, std::string &err, bool io = false) {
    DeviceState &D = *P.dev;
    if (!io && Pools<VT>::dirty(D) && walk_polls(P, K)) {  // the sync-free kernels poll x for the sentinel
        const long long cnt = (long long)P.n * D.kcap;
        k_fill<VT><<<grid_for(cnt, 256, D.num_sms), 256, 0, D.stream>>>(Pools<VT>::xw(D), cnt, Pools<VT>::sent());
        Pools<VT>::dirty(D) = false;
    }
    // per-block timing needs real event timestamps, which captured event
    // records are not: profiled solves launch eagerly
    if (!D.use_graphs || D.profile) return launch_blocks<VT, K>(P, err, io);
    const long long key = (long long)K * 8 + (sizeof(VT) == 8 ? 0 : 2) + (io ? 4 : 0);
    auto it = D.graphs.find(key);
    if (it != D.graphs.end()) {
        CK(cudaGraphLaunch(it->second, D.stream));
        return RBS_OK;
    }
    if (!D.graph_seen.count(key)) {
        D.graph_seen.insert(key);
        return launch_blocks<VT, K>(P, err, io);
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(D.stream, cudaStreamCaptureModeThreadLocal));
    int rc = launch_blocks<VT, K>(P, err, io);
    cudaError_t e = cudaStreamEndCapture(D.stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) {
        err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
        return RBS_ERR_CUDA;
    }
    cudaGraphExec_t ex = nullptr;
    // captured kernels keep the priority of the stream they were captured on
    e = cudaGraphInstantiate(&ex, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
        return RBS_ERR_CUDA;
    }
    D.graphs[key] = ex;
    CK(cudaGraphLaunch(ex, D.stream));
    return RBS_OK;
}

void drop_graphs(DeviceState &D) {
    for (auto &kv : D.graphs) cudaGraphExecDestroy(kv.second);
    D.graphs.clear();
    D.graph_seen.clear();
}
void drop_graphs_fwd(DeviceState &D) { drop_graphs(D); }

// Right-hand sides into processing order: the caller's columns (b + c*ld,
// or the device table cols) into the work vector out (and out2 in a second
// precision, when given): grouped (GL > 0) by one thread per processing
// position and chunk of column groups, row-interleaved with many columns by
// the transposing tile kernel, whose reads and writes are both coalesced.
template <typename VT, typename VT2, int K>
void gather_in(DeviceState &D, int n, const double *b, int ld, const double *const *cols, int k, VT *out,
               VT2 *out2, int GL, GroupCols grp = GroupCols{}) {
    const int tgrid = std::max(1, (int)std::min<long long>(((long long)n + TP_ROWS - 1) / TP_ROWS, (long long)D.num_sms * 8));
    if (GL) {
        gather_grp<VT, VT2, K>(D, D.stream, n, b, ld, cols, k, out, out2, GL, grp, 0, n);
    } else if (K >= 8 || grp.tab) {
        k_gather_t<VT, VT2, K><<<tgrid, 256, 0, D.stream>>>(b, ld, cols, k, D.ipos, n, out, out2, grp);
    } else {
        const int grid = grid_for((long long)n * K, 256, D.num_sms);
        if (cols) k_gather_cols<VT, K><<<grid, 256, 0, D.stream>>>(cols, k, D.perm, n, out);
        else k_gather<VT, K><<<grid, 256, 0, D.stream>>>(b, ld, k, D.perm, n, out);
        if (out2) {
            if (cols) k_gather_cols<VT2, K><<<grid, 256, 0, D.stream>>>(cols, k, D.perm, n, out2);
            else k_gather<VT2, K><<<grid, 256, 0, D.stream>>>(b, ld, k, D.perm, n, out2);
        }
    }
}

// Solutions out of processing order into the caller's columns (x + c*ld or
// the table cols); RESET puts the sentinel back into the work vector.
template <typename VT, int K, bool RESET>
void scatter_out(DeviceState &D, int n, VT *xw, int k, double *x, int ld, double *const *cols, int GL,
                 GroupCols grp = GroupCols{}) {
    const int tgrid = std::max(1, (int)std::min<long long>(((long long)n + TP_ROWS - 1) / TP_ROWS, (long long)D.num_sms * 8));
    if (GL) {
        scatter_grp<VT, K, RESET>(D, D.stream, n, xw, k, x, ld, cols, GL, grp, 0, n);
    } else if (K >= 8 || grp.tab) {
        k_scatter_t<VT, K, RESET><<<tgrid, 256, 0, D.stream>>>(xw, D.ipos, n, k, x, ld, cols, grp);
    } else {
        const int grid = grid_for((long long)n * K, 256, D.num_sms);
        if constexpr (RESET) {
            if (cols) k_scatter_cols<VT, K><<<grid, 256, 0, D.stream>>>(xw, D.perm, n, k, cols);
            else k_scatter_reset<VT, K><<<grid, 256, 0, D.stream>>>(xw, D.perm, n, k, x, ld);
        } else {
            static_assert(RESET || std::is_same<VT, double>::value, "FP64 accumulator only");
            if (cols) k_scatter64_cols<K><<<grid, 256, 0, D.stream>>>(xw, D.perm, n, k, cols);
            else k_scatter64<K><<<grid, 256, 0, D.stream>>>(xw, D.perm, n, k, x, ld);
        }
    }
}

// Several columns in the grouped layout: the walk moves the columns itself,
// overlapped with the blocks (launch_blocks), reading them through the device
// table D.iotab set just before it on the same stream.
template <int K>
int solve_fp64(Plan &P, const double *b, double *x, int k, int ld, std::string &err) {
    DeviceState &D = *P.dev;
    const int GL = plan_group<double>(P, K);
    if (K > 1 && GL) {
        int rc = ensure_io_rows(P, err);
        if (rc) return rc;
        k_set_io<<<1, RBS_IO_COLS, 0, D.stream>>>(D.iotab, b, x, ld, k);
        if ((rc = run_blocks<double, K>(P, err, true))) return rc;
        D.xw_dirty64 = true;
        CK(cudaGetLastError());
        return RBS_OK;
    }
    gather_in<double, double, K>(D, P.n, b, ld, nullptr, k, D.bw64, nullptr, GL);
    int rc = run_blocks<double, K>(P, err);
    if (rc) return rc;
    scatter_out<double, K, true>(D, P.n, D.xw64, k, x, ld, nullptr, GL);
    CK(cudaGetLastError());
    return RBS_OK;
}

template <int K>
int solve_fp32(Plan &P, const double *b, double *x, int k, int ld, std::string &err) {
    DeviceState &D = *P.dev;
    const int GL = plan_group<float>(P, K);
    if (K > 1 && GL) {
        int rc = ensure_io_rows(P, err);
        if (rc) return rc;
        k_set_io<<<1, RBS_IO_COLS, 0, D.stream>>>(D.iotab, b, x, ld, k);
        if ((rc = run_blocks<float, K>(P, err, true))) return rc;
        D.xw_dirty32 = true;
        CK(cudaGetLastError());
        return RBS_OK;
    }
    gather_in<float, float, K>(D, P.n, b, ld, nullptr, k, D.bw32, nullptr, GL);
    int rc = run_blocks<float, K>(P, err);
    if (rc) return rc;
    scatter_out<float, K, true>(D, P.n, D.xw32, k, x, ld, nullptr, GL);
    CK(cudaGetLastError());
    return RBS_OK;
}

// FP32 sweeps with FP64 residuals and FP64 accumulation:
//   x0 = L32^-1 b;  repeat  r = b - L x (FP64),  d = L32^-1 r,  x += d
// until ||d||/||x|| <= ir_tol for every right-hand side.
//
// mixed_first: x0 = L32^-1 b (b already gathered into b64keep and bw32).
// x64 (+)= d32 with the per-column norms, in the layout of the FP32 sweeps
template <int K>
void mixed_update(Plan &P, int first) {
    DeviceState &D = *P.dev;
    const int GL = plan_group<float>(P, K);
    if (GL) {
        const dim3 grid((unsigned)std::max(1, std::min((P.n + 255) / 256, 2 * D.num_sms)), K);
        if (GL == 1) k_update_grp<K, 1><<<grid, 256, 0, D.stream>>>(D.x64acc, D.xw32, P.n, first, D.norms);
        else k_update_grp<K, 2><<<grid, 256, 0, D.stream>>>(D.x64acc, D.xw32, P.n, first, D.norms);
        return;
    }
    k_update<K><<<grid_for((long long)P.n * K, 256, D.num_sms), 256, 0, D.stream>>>(D.x64acc, D.xw32, P.n, first,
                                                                                      D.norms);
}

template <int K>
int mixed_first(Plan &P, std::string &err) {
    DeviceState &D = *P.dev;
    int rc = run_blocks<float, K>(P, err);
    if (rc) return rc;
    CK(cudaMemsetAsync(D.norms, 0, sizeof(double) * 2 * K, D.stream));
    mixed_update<K>(P, 1);
    return RBS_OK;
}

// mixed_step: one correction r = b - L x, d = L32^-1 r, x += d, with the
// per-column sums of squares of d and x copied to the host (h_norms).
template <int K>
int mixed_step(Plan &P, std::string &err) {
    DeviceState &D = *P.dev;
    const int n = P.n;
    const int G = P.nnz / std::max(1, n) < 6 ? 4 : 8;
    const int GL = plan_group<float>(P, K);
    if (GL == 1)
        k_residual_grp<1><<<grid_for((long long)n * K, 256, D.num_sms), 256, 0, D.stream>>>(
            D.full_rp, D.full_col, D.full_val, D.x64acc, D.b64keep, D.bw32, n, K, (long long)n);
    else if (GL == 2)
        k_residual_grp<2><<<grid_for((long long)n * (K / 2), 256, D.num_sms), 256, 0, D.stream>>>(
            D.full_rp, D.full_col, D.full_val, D.x64acc, D.b64keep, D.bw32, n, K / 2, 2LL * n);
    else
        k_residual<K><<<grid_for((long long)n * (K == 1 ? G : std::min(K, 32)), 256, D.num_sms), 256, 0, D.stream>>>(
            D.full_rp, D.full_col, D.full_val, D.x64acc, D.b64keep, D.bw32, n, G);
    int rc = run_blocks<float, K>(P, err);
    if (rc) return rc;
    CK(cudaMemsetAsync(D.norms, 0, sizeof(double) * 2 * K, D.stream));
    mixed_update<K>(P, 0);
    CK(cudaMemcpyAsync(D.h_norms, D.norms, sizeof(double) * 2 * K, cudaMemcpyDeviceToHost, D.stream));
    return RBS_OK;
}

// Largest ||d||/||x|| over the first k columns of the last step's norms
// (NaN propagates).
double mixed_correction(const DeviceState &D, int K, int k) {
    double corr = 0;
    for (int c = 0; c < k; ++c) {
        const double dn = std::sqrt(D.h_norms[c]), xn = std::sqrt(D.h_norms[K + c]);
        const double r = xn > 0 ? dn / xn : dn;
        if (!(r <= corr)) corr = r;
    }
    return corr;
}

template <int K>
int solve_mixed(Plan &P, const double *b, double *x, int k, int ld, int &iters, double &corr, std::string &err) {
    DeviceState &D = *P.dev;
    const int GL = plan_group<float>(P, K);
    gather_in<double, float, K>(D, P.n, b, ld, nullptr, k, D.b64keep, D.bw32, GL);
    int rc = mixed_first<K>(P, err);
    if (rc) return rc;
    iters = 0;
    corr = 1.0;
    for (int it = 0; it < P.opt.ir_max_iter; ++it) {
        if ((rc = mixed_step<K>(P, err))) return rc;
        CK(cudaStreamSynchronize(D.stream));
        ++iters;
        corr = mixed_correction(D, K, k);
        if (corr <= P.opt.ir_tol) break;
    }
    scatter_out<double, K, false>(D, P.n, D.x64acc, k, x, ld, nullptr, GL);
    CK(cudaGetLastError());
    if (!(corr <= P.opt.ir_tol)) {
        err = "mixed-precision refinement stopped at ||dx||/||x|| = " + std::to_string(corr);
        return RBS_ERR_NOCONV;
    }
    return RBS_OK;
}

// ---------------------------------------------------------------------------
// Asynchronous batches for the request server: the right-hand sides and the
// solutions are given as device tables of column pointers (the columns of
// several requests side by side).  Nothing here waits for the device; the
// caller drains the plan's stream between the phases (an event), so one
// host thread can keep many plans' solves in flight.
// ---------------------------------------------------------------------------
#define RBS_FOR_K(K, EXPR)                                   \
    switch (K) {                                             \
    case 1: { constexpr int KC = 1; EXPR; } break;           \
    case 2: { constexpr int KC = 2; EXPR; } break;           \
    case 4: { constexpr int KC = 4; EXPR; } break;           \
    case 8: { constexpr int KC = 8; EXPR; } break;           \
    case 16: { constexpr int KC = 16; EXPR; } break;         \
    case 32: { constexpr int KC = 32; EXPR; } break;         \
    case 64: { constexpr int KC = 64; EXPR; } break;         \
    default: { constexpr int KC = 128; EXPR; } break;        \
    }

template <int K>
int batch_start_k(Plan &P, const double *const *bcols, double *const *xcols, int k, int prec, const GroupCols &gb,
                  const GroupCols &gx, std::string &err) {
    DeviceState &D = *P.dev;
    const int n = P.n;
    int rc;
    if (prec == RBS_PREC_FP64) {
        const int GL = plan_group<double>(P, K);
        gather_in<double, double, K>(D, n, nullptr, n, bcols, k, D.bw64, nullptr, GL, gb);
        if ((rc = run_blocks<double, K>(P, err))) return rc;
        scatter_out<double, K, true>(D, n, D.xw64, k, nullptr, n, xcols, GL, gx);
    } else if (prec == RBS_PREC_FP32) {
        const int GL = plan_group<float>(P, K);
        gather_in<float, float, K>(D, n, nullptr, n, bcols, k, D.bw32, nullptr, GL, gb);
        if ((rc = run_blocks<float, K>(P, err))) return rc;
        scatter_out<float, K, true>(D, n, D.xw32, k, nullptr, n, xcols, GL, gx);
    } else {
        gather_in<double, float, K>(D, n, nullptr, n, bcols, k, D.b64keep, D.bw32, plan_group<float>(P, K), gb);
        if ((rc = mixed_first<K>(P, err))) return rc;
        if ((rc = mixed_step<K>(P, err))) return rc;
    }
    CK(cudaGetLastError());
    return RBS_OK;
}

template <int K>
int batch_end_k(Plan &P, double *const *xcols, int k, const GroupCols &gx, std::string &err) {
    DeviceState &D = *P.dev;
    scatter_out<double, K, false>(D, P.n, D.x64acc, k, nullptr, P.n, xcols, plan_group<float>(P, K), gx);
    CK(cudaGetLastError());
    return RBS_OK;
}

}  // namespace

int device_reserve(Plan &P, int k, std::string &err) {
    if (!P.dev) {
        err = "plan has no device state";
        return RBS_ERR_ARG;
    }
    if (k < 1 || k > 128) {
        err = "reserve: k must be in [1, 128]";
        return RBS_ERR_ARG;
    }
    int rc = ensure_work(P, pow2_at_least(k), err);
    if (rc) return rc;
    CK(cudaStreamSynchronize(P.dev->stream));
    return RBS_OK;
}

int device_batch_start(Plan &P, const double *const *bcols, double *const *xcols, int k, int prec, int *more,
                       std::string &err, const BatchGroup *grp) {
    DeviceState &D = *P.dev;
    if (k < 1 || k > 128 || (prec != RBS_PREC_FP64 && !D.mixed)) {
        err = "batch: k must be in [1, 128]; FP32 and mixed batches need a plan with FP32 copies";
        return RBS_ERR_ARG;
    }
    const int K = pow2_at_least(k);
    int rc = ensure_work(P, K, err);
    if (rc) return rc;
    D.bat_K = K;
    D.bat_k = k;
    D.bat_prec = prec;
    D.bat_iters = 0;
    D.bat_corr = 0;
    D.bat_xcols = xcols;
    GroupCols gb{}, gx{};
    if (grp) {
        gb = GroupCols{grp->btab, grp->seg, grp->off, grp->count};
        gx = GroupCols{grp->xtab, grp->seg, grp->off, grp->count};
    }
    D.bat_gx = gx;
    RBS_FOR_K(K, rc = batch_start_k<KC>(P, bcols, xcols, k, prec, gb, gx, err));
    if (rc) return rc;
    *more = prec == RBS_PREC_MIXED ? 1 : 0;
    if (!*more) CK(cudaMemcpyAsync(D.h_status, D.status, sizeof(int), cudaMemcpyDeviceToHost, D.stream));
    return RBS_OK;
}

int device_batch_next(Plan &P, int *more, std::string &err) {
    DeviceState &D = *P.dev;
    const int K = D.bat_K;
    ++D.bat_iters;
    D.bat_corr = mixed_correction(D, K, D.bat_k);
    int rc = RBS_OK;
    if (D.bat_corr <= P.opt.ir_tol || D.bat_iters >= P.opt.ir_max_iter) {
        RBS_FOR_K(K, rc = batch_end_k<KC>(P, D.bat_xcols, D.bat_k, D.bat_gx, err));
        if (rc) return rc;
        CK(cudaMemcpyAsync(D.h_status, D.status, sizeof(int), cudaMemcpyDeviceToHost, D.stream));
        *more = 0;
        return RBS_OK;
    }
    RBS_FOR_K(K, rc = mixed_step<KC>(P, err));
    if (rc) return rc;
    *more = 1;
    return RBS_OK;
}

int device_batch_finish(Plan &P, int *iters, double *corr, std::string &err) {
    DeviceState &D = *P.dev;
    if (iters) *iters = D.bat_iters;
    if (corr) *corr = D.bat_corr;
    if (*D.h_status & RBS_STATUS_TIMEOUT) return device_sync(P, err);  // resets the status and the work vectors
    if (D.bat_prec == RBS_PREC_MIXED && !(D.bat_corr <= P.opt.ir_tol)) {
        err = "mixed-precision refinement stopped at ||dx||/||x|| = " + std::to_string(D.bat_corr);
        return RBS_ERR_NOCONV;
    }
    return RBS_OK;
}

namespace {

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
    CK(cudaDeviceGetAttribute(&D.smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, D.device));
    CK(cudaDeviceGetAttribute(&D.smem_reserved, cudaDevAttrReservedSharedMemoryPerBlock, D.device));
    // The walk's stream at the greatest priority, its side stream (prefetch,
    // the overlapped walk's moves) at the lowest: when both have CTAs
    // waiting, an SM that frees up takes the walk's.
    int prio_low = 0, prio_high = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    CK(cudaStreamCreateWithPriority(&D.stream, cudaStreamNonBlocking, prio_high));
    D.own_stream = true;
    CK(cudaEventCreate(&D.ev0));
    CK(cudaEventCreate(&D.ev1));
    {
        const char *ng = std::getenv("RBS_NO_GRAPHS");
        D.use_graphs = !(ng && ng[0] == '1');
    }
    int rc;
    if ((rc = upload(D, D.rp, P.rp_pool, err))) return rc;
    if ((rc = upload(D, D.col, P.col_pool, err))) return rc;
    if ((rc = upload(D, D.val, P.val_pool, err))) return rc;
    if ((rc = upload(D, D.lvl, P.lvl_pool, err))) return rc;
    if ((rc = upload(D, D.map, P.map_pool, err))) return rc;
    if ((rc = upload(D, D.rows, P.rows_pool, err))) return rc;
    if ((rc = upload(D, D.perm, P.perm, err))) return rc;
    {
        std::vector<int> ipos(P.perm.size());
        for (size_t p = 0; p < P.perm.size(); ++p) ipos[(size_t)P.perm[p]] = (int)p;
        if ((rc = upload(D, D.ipos, ipos, err))) return rc;
    }
    if ((rc = upload(D, D.inv, P.inv_diag, err))) return rc;
    D.mixed = P.opt.mixed != 0;
    if (D.mixed) {
        const auto v32 = to_f32(P.val_pool), i32 = to_f32(P.inv_diag);
        if ((rc = upload(D, D.val32, v32, err))) return rc;
        if ((rc = upload(D, D.inv32, i32, err))) return rc;
        if ((rc = upload(D, D.full_rp, P.full_rp, err))) return rc;
        if ((rc = upload(D, D.full_col, P.full_col, err))) return rc;
        if ((rc = upload(D, D.full_val, P.full_val, err))) return rc;
    }
    if ((rc = upload(D, D.band_coef, P.band_coef, err))) return rc;
    if ((rc = upload(D, D.band_inv, P.band_inv, err))) return rc;
    {
        // every triangle with a band layout may run the band scan (the tuner
        // switches kernels after this point), so size for all of them
        size_t maps = 1, states = 1;
        for (const ExecBlock &B : P.blocks)
            if (B.tri && B.band_w > 0) {
                maps = std::max(maps, (size_t)band_blocks(B.band_nch) * (B.band_w * B.band_w + B.band_w));
                states = std::max(states, ((size_t)band_blocks(B.band_nch) + 1) * sizeof(int) / sizeof(double) + 1);
            }
        D.band_maps1 = maps;  // per right-hand side; allocated with the work vectors
        D.band_states1 = states;
    }
    if (D.mixed) {
        const auto c32 = to_f32(P.band_coef), i32 = to_f32(P.band_inv);
        if ((rc = upload(D, D.band_coef32, c32, err))) return rc;
        if ((rc = upload(D, D.band_inv32, i32, err))) return rc;
    }
    if ((rc = upload(D, D.ell_col, P.ell_col, err))) return rc;
    if ((rc = upload(D, D.ell_val, P.ell_val, err))) return rc;
    {
        std::vector<EllChunk> ec(P.ell_chunks.size() / 4);
        std::memcpy(ec.data(), P.ell_chunks.data(), ec.size() * sizeof(EllChunk));
        if ((rc = upload(D, D.ell_chunks, ec, err))) return rc;
    }
    if ((rc = upload(D, D.ca_tab, P.ca_tab, err))) return rc;
    if ((rc = upload(D, D.ca_col, P.ca_col, err))) return rc;
    {
        // window slots (0..CA_WINDOW_ROWS) fit 16 bits; other blocks' entries stay 0
        std::vector<short> c16(P.ca_col.size(), 0);
        for (const ExecBlock &B : P.blocks)
            if (B.tri && B.ca_ok && B.ca_win && B.ca_w >= 2)
                for (long long e = B.ca_lo; e < B.ca_hi; ++e) c16[(size_t)e] = (short)P.ca_col[(size_t)e];
        if ((rc = upload(D, D.ca_col16, c16, err))) return rc;
    }
    if ((rc = upload(D, D.ca_val, P.ca_val, err))) return rc;
    if (D.mixed) {
        const auto c32 = to_f32(P.ca_val);
        if ((rc = upload(D, D.ca_val32, c32, err))) return rc;
    }
    if (D.mixed) {
        const auto e32 = to_f32(P.ell_val);
        if ((rc = upload(D, D.ell_val32, e32, err))) return rc;
    }
    if (!P.lc_tab.empty()) {
        std::vector<LcChunk> tab(P.lc_tab.size() / LC_TAB_INTS);
        std::memcpy(tab.data(), P.lc_tab.data(), tab.size() * sizeof(LcChunk));
        if ((rc = upload(D, D.lc_tab, tab, err))) return rc;
        if ((rc = upload(D, D.lc_rec64, P.lc_rec64, err))) return rc;
        if (D.mixed && (rc = upload(D, D.lc_rec32, P.lc_rec32, err))) return rc;
        std::vector<LcSeg> segs(P.lc_segs.size() / 3);
        for (size_t q = 0; q < segs.size(); ++q)
            segs[q] = LcSeg{D.lc_tab + P.lc_segs[3 * q], P.lc_segs[3 * q + 1], P.lc_segs[3 * q + 2]};
        if ((rc = upload(D, D.lc_segs, segs, err))) return rc;
        if ((rc = alloc(D, D.lc_queue, (size_t)(1 << P.lv), err))) return rc;
    }
    {
        int prio_low = 0, prio_high = 0;
        CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
        CK(cudaStreamCreateWithPriority(&D.side, cudaStreamNonBlocking, prio_low));
    }
    CK(cudaEventCreateWithFlags(&D.ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&D.ev_join, cudaEventDisableTiming));
    D.ntri = 1 << P.lv;
    if ((rc = alloc(D, D.iotab, 2 * RBS_IO_COLS, err))) return rc;
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

void pipe_release(DeviceState &D) {
    DeviceState::HostPipe &H = D.pipe;
    if (H.cin) cudaStreamSynchronize(H.cin);
    if (H.cout) cudaStreamSynchronize(H.cout);
    for (int s = 0; s < 2; ++s) {
        cudaFree(H.db[s]);
        cudaFree(H.dx[s]);
        H.db[s] = H.dx[s] = nullptr;
        for (cudaEvent_t *e : {&H.in_done[s], &H.solved[s], &H.out_done[s]})
            if (*e) {
                cudaEventDestroy(*e);
                *e = nullptr;
            }
        H.used[s] = false;
    }
    D.bytes -= 4 * (long long)H.bytes;
    H.bytes = 0;
    if (H.cin) cudaStreamDestroy(H.cin);
    if (H.cout) cudaStreamDestroy(H.cout);
    H.cin = H.cout = nullptr;
}

int device_host_async(Plan &P, const double *b, double *x, int k, int ld, int prec, std::string &err) {
    DeviceState &D = *P.dev;
    DeviceState::HostPipe &H = D.pipe;
    const size_t bytes = sizeof(double) * (size_t)ld * (size_t)k;
    if (!H.cin) {
        CK(cudaStreamCreateWithFlags(&H.cin, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&H.cout, cudaStreamNonBlocking));
        for (int s = 0; s < 2; ++s) {
            CK(cudaEventCreateWithFlags(&H.in_done[s], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&H.solved[s], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&H.out_done[s], cudaEventDisableTiming));
        }
    }
    if (bytes > H.bytes) {  // wider than before: drain, then larger slots
        CK(cudaStreamSynchronize(D.stream));
        CK(cudaStreamSynchronize(H.cin));
        CK(cudaStreamSynchronize(H.cout));
        for (int s = 0; s < 2; ++s) {
            cudaFree(H.db[s]);
            cudaFree(H.dx[s]);
            H.db[s] = H.dx[s] = nullptr;
            H.used[s] = false;
        }
        D.bytes -= 4 * (long long)H.bytes;
        H.bytes = 0;
        int rc;
        for (int s = 0; s < 2; ++s) {
            if ((rc = alloc(D, H.db[s], bytes / sizeof(double), err))) return rc;
            if ((rc = alloc(D, H.dx[s], bytes / sizeof(double), err))) return rc;
        }
        H.bytes = bytes + 256;
    }
    const int s = H.next;
    H.next ^= 1;
    const size_t nbytes = sizeof(double) * (size_t)P.n;
    // the slot's previous solve has read db[s]; its previous download has read dx[s]
    if (H.used[s]) {
        CK(cudaStreamWaitEvent(H.cin, H.solved[s], 0));
        CK(cudaStreamWaitEvent(D.stream, H.out_done[s], 0));
    }
    for (int c = 0; c < k; ++c)
        CK(cudaMemcpyAsync(H.db[s] + (size_t)c * ld, b + (size_t)c * ld, nbytes, cudaMemcpyHostToDevice, H.cin));
    CK(cudaEventRecord(H.in_done[s], H.cin));
    CK(cudaStreamWaitEvent(D.stream, H.in_done[s], 0));
    int rc = device_solve(P, H.db[s], H.dx[s], k, ld, prec, false, nullptr, err);
    if (rc) return rc;
    CK(cudaEventRecord(H.solved[s], D.stream));
    CK(cudaStreamWaitEvent(H.cout, H.solved[s], 0));
    for (int c = 0; c < k; ++c)
        CK(cudaMemcpyAsync(x + (size_t)c * ld, H.dx[s] + (size_t)c * ld, nbytes, cudaMemcpyDeviceToHost, H.cout));
    CK(cudaEventRecord(H.out_done[s], H.cout));
    H.used[s] = true;
    return RBS_OK;
}

namespace {

void drop_descs(DeviceState &D) {
    for (auto &kv : D.desc_cache) cudaFree(kv.second);
    D.desc_cache.clear();
    for (auto &kv : D.ell_cache) cudaFree(kv.second);
    D.ell_cache.clear();
    for (auto &kv : D.ca_cache) cudaFree(kv.second);
    D.ca_cache.clear();
    drop_graphs(D);
}

// RBS_SELECT_TUNE: run the plan with every triangle on one candidate kernel
// at a time (sync-free; the single-CTA level kernels: level chunks, staged
// level-ELL, CTA sync-free, plain; band scan where a band layout exists),
// time each triangle with CUDA events, and keep for every triangle the
// fastest.  Squares keep their SpMV plan.
int tune_kernels(Plan &P, std::string &err) {
    DeviceState &D = *P.dev;
    const size_t nb = P.blocks.size();
    std::vector<int> orig(nb), origv(nb);
    for (size_t b = 0; b < nb; ++b) {
        orig[b] = P.blocks[b].kernel;
        origv[b] = P.blocks[b].lvl_var;
    }
    std::vector<double> best(nb, 1e300);
    std::vector<int> pick(orig), pickv(origv);
    double *db = nullptr, *dx = nullptr;
    CK(cudaMalloc(&db, sizeof(double) * (size_t)P.n));
    CK(cudaMalloc(&dx, sizeof(double) * (size_t)P.n));
    k_fill<double><<<grid_for(P.n, 256, D.num_sms), 256, 0, D.stream>>>(db, P.n, 1.0);
    int rc = RBS_OK;
    // (kernel, single-CTA level variant) candidates
    const int cands[6][2] = {{RBS_K_SYNCFREE, LVL_PLAIN}, {RBS_K_LEVEL, LVL_LC},  {RBS_K_LEVEL, LVL_CA},
                             {RBS_K_LEVEL, LVL_CSF},      {RBS_K_LEVEL, LVL_PLAIN}, {RBS_K_BANDSCAN, LVL_PLAIN}};
    for (int ci = 0; ci < 6 && rc == RBS_OK; ++ci) {
        const int cand = cands[ci][0], var = cands[ci][1];
        bool any = false;
        for (size_t b = 0; b < nb; ++b) {
            ExecBlock &B = P.blocks[b];
            if (!B.tri || B.nnz == B.m) continue;
            bool ok = true;
            if (cand == RBS_K_BANDSCAN) ok = B.band_w > 0;
            if (cand == RBS_K_LEVEL)
                ok = var == LVL_LC ? B.lc_ok : var == LVL_CA ? B.ca_ok : var == LVL_CSF ? B.ell_ok : B.lvl_off >= 0;
            B.kernel = ok ? cand : orig[b];
            B.lvl_var = ok ? var : origv[b];
            any = any || ok;
        }
        if (!any) continue;
        drop_descs(D);
        if ((rc = device_profile(P, 1, err))) break;
        for (int rep = 0; rep < 3 && rc == RBS_OK; ++rep) {
            if (rep == 1 && (rc = device_profile(P, 1, err))) break;  // first solve is the warm-up
            rc = device_solve(P, db, dx, 1, P.n, RBS_PREC_FP64, true, nullptr, err);
        }
        if (rc) break;
        std::vector<double> ms;
        long long solves = 0;
        device_block_times(P, ms, solves);
        for (size_t b = 0; b < nb; ++b) {
            const ExecBlock &B = P.blocks[b];
            if (!B.tri || B.nnz == B.m || B.kernel != cand || B.lvl_var != var) continue;
            const double t = ms[b] / std::max(1ll, solves);
            if (t < best[b]) {
                best[b] = t;
                pick[b] = cand;
                pickv[b] = var;
            }
        }
    }
    for (size_t b = 0; b < nb; ++b) {
        P.blocks[b].kernel = rc == RBS_OK ? pick[b] : orig[b];
        P.blocks[b].lvl_var = rc == RBS_OK ? pickv[b] : origv[b];
    }
    drop_descs(D);
    device_profile(P, 0, err);
    cudaFree(db);
    cudaFree(dx);
    return rc;
}

}  // namespace

int device_tune(Plan &P, std::string &err) {
    if (!P.dev) {
        err = "plan has no device state";
        return RBS_ERR_ARG;
    }
    return tune_kernels(P, err);
}

void device_free(Plan &P) {
    if (!P.dev) return;
    DeviceState &D = *P.dev;
    if (D.stream) cudaStreamSynchronize(D.stream);
    pipe_release(D);
    free_work(D);
    drop_graphs(D);
    for (auto &e : D.bev) cudaEventDestroy(e);
    if (D.side) cudaStreamSynchronize(D.side);
    if (D.side) cudaStreamDestroy(D.side);
    if (D.ev_fork) cudaEventDestroy(D.ev_fork);
    if (D.ev_join) cudaEventDestroy(D.ev_join);
    for (auto &e : D.ov_ev) cudaEventDestroy(e);
    cudaFree(D.iotab);
    cudaFree(D.io_rows);
    cudaFree(D.ell_col);
    cudaFree(D.ell_val);
    cudaFree(D.ell_val32);
    cudaFree(D.ell_chunks);
    cudaFree(D.ca_tab);
    cudaFree(D.ca_col);
    cudaFree(D.ca_col16);
    cudaFree(D.ca_val);
    cudaFree(D.ca_val32);
    cudaFree(D.lc_rec64);
    cudaFree(D.lc_rec32);
    cudaFree(D.lc_tab);
    cudaFree(D.lc_segs);
    cudaFree(D.lc_queue);
    cudaFree(D.stage_b);
    cudaFree(D.stage_x);
    void *ptrs[] = {D.rp, D.col, D.lvl, D.map, D.rows, D.perm, D.ipos, D.val, D.inv, D.val32, D.inv32,
                    D.full_rp, D.full_col, D.full_val, D.tickets, D.status, D.norms, D.band_coef,
                    D.band_inv, D.band_coef32, D.band_inv32};
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
        int prio_low = 0, prio_high = 0;
        CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
        CK(cudaStreamCreateWithPriority(&D.stream, cudaStreamNonBlocking, prio_high));
        D.own_stream = true;
    }
    return RBS_OK;
}

int device_sync(Plan &P, std::string &err) {
    DeviceState &D = *P.dev;
    CK(cudaMemcpyAsync(D.h_status, D.status, sizeof(int), cudaMemcpyDeviceToHost, D.stream));
    CK(cudaStreamSynchronize(D.stream));
    if (D.pipe.cout) CK(cudaStreamSynchronize(D.pipe.cout));  // asynchronous host-array solves' downloads
    if (*D.h_status & RBS_STATUS_TIMEOUT) {
        CK(cudaMemsetAsync(D.status, 0, sizeof(int), D.stream));
        // the solution work vectors may hold leftovers of the aborted solve
        size_t cnt = (size_t)P.n * D.kcap;
        if (D.xw64)
            k_fill<double><<<grid_for((long long)cnt, 256, D.num_sms), 256, 0, D.stream>>>(
                D.xw64, (long long)cnt, sent64_host());
        if (D.xw32)
            k_fill<float><<<grid_for((long long)cnt, 256, D.num_sms), 256, 0, D.stream>>>(
                D.xw32, (long long)cnt, sent32_host());
        D.xw_dirty64 = D.xw_dirty32 = false;
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
        cudaGetLastError();  // a block without kernels has no timing: do not leave the error behind
        ++D.bsolves;
    }
    if (stats) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, D.ev0, D.ev1) != cudaSuccess) cudaGetLastError();
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
