// rbs_internal.h -- plan layout shared by the host analysis and the executor.
//
// Orders used in this library
//   original row i      : the caller's numbering
//   reference label     : the reference's level-set relabelling
//                         (utils_reordering.h:130-159): forward label =
//                         position in the BFS level order, backward label =
//                         m-1-position
//   processing position : the order in which rows are solved.  Forward:
//                         p = label.  Backward: p = m-1-label (= BFS
//                         position).  In processing order every system is
//                         LOWER triangular, so every kernel is written once
//                         for forward substitution.
//
// In processing order the recursive-block geometry of both directions is the
// forward geometry of recblocking_preprocess.h:57-178: triangle i covers
// rows [i*s, (i+1)*s) (the last one runs to m), and the square after t
// triangles covers rows [t*s, (t+lowbit(t))*s) x cols [(t-lowbit(t))*s, t*s)
// (rows run to m when t+lowbit(t) == 2^lv).
#pragma once

#include <cuda_runtime_api.h>
#include <sys/mman.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "rbs.h"

namespace rbs {

// Allocator of the plan's arrays of matrix entries (input, processing-order
// and pool layouts).  resize() leaves new elements uninitialised: each of
// these arrays is written in full by the pass that sizes it, on host
// threads, so its pages are first touched in parallel instead of zeroed by
// one thread.  Blocks of 32 MB or more are 2 MB aligned and advised for
// transparent huge pages.
template <typename T> struct BulkAlloc {
    using value_type = T;
    BulkAlloc() noexcept = default;
    template <typename U> BulkAlloc(const BulkAlloc<U> &) noexcept {}
    T *allocate(size_t n) {
        constexpr size_t kHuge = size_t(2) << 20;
        const size_t bytes = n * sizeof(T);
        void *p;
        if (bytes >= 16 * kHuge) {
            const size_t rounded = (bytes + kHuge - 1) & ~(kHuge - 1);
            p = std::aligned_alloc(kHuge, rounded);
            if (p) madvise(p, rounded, MADV_HUGEPAGE);
        } else {
            p = std::malloc(bytes ? bytes : 1);
        }
        if (!p) throw std::bad_alloc();
        return static_cast<T *>(p);
    }
    void deallocate(T *p, size_t) noexcept { std::free(p); }
    template <typename U> void construct(U *p) noexcept { ::new ((void *)p) U; }
    template <typename U, typename... A> void construct(U *p, A &&...a) { ::new ((void *)p) U(std::forward<A>(a)...); }
};
template <typename T, typename U> bool operator==(const BulkAlloc<T> &, const BulkAlloc<U> &) { return true; }
template <typename T, typename U> bool operator!=(const BulkAlloc<T> &, const BulkAlloc<U> &) { return false; }
template <typename T> using bulk_vector = std::vector<T, BulkAlloc<T>>;

// Host threads of the analysis: RBS_HOST_THREADS (1..64) when set, else the
// hardware's, at most 16.  Results do not depend on the count.
inline unsigned host_threads() {
    static const unsigned n = [] {
        const char *e = std::getenv("RBS_HOST_THREADS");
        const int v = e ? std::atoi(e) : 0;
        if (v >= 1) return (unsigned)std::min(v, 64);
        return std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    }();
    return n;
}

// fn(i) for every i in [0, count) on up to host_threads() threads (an
// atomic work counter); fn writes only what index i owns.
template <typename F> void parallel_for(size_t count, F &&fn) {
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t i; (i = next.fetch_add(1)) < count;) fn(i);
    };
    const unsigned nth = (unsigned)std::min<size_t>(count, host_threads());
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nth; ++t) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
}

// FP32 copy of an FP64 array (each value rounded to nearest), converted on
// host threads.
template <typename V> bulk_vector<float> to_f32(const V &src) {
    bulk_vector<float> out(src.size());
    constexpr size_t kChunk = size_t(1) << 20;
    parallel_for((src.size() + kChunk - 1) / kChunk, [&](size_t c) {
        const size_t e = std::min(src.size(), (c + 1) * kChunk);
        for (size_t i = c * kChunk; i < e; ++i) out[i] = (float)src[i];
    });
    return out;
}

// Smallest i in [0, count) with bad(i), or -1 (chunks scanned on host
// threads): the index a serial check would stop at.
template <typename F> long long first_bad(long long count, F &&bad) {
    constexpr long long kChunk = 1 << 18;
    const size_t nchunk = (size_t)((count + kChunk - 1) / kChunk);
    std::vector<long long> found(nchunk, -1);
    parallel_for(nchunk, [&](size_t c) {
        for (long long i = (long long)c * kChunk, e = std::min(count, i + kChunk); i < e; ++i)
            if (bad(i)) {
                found[c] = i;
                return;
            }
    });
    for (long long f : found)
        if (f >= 0) return f;
    return -1;
}

// Per-block execution record (processing order).  Offsets index the pools
// of the plan.
struct ExecBlock {
    int index;          // block index in the reference's order (T0, S1, T2, ...)
    int tri;            // 1 triangle, 0 square
    int r0, m;          // rows [r0, r0+m)
    int c0, ncols;      // squares: columns [c0, c0+ncols); triangles: c0 = r0
    int nnz;            // reference blk_nnz (triangles include the diagonal)
    int ref_method;     // reference method code (recblocking_preprocess.h:472-709, 835-922)
    int kernel;         // RBS_K_*
    int group;          // lanes per row for k == 1
    // triangles
    int sf_group;       // lanes per row of the sync-free kernel for k == 1: sized for the row-length tail
    int nlv;            // local level count
    int contiguous;     // 1 if local levels are contiguous row ranges in processing order
    int bandwidth;      // max over rows of (p - smallest column) inside the triangle
    int maxwidth;       // widest local level
    long long lvl_off;  // level pointer pool offset (nlv+1 entries)
    long long map_off;  // row list offset (m entries) when !contiguous, else -1
    // all blocks
    long long rp_off;   // row pointer pool offset (m+1 entries, or nrows+1 for DCSR)
    int nrows;          // rows listed in the row pointer (m, or nonempty rows for DCSR)
    long long rows_off; // DCSR row list offset or -1
    int nonempty;       // squares: nonempty rows
    int longrows;       // squares: rows longer than 2048 (handled by the split kernel)
    long long long_off; // long-row list offset or -1
    int medrows;        // squares with a lane group < 32: rows of 9..2048 entries (a warp each, single RHS)
    long long med_off;  // medium-row list offset or -1
    int lenmax;
    // band-scan triangles: W = power of two >= bandwidth, chunks of C rows
    int band_w, band_c, band_nch;
    long long band_off;  // coefficient pool offset (band_nch*band_c*band_w); inverse pool at band_off / band_w
    // level triangles staged per thread with cp.async (level-ELL layout);
    // ca_win: every dependency lies within the last CA_WINDOW_ROWS rows of
    // its level's end, and columns are stored as window slots (padding ->
    // the always-zero slot CA_WINDOW_ROWS)
    int ca_ok, ca_w, ca_win;
    long long ca_tab_off;     // level table offset in ca_tab (3*nlv+1 ints)
    long long ca_lo, ca_hi;   // element range of the block in the level-ELL pools
    // single-CTA triangles in ELL chunks (CTA sync-free kernel)
    int ell_ok, ell_nchunks;
    long long ell_chunk_off;  // first chunk in ell_chunks (4 ints per chunk: R0, R1, W, pool offset)
    long long ell_lo, ell_hi; // element range of the block in the ELL pools
    // single-CTA triangles in level chunks (bulk-copied records, level_lc.cuh)
    int lc_ok, lc_nseg;
    long long lc_seg_off;     // first segment in lc_segs (3 ints per segment)
    // which single-CTA level kernel runs a RBS_K_LEVEL triangle
    int lvl_var;              // LVL_* below
};

// rows of the shared-memory x window of the staged level kernel (power of 2)
constexpr int CA_WINDOW_ROWS = 4096;
// Row-length classes of the squares (single right-hand side, narrow lane
// group): rows of more than SQ_MEDROW entries, up to SQ_LONGROW, are listed
// for a warp each; longer rows are split over warps (utils_spmv_cuda.h:9
// LONGROW_THRESHOLD).  The kernels' RBS_MEDROW / RBS_LONGROW are the same.
constexpr int SQ_MEDROW = 8;
constexpr int SQ_LONGROW = 2048;

// single-CTA level kernels of a RBS_K_LEVEL triangle
enum { LVL_PLAIN = 0, LVL_CA = 1, LVL_CSF = 2, LVL_LC = 3 };

struct DeviceState;  // executor side (solve.cu)

// The reference-format packed arrays (recblock_Ptr/Index/Val, DCSR row
// lists, block offsets, local level sets), rebuilt from a plan by
// export_reference on the first request and kept with the plan.
struct RefPack {
    std::vector<int> ptr_offset, index_offset, dcsr_offset;
    std::vector<int> Ptr, Index, Dcsr;
    std::vector<double> Val;
    std::vector<int> nlv, longrow, m_new_dcsr;
    std::vector<int> lvl_ptr, lvl_item, m_lv, off_lv, nnz_lv;
};

struct Plan {
    int n = 0, nnz = 0, lv = 0, sub = 0, nlevel = 0, sum_block = 0, step = 0;
    rbs_options opt{};
    double analyse_ms = 0;
    double device_analyse_ms = 0;  // part of analyse_ms spent in the device analysis (0: host analysis)
    int device_bfs = 0;            // 1: the level search itself ran on the device

    // inputs kept for the reference-format export (CSC, caller's entry order)
    std::vector<int> in_cp;
    bulk_vector<int> in_ri;
    bulk_vector<double> in_va;
    std::vector<int> bfs_item;   // BFS level order (findlevel.h:7-83)
    std::vector<int> bfs_ptr;    // level pointers (nlevel+1)
    std::vector<int> label;      // original row -> reference label

    // processing order
    std::vector<int> perm;       // processing position -> original row
    std::vector<ExecBlock> blocks;
    // pools (uploaded to the device)
    std::vector<int> rp_pool, lvl_pool, map_pool, rows_pool;
    bulk_vector<int> col_pool;
    bulk_vector<double> val_pool;
    std::vector<double> inv_diag;
    std::vector<double> band_coef, band_inv;  // chunk-interleaved band layout of band-scan triangles
    bulk_vector<int> ell_col;                  // ELL columns of single-CTA triangles (-1 = padding)
    bulk_vector<double> ell_val;
    std::vector<int> ell_chunks;
    std::vector<int> ca_tab, ca_col;           // level tables and level-ELL columns (-1 = padding)
    std::vector<double> ca_val;
    // level-chunk records (level_lc.cuh): 16-byte words of the FP64 and FP32
    // layouts, one LcChunk (lc_layout.h) per chunk, 3 ints per segment (first
    // chunk, chunks, ring offset of the first chunk)
    bulk_vector<uint32_t> lc_rec64, lc_rec32;
    std::vector<int> lc_tab, lc_segs;
    // original-row offsets of independent systems (batched plans); empty
    // for a single system
    std::vector<int> seg_rows;
    // the reference's reordered CSC (utils_reordering.h:102-210) as computed
    // by the device analysis (rbs_analyse_device); empty after a host analysis
    std::vector<int> dev_reorder_cp, dev_reorder_ri;
    // full processing-order CSR (with diagonal) for FP64 residuals
    std::vector<int> full_rp;
    bulk_vector<int> full_col;
    bulk_vector<double> full_val;

    DeviceState *dev = nullptr;
    // reference-format export cache (export_reference); exports of one plan
    // from several threads at once are not supported
    mutable std::shared_ptr<const RefPack> ref_pack;
};

// analysis.cpp
int analyse_host(Plan &P, const int *ptr, const int *idx, const double *val, int n, int nnz, int fmt,
                 int substitution, int lv, const rbs_options &opt, std::string &err,
                 const std::vector<int> *seg_rows = nullptr);
int export_reference(const Plan &P, const std::string &name, std::vector<int> &iv, std::vector<double> &dv,
                     bool &is_double, std::string &err);
int auto_lv(int m, int device_id);

// The processing-order CSR that device_analyse leaves on the device for the
// block extraction on the device (dev_pools.cu), with that step's buffers.
// The memory comes from the per-device pool and is released, stream-ordered,
// with the object.
struct DevRows {
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;
    int *frp = nullptr, *fcol = nullptr;
    double *fval = nullptr;
    int *rowcnt = nullptr, *status = nullptr;
    long long *slot_base = nullptr;
    int n = 0, nnz = 0, sms = 148;
    DevRows() = default;
    DevRows(const DevRows &) = delete;
    DevRows &operator=(const DevRows &) = delete;
    ~DevRows();
};

// dev_analysis.cu: validation, findlevel, reordering and the processing-order
// CSR on the device (fills in_*, bfs_*, nlevel, label, perm, full_*,
// dev_reorder_*); with keep, the processing-order CSR also stays on the
// device in *keep
int device_analyse(Plan &P, const int *d_ptr, const int *d_idx, const double *d_val, int n, int nnz, int fmt,
                   int substitution, std::string &err, DevRows *keep = nullptr);
// dev_pools.cu: per (block, row) entry counts (blocks in order, slot_base[b]
// = first slot of block b), inverse diagonal and reach of every row
int dev_block_counts(DevRows &R, int T, int s, const std::vector<long long> &slot_base, std::vector<int> &rowcnt,
                     std::vector<double> &inv_diag, std::vector<int> &reach, std::string &err);
// dev_pools.cu: local levels of the triangles (T > 1)
int dev_local_levels(DevRows &R, int T, int s, long long spin_limit, std::vector<int> &level, std::string &err);
// dev_pools.cu: the entry pools (col_pool, val_pool) from the counts
int dev_pool_fill(DevRows &R, int T, int s, long long slots, long long entries, bulk_vector<int> &col_pool,
                  bulk_vector<double> &val_pool, std::string &err);
// analysis.cpp: findlevel's breadth-first search on the host (levelPtr, levelItem;
// returns the level count or -1 when stuck)
int host_bfs_levels(const int *cp, const int *ri, int m, std::vector<int> &levelPtr, std::vector<int> &item);
// analysis.cpp: the layout steps after the level sets, from the fields
// device_analyse filled
int analyse_after_levels(Plan &P, int n, int nnz, int substitution, int lv, const rbs_options &opt, std::string &err,
                         const std::vector<int> *seg_rows = nullptr, DevRows *dev_rows = nullptr);

// ilu0.cu: ILU(0) of a device CSR matrix into d_lu (A's pattern)
int device_ilu0(const int *d_rp, const int *d_ci, const double *d_val, int n, int nnz, double *d_lu,
                const rbs_options &opt, std::string &err);
// ilu0.cu: IC(0) of an SPD matrix's lower-triangle CSR into d_l (its pattern)
int device_ic0(const int *d_rp, const int *d_ci, const double *d_val, int n, int nnz, double *d_l,
               const rbs_options &opt, std::string &err);

// mtx.cu: the per-device stream-ordered memory pool for temporaries
// (allocate with cudaMallocFromPoolAsync, free with cudaFreeAsync)
cudaError_t device_mem_pool(int dev, cudaMemPool_t &pool);

// mtx.cu: a Matrix Market coordinate file parsed on the device into CSR
// (mmio_data's layout: rows ascending, file order inside a row, symmetric
// files mirrored); rowof holds the row of every entry
struct DeviceMtx {
    int m = 0, n = 0, field = 0, symmetric = 0, device = 0;
    long long nnz_file = 0, nnz = 0, nnz_lower = 0, nnz_upper = 0, host_values = 0;
    double read_ms = 0, parse_ms = 0;
    int *rowptr = nullptr, *colidx = nullptr, *rowof = nullptr;
    double *val = nullptr;
};
// path != NULL: read the file; else parse bytes[0, len) from host memory
int mtx_read(const char *path, const void *bytes, long long len, const rbs_options &opt, DeviceMtx &M,
             std::string &err);
int mtx_csr(const DeviceMtx &M, int *d_rowptr, int *d_colidx, double *d_val, std::string &err);
// the unit-diagonal triangle of main.cu:157-198 in CSR or CSC (fmt)
int mtx_triangle(const DeviceMtx &M, int substitution, int fmt, const double *d_strict, int *d_ptr, int *d_idx,
                 double *d_val, std::string &err);
void mtx_free(DeviceMtx &M);
int mtx_write(const char *path, int m, int n, const int *rp, const int *ci, const double *val, int symmetric,
              std::string &err);

// plan_io.cpp: the plan's host side to and from a file
int plan_save(const Plan &P, const char *path, std::string &err);
int plan_load(Plan &P, const char *path, std::string &err);

// solve.cu
int device_build(Plan &P, std::string &err);
void device_free(Plan &P);
int device_solve(Plan &P, const double *d_b, double *d_x, int k, int ld, int prec, bool sync,
                 rbs_stats *stats, std::string &err);
int device_sync(Plan &P, std::string &err);
int device_finish(Plan &P, rbs_stats *stats, int k, int prec, std::string &err);
void *device_stream(Plan &P);
int device_set_stream(Plan &P, void *stream, std::string &err);
int device_profile(Plan &P, int enable, std::string &err);
int device_tune(Plan &P, std::string &err);
int device_block_times(const Plan &P, std::vector<double> &ms, long long &solves);
int device_staging(Plan &P, size_t bytes, double *&db, double *&dx, std::string &err);
// host-array solve enqueued without waiting: upload on a copy stream,
// solve on the plan's stream, download on another copy stream; two staging
// slots in turn (device_sync waits for everything)
int device_host_async(Plan &P, const double *b, double *x, int k, int ld, int prec, std::string &err);
// work vectors for k right-hand sides allocated now, so solves up to that
// width allocate nothing
int device_reserve(Plan &P, int k, std::string &err);
// Asynchronous solve of k columns on the plan's stream: bcols / xcols are
// device tables of k column pointers (right-hand sides read, solutions
// written).  After start, and after every next that sets *more, the caller
// waits for the stream and calls next again while *more is set (mixed
// refinement: one correction per call); then finish reports the status.
// The systems of a block-diagonal plan (rbs_batch_analyse) served as one
// unit: column c of system f reads btab[c*count + f] and writes
// xtab[c*count + f] (device tables; NULL: no request, zeros in and nothing
// out); seg[i] is the system of original row i and off[f] its first row
// (device arrays).  With it, device_batch_start ignores bcols / xcols.
struct BatchGroup {
    const double *const *btab;
    double *const *xtab;
    const int *seg, *off;
    int count;
};
int device_batch_start(Plan &P, const double *const *bcols, double *const *xcols, int k, int prec, int *more,
                       std::string &err, const BatchGroup *grp = nullptr);
int device_batch_next(Plan &P, int *more, std::string &err);
int device_batch_finish(Plan &P, int *iters, double *corr, std::string &err);
double block_bytes(const Plan &P, const ExecBlock &B);
long long device_bytes(const Plan &P);

void set_error(const std::string &msg);

}  // namespace rbs

// the opaque handle of include/rbs.h
struct rbs_plan {
    rbs::Plan p;
};
