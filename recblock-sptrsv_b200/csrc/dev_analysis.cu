// dev_analysis.cu -- the reference's level-set analysis rebuilt on the
// device: input validation, findlevel (findlevel.h:7-83, device version
// utils_cuda.h:29-97), level-set reordering (utils_reordering.h:102-210,
// device version utils_cuda.h:706-779) and the stable CSR/CSC
// transpositions (tranpose.h:7-54, utils_cuda.h:644-670).  Integer outputs
// are bit-identical to the reference's; the plan layout is then built from
// them by the host (analysis.cpp).
//
// findlevel is Kahn's breadth-first search: in-degree = entries per row
// (diagonal included), level 0 = rows whose only entry is the diagonal in
// ascending row order, and while walking level l in its discovery order and
// each column in stored order, a row joins level l+1 the moment its
// in-degree drops to 1.  In parallel, one level at a time:
//   expand  every entry (row r, column p) of the level's columns decrements
//           deg[r] and raises key[r] to the (global) BFS position of p;
//   count   a row r that reached deg 1 during this level is a child of the
//           parent p whose position equals key[r] -- the parent processed
//           last in serial order, i.e. the one whose decrement was final;
//   write   the parents, in level order, append their children in column
//           order at offsets given by a scan of the counts.
// This reproduces the serial discovery order exactly.  Narrow levels run
// inside one persistent CTA (several levels per launch); a level wider than
// BFS_MAXF rows runs as grid-wide kernels.
//
// Integer sorts (stable radix sort) and scans use CUB, the
// CUDA toolkit's primitives; the reference uses thrust for the same steps
// (utils_cuda.h:659,725,741,752).
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "rbs_internal.h"

namespace rbs {

namespace {

constexpr int BFS_T = 1024;
constexpr int BFS_MAXF = 4096;   // widest level the single-CTA kernel takes (rows)
constexpr int BFS_EMAX = 16384;  // and column entries
constexpr int BFS_SMEM = (BFS_MAXF + 1 + 2 * BFS_EMAX) * 4;

enum { BFS_DONE = 1, BFS_BIG = 2, BFS_STUCK = 3, BFS_PAUSED = 4 };
constexpr int BFS_PAUSE = 2048;        // levels per launch of the single-CTA kernel
constexpr int BFS_NARROW = 16;         // mean rows per level below which ...
constexpr int BFS_HOST_ROWS = 65536;   // ... and with more rows than this left, the host takes over
enum { VAL_PTR = 1, VAL_NODIAG, VAL_DIAGPOS, VAL_ZERODIAG, VAL_OUTSIDE, VAL_DUPDIAG, VAL_INDEX };

#define DCK(call)                                                                    \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            err = std::string("device analysis: ") + #call + ": " + cudaGetErrorString(e_); \
            return RBS_ERR_CUDA;                                                     \
        }                                                                            \
    } while (0)

int grid_of(long long work, int threads) {
    long long g = (work + threads - 1) / threads;
    return (int)std::max(1LL, std::min(g, 148LL * 16));
}

// One failing column at most is reported: the smallest, with its error kind.
__global__ void k_validate(const int *__restrict__ cp, const int *__restrict__ ri, const double *__restrict__ va,
                           int n, int nnz, int fwd, unsigned long long *bad) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int b = cp[c], e = cp[c + 1];
        int code = 0;
        if (b < 0 || e < b || e > nnz) code = VAL_PTR;
        else if (b == e) code = VAL_NODIAG;
        else {
            const int dpos = fwd ? b : e - 1;
            if (ri[dpos] != c) code = VAL_DIAGPOS;
            else if (va[dpos] == 0.0) code = VAL_ZERODIAG;
            else
                for (int k = b; k < e && !code; ++k) {
                    const int r = ri[k];
                    if (r < 0 || r >= n) code = VAL_INDEX;
                    else if (fwd ? r < c : r > c) code = VAL_OUTSIDE;
                    else if (k != dpos && r == c) code = VAL_DUPDIAG;
                }
        }
        if (code) atomicMin(bad, ((unsigned long long)c << 8) | (unsigned long long)code);
    }
}

__global__ void k_check_csr(const int *__restrict__ rp, const int *__restrict__ ci, int n, int nnz,
                            unsigned long long *bad) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int b = rp[r], e = rp[r + 1];
        int code = 0;
        if (b < 0 || e < b || e > nnz) code = VAL_PTR;
        else
            for (int k = b; k < e && !code; ++k)
                if (ci[k] < 0 || ci[k] >= n) code = VAL_INDEX;
        if (code) atomicMin(bad, ((unsigned long long)r << 8) | (unsigned long long)code);
    }
}
__global__ void k_entry_rows(const int *__restrict__ rp, int n, int *rows) {
    const int lane = threadIdx.x & 31;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5)
        for (int k = rp[r] + lane; k < rp[r + 1]; k += 32) rows[k] = r;
}

__global__ void k_degree(const int *__restrict__ ri, long long nnz, int *deg) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x)
        atomicAdd(deg + ri[k], 1);
}

__global__ void k_root_flags(const int *__restrict__ deg, int n, int *flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flag[i] = deg[i] == 1;
}
__global__ void k_root_scatter(const int *__restrict__ flag, const int *__restrict__ pos, int n, int *item) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) item[pos[i]] = i;
}

// Block-wide exclusive scan of v[0, n) in place (n <= BFS_EMAX), returns the
// total; every thread of the CTA calls it.
__device__ int block_exclusive_scan(int *v, int n, int *wsum) {
    const int tid = threadIdx.x;
    const int per = (n + BFS_T - 1) / BFS_T;
    const int a = min(n, tid * per), z = min(n, a + per);
    int run = 0;
    for (int t = a; t < z; ++t) run += v[t];
    int incl = run;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if ((tid & 31) >= o) incl += u;
    }
    if ((tid & 31) == 31) wsum[tid >> 5] = incl;
    __syncthreads();
    if (tid < 32) {
        int w = tid < BFS_T / 32 ? wsum[tid] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, w, o);
            if (tid >= o) w += u;
        }
        if (tid < BFS_T / 32) wsum[tid] = w;
    }
    __syncthreads();
    int base = incl - run + ((tid >> 5) ? wsum[(tid >> 5) - 1] : 0);
    const int total = wsum[BFS_T / 32 - 1];
    for (int t = a; t < z; ++t) {
        const int c = v[t];
        v[t] = base;
        base += c;
    }
    __syncthreads();
    return total;
}

// Narrow levels: one CTA walks level after level until the graph is done, a
// level has more than BFS_MAXF rows or BFS_EMAX column entries, maxlev
// levels were done in this launch, or a level is empty (no progress).  The
// level's (parent, entry) pairs are spread over all threads: the parents'
// column lengths are scanned, every thread takes entries and finds its
// parent by binary search.  deg, key and item are read with ld.global.cg:
// other threads of this CTA changed them through L2 (atomics,
// st.global.cg) since the last barrier.
__global__ void __launch_bounds__(BFS_T) k_bfs_small(const int *__restrict__ cp, const int *__restrict__ ri, int n,
                                                   int *deg, int *key, int *item, int *lptr, int *meta, int maxlev) {
    extern __shared__ int bfs_sm[];
    int *cst = bfs_sm;                  // [BFS_MAXF + 1] column starts of the level's parents
    int *ent = cst + BFS_MAXF + 1;      // [BFS_EMAX] row of each entry (-1: diagonal / not a child)
    int *pos = ent + BFS_EMAX;          // [BFS_EMAX] child flags, then their scan
    __shared__ int wsum[BFS_T / 32];
    const int tid = threadIdx.x;
    int nl = meta[0];
    int lo = lptr[nl - 1], hi = lptr[nl];
    int status = 0, done_here = 0;
    for (;;) {
        if (hi >= n) { status = BFS_DONE; break; }
        const int f = hi - lo;
        if (f == 0) { status = BFS_STUCK; break; }
        if (f > BFS_MAXF) { status = BFS_BIG; break; }
        if (done_here >= maxlev) { status = BFS_PAUSED; break; }
        for (int t = tid; t < f; t += BFS_T) {
            const int p = __ldcg(item + lo + t);
            cst[t] = cp[p + 1] - cp[p];
        }
        __syncthreads();
        const int E = block_exclusive_scan(cst, f, wsum);
        if (E > BFS_EMAX) { status = BFS_BIG; break; }
        if (tid == 0) cst[f] = E;
        __syncthreads();
        // expand: every entry decrements its row and raises the row's key
        for (int e = tid; e < E; e += BFS_T) {
            int a = 0, z = f;  // parent t: cst[t] <= e < cst[t+1]
            while (z - a > 1) {
                const int mid = (a + z) >> 1;
                if (cst[mid] <= e) a = mid;
                else z = mid;
            }
            const int p = __ldcg(item + lo + a);
            const int r = ri[cp[p] + (e - cst[a])];
            if (r == p) {
                ent[e] = -1;
                __stcg(deg + p, 0);  // expanded: never a child again
            } else {
                ent[e] = r;
                atomicMax(key + r, lo + a);
                atomicSub(deg + r, 1);
            }
        }
        __syncthreads();
        // an entry is a child link when its row reached deg 1 and its parent
        // is the one with the row's key (the last in serial order)
        for (int e = tid; e < E; e += BFS_T) {
            const int r = ent[e];
            int flag = 0;
            if (r >= 0 && __ldcg(deg + r) == 1) {
                int a = 0, z = f;
                while (z - a > 1) {
                    const int mid = (a + z) >> 1;
                    if (cst[mid] <= e) a = mid;
                    else z = mid;
                }
                flag = __ldcg(key + r) == lo + a;
            }
            pos[e] = flag;
        }
        __syncthreads();
        // children in (parent, column) order = entry order
        for (int e = tid; e < E; e += BFS_T) ent[e] = pos[e] ? ent[e] : -1;
        const int total = block_exclusive_scan(pos, E, wsum);
        for (int e = tid; e < E; e += BFS_T)
            if (ent[e] >= 0) __stcg(item + hi + pos[e], ent[e]);
        __syncthreads();
        lo = hi;
        hi += total;
        ++nl;
        ++done_here;
        if (tid == 0) lptr[nl] = hi;
    }
    if (tid == 0) {
        meta[0] = nl;
        meta[1] = status;
    }
}

// Wide levels: warp per parent.
__global__ void k_bfs_expand(const int *__restrict__ cp, const int *__restrict__ ri, const int *__restrict__ item,
                             int lo, int f, int *deg, int *key) {
    const int lane = threadIdx.x & 31;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < f; t += (gridDim.x * blockDim.x) >> 5) {
        const int p = item[lo + t];
        for (int k = cp[p] + lane; k < cp[p + 1]; k += 32) {
            const int r = ri[k];
            if (r == p) continue;
            atomicMax(key + r, lo + t);
            atomicSub(deg + r, 1);
        }
    }
}
__global__ void k_bfs_retire(const int *__restrict__ item, int lo, int f, int *deg) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < f; t += gridDim.x * blockDim.x) deg[item[lo + t]] = 0;
}
__global__ void k_bfs_count(const int *__restrict__ cp, const int *__restrict__ ri, const int *__restrict__ item,
                            int lo, int f, const int *__restrict__ deg, const int *__restrict__ key, int *cnt) {
    const int lane = threadIdx.x & 31;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < f; t += (gridDim.x * blockDim.x) >> 5) {
        const int p = item[lo + t];
        int c = 0;
        for (int k = cp[p] + lane; k < cp[p + 1]; k += 32) {
            const int r = ri[k];
            c += r != p && deg[r] == 1 && key[r] == lo + t;
        }
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) cnt[t] = c;
    }
}
__global__ void k_bfs_write(const int *__restrict__ cp, const int *__restrict__ ri, int *item, int lo, int hi, int f,
                            const int *__restrict__ deg, const int *__restrict__ key, const int *__restrict__ off) {
    const int lane = threadIdx.x & 31;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < f; t += (gridDim.x * blockDim.x) >> 5) {
        const int p = item[lo + t];
        int o = hi + off[t];
        const int e = cp[p + 1];
        for (int k0 = cp[p]; k0 < e; k0 += 32) {
            const int k = k0 + lane;
            int r = -1;
            bool child = false;
            if (k < e) {
                r = ri[k];
                child = r != p && deg[r] == 1 && key[r] == lo + t;
            }
            const unsigned m = __ballot_sync(0xffffffffu, child);
            if (child) item[o + __popc(m & ((1u << lane) - 1u))] = r;
            o += __popc(m);
        }
    }
}

__global__ void k_labels(const int *__restrict__ item, int n, int fwd, int *label, int *pos) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = item[i];
        label[o] = fwd ? i : n - 1 - i;
        pos[o] = i;
    }
}
// column lengths of a column order: len[j] = length of column src(j)
__global__ void k_collen(const int *__restrict__ cp, const int *__restrict__ item, int n, int reverse, int *len) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int s = item[reverse ? n - 1 - j : j];
        len[j] = cp[s + 1] - cp[s];
    }
}
// copy the columns in the new order, entries in stored order, rows mapped
// through map[]; keys/vals variant writes (mapped row, entry index)
__global__ void k_colcopy(const int *__restrict__ cp, const int *__restrict__ ri, const double *__restrict__ va,
                          const int *__restrict__ item, int n, int reverse, const int *__restrict__ ncp,
                          const int *__restrict__ map, int *nri, double *nva, int *ncol) {
    const int lane = threadIdx.x & 31;
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < n; j += (gridDim.x * blockDim.x) >> 5) {
        const int s = item[reverse ? n - 1 - j : j];
        const int b = cp[s], d = ncp[j];
        for (int k = lane; k < cp[s + 1] - b; k += 32) {
            nri[d + k] = map[ri[b + k]];
            if (nva) nva[d + k] = va[b + k];
            if (ncol) ncol[d + k] = j;
        }
    }
}
__global__ void k_iota(int *v, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = (int)i;
}
__global__ void k_gather_pairs(const int *__restrict__ idx, long long nnz, const int *__restrict__ col,
                               const double *__restrict__ val, int *ocol, double *oval) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nnz; t += (long long)gridDim.x * blockDim.x) {
        const int k = idx[t];
        ocol[t] = col[k];
        oval[t] = val[k];
    }
}
__global__ void k_row_count(const int *__restrict__ rows, long long nnz, int *cnt) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nnz; t += (long long)gridDim.x * blockDim.x)
        atomicAdd(cnt + rows[t], 1);
}

// device buffers of one analysis, stream-ordered on the analysis stream
// from the per-device pool, freed on every path
struct Buf {
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;
    std::vector<void *> ptrs;
    ~Buf() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
    }
    template <typename T>
    cudaError_t get(T *&p, size_t count) {
        void *q = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&q, std::max<size_t>(count, 1) * sizeof(T), pool, st);
        if (e == cudaSuccess) {
            ptrs.push_back(q);
            p = static_cast<T *>(q);
        }
        return e;
    }
};

int bits_for(int n) {
    int b = 1;
    while (b < 31 && (1LL << b) < (long long)n) ++b;
    return b;
}

// stable sort of (key, value) pairs by key (values: entry indices)
int sort_pairs(Buf &buf, const int *keys_in, int *keys_out, const int *vals_in, int *vals_out, long long count,
               int nbits, cudaStream_t st, std::string &err) {
    size_t tmp = 0;
    DCK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys_in, keys_out, vals_in, vals_out, (int)count, 0, nbits, st));
    void *t = nullptr;
    DCK(buf.get(reinterpret_cast<char *&>(t), tmp));
    DCK(cub::DeviceRadixSort::SortPairs(t, tmp, keys_in, keys_out, vals_in, vals_out, (int)count, 0, nbits, st));
    return RBS_OK;
}
int exclusive_sum(Buf &buf, const int *in, int *out, long long count, cudaStream_t st, std::string &err) {
    size_t tmp = 0;
    DCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, (int)count, st));
    void *t = nullptr;
    DCK(buf.get(reinterpret_cast<char *&>(t), tmp));
    DCK(cub::DeviceScan::ExclusiveSum(t, tmp, in, out, (int)count, st));
    return RBS_OK;
}

}  // namespace

// Validation, findlevel, reordering and the processing-order CSR on the
// device; results land in the plan's host arrays (in_*, bfs_*, nlevel,
// label, perm, full_*, dev_reorder_*) for the host layout step.
// Device-to-host copies of the results into pageable host vectors, through
// two pinned staging buffers: a chunk's transfer (DMA into pinned memory)
// overlaps the host threads' copy of the previous chunk into the vector.  A
// plain copy into pageable memory moved the 4M-row factor's 1.2 GB of
// results at about 4 GB/s (300 ms).  The staging buffers (2 x 32 MB of
// pinned, portable host memory) are allocated by the first large copy and
// kept for the life of the process (pinning them costs tens of
// milliseconds, more than a small analysis); concurrent analyses take turns.
class HostCopy {
  public:
    explicit HostCopy(cudaStream_t st) : st_(st) {}
    ~HostCopy() {
        for (int i = 0; i < 2; ++i)
            if (ev_[i]) cudaEventDestroy(ev_[i]);
    }
    // dst <- src (bytes); small copies go straight to pageable memory
    cudaError_t copy(void *dst, const void *src, size_t bytes) {
        if (bytes < kMin) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st_);
        cudaError_t e;
        for (int i = 0; i < 2; ++i)
            if (!ev_[i] && (e = cudaEventCreateWithFlags(&ev_[i], cudaEventDisableTiming)) != cudaSuccess) return e;
        std::lock_guard<std::mutex> lock(pool().mu);
        char **stage = pool().stage;
        for (int i = 0; i < 2; ++i)
            if (!stage[i] && (e = cudaHostAlloc(reinterpret_cast<void **>(&stage[i]), kChunk,
                                                cudaHostAllocPortable)) != cudaSuccess)
                return e;
        const size_t nch = (bytes + kChunk - 1) / kChunk;
        auto host_part = [&](size_t c) {  // chunk c from its staging buffer into dst
            const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
            char *d = static_cast<char *>(dst) + off;
            const char *s = stage[c % 2];
            const size_t piece = (len + 15) / 16;
            parallel_for(16, [&](size_t q) {
                const size_t a = q * piece, b = std::min(len, a + piece);
                if (a < b) std::memcpy(d + a, s + a, b - a);
            });
        };
        for (size_t c = 0; c < nch; ++c) {
            const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
            if ((e = cudaMemcpyAsync(stage[c % 2], static_cast<const char *>(src) + off, len, cudaMemcpyDeviceToHost,
                                     st_)) != cudaSuccess)
                return e;
            if ((e = cudaEventRecord(ev_[c % 2], st_)) != cudaSuccess) return e;
            if (c > 0) {  // the previous chunk has landed: copy it out while this one moves
                if ((e = cudaEventSynchronize(ev_[(c - 1) % 2])) != cudaSuccess) return e;
                host_part(c - 1);
            }
        }
        if ((e = cudaEventSynchronize(ev_[(nch - 1) % 2])) != cudaSuccess) return e;
        host_part(nch - 1);
        return cudaSuccess;
    }

  private:
    static constexpr size_t kChunk = size_t(32) << 20, kMin = size_t(8) << 20;
    struct Pool {
        std::mutex mu;
        char *stage[2] = {nullptr, nullptr};
    };
    static Pool &pool() {
        static Pool p;
        return p;
    }
    cudaStream_t st_;
    cudaEvent_t ev_[2] = {nullptr, nullptr};
};

int device_analyse(Plan &P, const int *d_ptr, const int *d_idx, const double *d_val, int n, int nnz, int fmt,
                   int substitution, std::string &err, DevRows *keep) {
    cudaStream_t st = nullptr;
    DCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    Buf buf;
    buf.st = st;
    {
        int dev = 0;
        DCK(cudaGetDevice(&dev));
        DCK(device_mem_pool(dev, buf.pool));
    }
    const int fwd = substitution == RBS_FORWARD;
    const int TPB = 256;
    // 1. CSC input (a CSR input is transposed: stable sort of its entries by
    //    column, so each column lists its rows ascending, tranpose.h:7-54)
    const int *cp = d_ptr, *ri = d_idx;
    const double *va = d_val;
    {
        int h[2];
        DCK(cudaMemcpyAsync(&h[0], d_ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
        DCK(cudaMemcpyAsync(&h[1], d_ptr + n, sizeof(int), cudaMemcpyDeviceToHost, st));
        DCK(cudaStreamSynchronize(st));
        if (h[0] != 0 || h[1] != nnz) {
            err = "rbs_analyse: pointer array must start at 0 and end at nnz";
            return RBS_ERR_STRUCTURE;
        }
    }
    if (fmt == RBS_FMT_CSR) {
        // the row pointer must be valid and every column in range before the
        // indices are used as sort keys and histogram bins
        unsigned long long *bad;
        DCK(buf.get(bad, 1));
        DCK(cudaMemsetAsync(bad, 0xff, sizeof(unsigned long long), st));
        k_check_csr<<<grid_of(n, TPB), TPB, 0, st>>>(d_ptr, d_idx, n, nnz, bad);
        unsigned long long hb = 0;
        DCK(cudaMemcpyAsync(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, st));
        DCK(cudaStreamSynchronize(st));
        if (hb != ~0ull) {
            err = "rbs_analyse: row " + std::to_string((int)(hb >> 8)) +
                  ((hb & 0xff) == VAL_PTR ? ": pointer array decreases" : ": column index out of range");
            return RBS_ERR_STRUCTURE;
        }
        int *rows, *cols_sorted, *idx, *idx_sorted, *ncp, *nri, *cnt;
        double *nva;
        DCK(buf.get(rows, (size_t)nnz));
        DCK(buf.get(cols_sorted, (size_t)nnz));
        DCK(buf.get(idx, (size_t)nnz));
        DCK(buf.get(idx_sorted, (size_t)nnz));
        DCK(buf.get(ncp, (size_t)n + 1));
        DCK(buf.get(nri, (size_t)nnz));
        DCK(buf.get(nva, (size_t)nnz));
        DCK(buf.get(cnt, (size_t)n + 1));
        k_entry_rows<<<grid_of((long long)n * 32, TPB), TPB, 0, st>>>(d_ptr, n, rows);
        k_iota<<<grid_of(nnz, TPB), TPB, 0, st>>>(idx, nnz);
        int rc;
        // stable by column: inside a column the rows ascend (entries are row-major)
        if ((rc = sort_pairs(buf, d_idx, cols_sorted, idx, idx_sorted, nnz, bits_for(n), st, err))) return rc;
        DCK(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)n + 1), st));
        k_row_count<<<grid_of(nnz, TPB), TPB, 0, st>>>(cols_sorted, nnz, cnt);
        if ((rc = exclusive_sum(buf, cnt, ncp, (long long)n + 1, st, err))) return rc;
        k_gather_pairs<<<grid_of(nnz, TPB), TPB, 0, st>>>(idx_sorted, nnz, rows, d_val, nri, nva);
        cp = ncp;
        ri = nri;
        va = nva;
    }
    // 2. validation (first failing column, in the host's wording)
    {
        unsigned long long *bad;
        DCK(buf.get(bad, 1));
        DCK(cudaMemsetAsync(bad, 0xff, sizeof(unsigned long long), st));
        k_validate<<<grid_of(n, TPB), TPB, 0, st>>>(cp, ri, va, n, nnz, fwd, bad);
        unsigned long long hb = 0;
        DCK(cudaMemcpyAsync(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, st));
        DCK(cudaStreamSynchronize(st));
        if (hb != ~0ull) {
            const int c = (int)(hb >> 8), code = (int)(hb & 0xff);
            const std::string col = std::to_string(c);
            switch (code) {
            case VAL_PTR: err = "rbs_analyse: pointer array decreases at " + col; break;
            case VAL_NODIAG: err = "rbs_analyse: column " + col + " has no diagonal"; break;
            case VAL_DIAGPOS:
                err = "rbs_analyse: diagonal of column " + col + " missing or not " + (fwd ? "first" : "last");
                break;
            case VAL_ZERODIAG: err = "rbs_analyse: zero diagonal in column " + col; break;
            case VAL_OUTSIDE:
                err = "rbs_analyse: an entry of column " + col + " lies outside the " + (fwd ? "lower" : "upper") +
                      " triangle";
                break;
            case VAL_DUPDIAG: err = "rbs_analyse: duplicate diagonal in column " + col; break;
            default: err = "rbs_analyse: index out of range in column " + col; break;
            }
            return RBS_ERR_STRUCTURE;
        }
    }
    // 3. findlevel
    int *deg, *key, *item, *lptr, *meta, *cnt, *off;
    DCK(buf.get(deg, (size_t)n));
    DCK(buf.get(key, (size_t)n));
    DCK(buf.get(item, (size_t)n));
    DCK(buf.get(lptr, (size_t)n + 1));
    DCK(buf.get(meta, 4));
    DCK(buf.get(cnt, (size_t)n));
    DCK(buf.get(off, (size_t)n));
    DCK(cudaMemsetAsync(deg, 0, sizeof(int) * (size_t)n, st));
    DCK(cudaMemsetAsync(key, 0xff, sizeof(int) * (size_t)n, st));
    k_degree<<<grid_of(nnz, TPB), TPB, 0, st>>>(ri, nnz, deg);
    {
        // level 0: rows whose only entry is the diagonal, ascending
        int *flag, *rpos;
        DCK(buf.get(flag, (size_t)n));
        DCK(buf.get(rpos, (size_t)n));
        k_root_flags<<<grid_of(n, TPB), TPB, 0, st>>>(deg, n, flag);
        int rc0;
        if ((rc0 = exclusive_sum(buf, flag, rpos, n, st, err))) return rc0;
        k_root_scatter<<<grid_of(n, TPB), TPB, 0, st>>>(flag, rpos, n, item);
        int h[2] = {0, 0}, tl[2];
        DCK(cudaMemcpyAsync(tl, rpos + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        DCK(cudaMemcpyAsync(tl + 1, flag + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        DCK(cudaStreamSynchronize(st));
        h[1] = tl[0] + tl[1];
        DCK(cudaMemcpyAsync(lptr, h, sizeof(int) * 2, cudaMemcpyHostToDevice, st));
        int m0[2] = {1, 0};
        DCK(cudaMemcpyAsync(meta, m0, sizeof(int) * 2, cudaMemcpyHostToDevice, st));
        DCK(cudaStreamSynchronize(st));
    }
    int nl = 0;
    P.device_bfs = 1;
    DCK(cudaFuncSetAttribute(k_bfs_small, cudaFuncAttributeMaxDynamicSharedMemorySize, BFS_SMEM));
    for (;;) {
        k_bfs_small<<<1, BFS_T, BFS_SMEM, st>>>(cp, ri, n, deg, key, item, lptr, meta, BFS_PAUSE);
        int hm[2];
        DCK(cudaMemcpyAsync(hm, meta, sizeof(hm), cudaMemcpyDeviceToHost, st));
        DCK(cudaStreamSynchronize(st));
        nl = hm[0];
        if (hm[1] == BFS_DONE) break;
        if (hm[1] == BFS_STUCK) {
            err = "rbs_analyse: level search stuck (dependency cycle)";
            return RBS_ERR_STRUCTURE;
        }
        if (hm[1] == BFS_PAUSED) {
            // a chain-like graph (levels of a few rows each) costs a few L2 round
            // trips per level here and far less in the host's serial search:
            // hand the level search to the host (same order, bit for bit)
            int done_rows = 0;
            DCK(cudaMemcpyAsync(&done_rows, lptr + nl, sizeof(int), cudaMemcpyDeviceToHost, st));
            DCK(cudaStreamSynchronize(st));
            if ((long long)done_rows < (long long)BFS_NARROW * nl && n - done_rows > BFS_HOST_ROWS) {
                std::vector<int> hcp((size_t)n + 1), hri((size_t)nnz), hptr, hitem;
                DCK(cudaMemcpyAsync(hcp.data(), cp, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost, st));
                DCK(cudaMemcpyAsync(hri.data(), ri, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost, st));
                DCK(cudaStreamSynchronize(st));
                const int hl = host_bfs_levels(hcp.data(), hri.data(), n, hptr, hitem);
                if (hl < 0) {
                    err = "rbs_analyse: level search stuck (dependency cycle)";
                    return RBS_ERR_STRUCTURE;
                }
                DCK(cudaMemcpyAsync(item, hitem.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st));
                DCK(cudaMemcpyAsync(lptr, hptr.data(), sizeof(int) * ((size_t)hl + 1), cudaMemcpyHostToDevice, st));
                DCK(cudaStreamSynchronize(st));
                nl = hl;
                P.device_bfs = 0;
                break;
            }
            continue;
        }
        // one wide level with grid-wide kernels
        int lh[2];
        DCK(cudaMemcpyAsync(lh, lptr + nl - 1, sizeof(lh), cudaMemcpyDeviceToHost, st));
        DCK(cudaStreamSynchronize(st));
        const int lo = lh[0], hi = lh[1], f = hi - lo;
        const int gw = grid_of((long long)f * 32, TPB);
        k_bfs_expand<<<gw, TPB, 0, st>>>(cp, ri, item, lo, f, deg, key);
        k_bfs_retire<<<grid_of(f, TPB), TPB, 0, st>>>(item, lo, f, deg);
        k_bfs_count<<<gw, TPB, 0, st>>>(cp, ri, item, lo, f, deg, key, cnt);
        int rc;
        if ((rc = exclusive_sum(buf, cnt, off, f, st, err))) return rc;
        k_bfs_write<<<gw, TPB, 0, st>>>(cp, ri, item, lo, hi, f, deg, key, off);
        int tail[2];
        DCK(cudaMemcpyAsync(&tail[0], off + f - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        DCK(cudaMemcpyAsync(&tail[1], cnt + f - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        DCK(cudaStreamSynchronize(st));
        const int nhi = hi + tail[0] + tail[1];
        if (nhi == hi && hi < n) {
            err = "rbs_analyse: level search stuck (dependency cycle)";
            return RBS_ERR_STRUCTURE;
        }
        const int m1[2] = {nl + 1, 0};
        DCK(cudaMemcpyAsync(lptr + nl + 1, &nhi, sizeof(int), cudaMemcpyHostToDevice, st));
        DCK(cudaMemcpyAsync(meta, m1, sizeof(m1), cudaMemcpyHostToDevice, st));
        DCK(cudaStreamSynchronize(st));
        nl += 1;
        if (nhi >= n) break;
    }
    // 4. labels, processing positions, the reference's reordered CSC
    //    (columns in label order, entries in stored order, rows relabelled;
    //    utils_reordering.h:130-187) and the processing-order CSR (stable
    //    sort of the processing-order CSC by row: columns ascend in a row)
    int *label, *pos, *len, *rcp, *rri, *pri, *pcol, *idx, *keys_sorted, *idx_sorted, *fcol, *frp, *rowcnt;
    double *pva, *fval;
    DCK(buf.get(label, (size_t)n));
    DCK(buf.get(pos, (size_t)n));
    DCK(buf.get(len, (size_t)n + 1));
    DCK(buf.get(rcp, (size_t)n + 1));
    DCK(buf.get(rri, (size_t)nnz));
    DCK(buf.get(pri, (size_t)nnz));
    DCK(buf.get(pcol, (size_t)nnz));
    DCK(buf.get(pva, (size_t)nnz));
    DCK(buf.get(idx, (size_t)nnz));
    DCK(buf.get(keys_sorted, (size_t)nnz));
    DCK(buf.get(idx_sorted, (size_t)nnz));
    if (keep) {  // the processing-order CSR outlives this function, owned by *keep
        DCK(cudaStreamCreateWithFlags(&keep->st, cudaStreamNonBlocking));
        keep->pool = buf.pool;
        keep->n = n;
        keep->nnz = nnz;
        void *q;
        DCK(cudaMallocFromPoolAsync(&q, sizeof(int) * std::max<size_t>((size_t)nnz, 1), buf.pool, st));
        keep->fcol = fcol = (int *)q;
        DCK(cudaMallocFromPoolAsync(&q, sizeof(double) * std::max<size_t>((size_t)nnz, 1), buf.pool, st));
        keep->fval = fval = (double *)q;
        DCK(cudaMallocFromPoolAsync(&q, sizeof(int) * ((size_t)n + 1), buf.pool, st));
        keep->frp = frp = (int *)q;
    } else {
        DCK(buf.get(fcol, (size_t)nnz));
        DCK(buf.get(fval, (size_t)nnz));
        DCK(buf.get(frp, (size_t)n + 1));
    }
    DCK(buf.get(rowcnt, (size_t)n + 1));
    k_labels<<<grid_of(n, TPB), TPB, 0, st>>>(item, n, fwd, label, pos);
    int rc;
    // reference order: column j of the new matrix is item[j] (forward) or item[n-1-j] (backward)
    DCK(cudaMemsetAsync(len + n, 0, sizeof(int), st));
    k_collen<<<grid_of(n, TPB), TPB, 0, st>>>(cp, item, n, fwd ? 0 : 1, len);
    if ((rc = exclusive_sum(buf, len, rcp, (long long)n + 1, st, err))) return rc;
    k_colcopy<<<grid_of((long long)n * 32, TPB), TPB, 0, st>>>(cp, ri, va, item, n, fwd ? 0 : 1, rcp, label, rri,
                                                               nullptr, nullptr);
    // processing order: processing column q is item[q] in both directions, rows by position
    k_collen<<<grid_of(n, TPB), TPB, 0, st>>>(cp, item, n, 0, len);
    int *pcp;
    DCK(buf.get(pcp, (size_t)n + 1));
    if ((rc = exclusive_sum(buf, len, pcp, (long long)n + 1, st, err))) return rc;
    k_colcopy<<<grid_of((long long)n * 32, TPB), TPB, 0, st>>>(cp, ri, va, item, n, 0, pcp, pos, pri, pva, pcol);
    k_iota<<<grid_of(nnz, TPB), TPB, 0, st>>>(idx, nnz);
    if ((rc = sort_pairs(buf, pri, keys_sorted, idx, idx_sorted, nnz, bits_for(n), st, err))) return rc;
    k_gather_pairs<<<grid_of(nnz, TPB), TPB, 0, st>>>(idx_sorted, nnz, pcol, pva, fcol, fval);
    DCK(cudaMemsetAsync(rowcnt, 0, sizeof(int) * ((size_t)n + 1), st));
    k_row_count<<<grid_of(nnz, TPB), TPB, 0, st>>>(keys_sorted, nnz, rowcnt);
    if ((rc = exclusive_sum(buf, rowcnt, frp, (long long)n + 1, st, err))) return rc;
    // 5. results to the plan
    P.nlevel = nl;
    P.bfs_item.resize((size_t)n);
    P.bfs_ptr.resize((size_t)nl + 1);
    P.label.resize((size_t)n);
    P.perm.resize((size_t)n);
    P.in_cp.resize((size_t)n + 1);
    P.in_ri.resize((size_t)nnz);
    P.in_va.resize((size_t)nnz);
    P.full_rp.resize((size_t)n + 1);
    P.full_col.resize((size_t)nnz);
    P.full_val.resize((size_t)nnz);
    P.dev_reorder_cp.resize((size_t)n + 1);
    P.dev_reorder_ri.resize((size_t)nnz);
    HostCopy hc(st);
    DCK(hc.copy(P.bfs_item.data(), item, sizeof(int) * (size_t)n));
    DCK(hc.copy(P.bfs_ptr.data(), lptr, sizeof(int) * ((size_t)nl + 1)));
    DCK(hc.copy(P.label.data(), label, sizeof(int) * (size_t)n));
    DCK(hc.copy(P.perm.data(), item, sizeof(int) * (size_t)n));
    DCK(hc.copy(P.in_cp.data(), cp, sizeof(int) * ((size_t)n + 1)));
    DCK(hc.copy(P.in_ri.data(), ri, sizeof(int) * (size_t)nnz));
    DCK(hc.copy(P.in_va.data(), va, sizeof(double) * (size_t)nnz));
    DCK(hc.copy(P.full_rp.data(), frp, sizeof(int) * ((size_t)n + 1)));
    DCK(hc.copy(P.full_col.data(), fcol, sizeof(int) * (size_t)nnz));
    DCK(hc.copy(P.full_val.data(), fval, sizeof(double) * (size_t)nnz));
    DCK(hc.copy(P.dev_reorder_cp.data(), rcp, sizeof(int) * ((size_t)n + 1)));
    DCK(hc.copy(P.dev_reorder_ri.data(), rri, sizeof(int) * (size_t)nnz));
    DCK(cudaStreamSynchronize(st));
    return RBS_OK;
}

}  // namespace rbs
