// dev_pools.cu -- block extraction and packing on the device.
//
// The reference extracts every block of the recursive partition and packs
// it on the GPU (store_into_subtrimat_* / store_into_subrecmat_* and
// store_to_recblockdata, utils_cuda.h:484-704, driven block by block by
// recblocking_solver_cuda.h:133-581, with <<<1,1>>> kernels for the
// per-row scans).  Here the same work runs over all blocks at once, from the
// processing-order CSR that the device analysis leaves on the device:
//   counts  one thread per row: the row's entries per block (every row meets
//           its triangle and at most lv squares, and with columns ascending
//           its entries form one run per block, in block order), its inverse
//           diagonal and its reach (row minus first column in the triangle);
//   levels  the triangles' local level sets: one more than the highest level
//           among a row's dependencies inside its triangle, computed by
//           lane groups that take rows in processing order from a ticket and
//           wait (bounded) for their dependencies' levels, so every row a
//           group waits on is owned by a group already running;
//   fill    one thread per row again: each run of entries goes to its
//           block's pool at the offset of (block, row) in a scan of the
//           counts -- pools block after block, rows in order, columns
//           ascending, exactly the host's layout.
// The host keeps what is O(rows): per-block statistics, the method codes and
// kernel choice, row pointers and row lists, and this library's
// kernel-specific layouts.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <string>
#include <vector>

#include "kernels.cuh"
#include "rbs_internal.h"

namespace rbs {

#define PCK(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            err = std::string("device pools: ") + #call + ": " + cudaGetErrorString(e_); \
            return RBS_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

DevRows::~DevRows() {
    if (st) {
        for (void *p : {(void *)frp, (void *)fcol, (void *)fval, (void *)rowcnt, (void *)slot_base, (void *)status})
            if (p) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
}

namespace {

__device__ __forceinline__ int square_of(int i, int j) {  // the square between triangles j < i
    const int h = 31 - __clz(i ^ j);
    const int t = i & ~((1 << h) - 1);
    return 2 * t - 1;
}

__global__ void k_block_counts(const int *__restrict__ frp, const int *__restrict__ fcol,
                               const double *__restrict__ fval, int n, int T, int s,
                               const long long *__restrict__ slot_base, int *__restrict__ rowcnt,
                               double *__restrict__ inv, int *__restrict__ reach) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int i = min(p / s, T - 1), r0 = i * s;
        int ct = 0, minq = p, cur = -1, cc = 0;
        for (int k = frp[p]; k < frp[p + 1]; ++k) {
            const int q = fcol[k];
            if (q == p) {
                inv[p] = 1.0 / fval[k];
                continue;
            }
            if (q >= r0) {
                ++ct;
                minq = min(minq, q);
                continue;
            }
            const int sb = square_of(i, min(q / s, T - 1));
            if (sb != cur) {
                if (cur >= 0) rowcnt[slot_base[cur] + p - (cur + 1) / 2 * s] = cc;
                cur = sb;
                cc = 0;
            }
            ++cc;
        }
        if (cur >= 0) rowcnt[slot_base[cur] + p - (cur + 1) / 2 * s] = cc;
        rowcnt[slot_base[2 * i] + p - r0] = ct;
        reach[p] = p - minq;
    }
}

__device__ __forceinline__ int ld_relaxed_i32(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_i32(int *p, int v) {
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Local levels (level[] starts at -1): groups of G lanes own a row each.
template <int G>
__global__ void __launch_bounds__(256) k_local_levels(const int *__restrict__ frp, const int *__restrict__ fcol,
                                                      int n, int T, int s, int *level, int *ticket, int *status,
                                                      long long limit) {
    const int lane = threadIdx.x & 31, sub = lane / G, sl = lane % G;
    constexpr int RPW = 32 / G;
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (sub * G));
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(ticket, RPW);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) return;
        const int p = base + sub;
        int mx = -1;
        if (p < n) {
            const int r0 = min(p / s, T - 1) * s;
            for (int k = frp[p] + sl; k < frp[p + 1]; k += G) {
                const int q = fcol[k];
                if (q == p || q < r0) continue;
                int v = ld_relaxed_i32(level + q);
                for (long long it = 0; v < 0; ++it) {
                    if (it >= limit) {
                        atomicOr(status, RBS_STATUS_TIMEOUT);
                        v = 0;
                        break;
                    }
                    if (it > 16) __nanosleep(64);
                    v = ld_relaxed_i32(level + q);
                }
                mx = max(mx, v);
            }
        }
        for (int off = G >> 1; off > 0; off >>= 1) mx = max(mx, __shfl_down_sync(gmask, mx, off, G));
        if (p < n && sl == 0) st_relaxed_i32(level + p, mx + 1);
        __syncwarp();
    }
}

__global__ void k_pool_fill(const int *__restrict__ frp, const int *__restrict__ fcol, const double *__restrict__ fval,
                            int n, int T, int s, const long long *__restrict__ slot_base,
                            const int *__restrict__ rowstart, int *__restrict__ col_pool,
                            double *__restrict__ val_pool) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int i = min(p / s, T - 1), r0 = i * s;
        int cur = -1, dst = 0;
        for (int k = frp[p]; k < frp[p + 1]; ++k) {
            const int q = fcol[k];
            if (q == p) continue;
            int b, lc, br0;
            if (q >= r0) {
                b = 2 * i;
                lc = q - r0;
                br0 = r0;
            } else {
                b = square_of(i, min(q / s, T - 1));
                const int t = (b + 1) / 2;
                lc = q - (t - (t & -t)) * s;
                br0 = t * s;
            }
            if (b != cur) {
                cur = b;
                dst = rowstart[slot_base[b] + p - br0];
            }
            col_pool[dst] = lc;
            val_pool[dst] = fval[k];
            ++dst;
        }
    }
}

int grid_for_rows(long long n, int dev_sms) { return (int)std::max(1LL, std::min((n + 255) / 256, 16LL * dev_sms)); }

}  // namespace

int dev_block_counts(DevRows &R, int T, int s, const std::vector<long long> &slot_base, std::vector<int> &rowcnt,
                     std::vector<double> &inv_diag, std::vector<int> &reach, std::string &err) {
    const int n = R.n;
    if (!R.st) PCK(cudaStreamCreateWithFlags(&R.st, cudaStreamNonBlocking));
    const long long slots = slot_base.back();
    int dev = 0, sms = 148;
    PCK(cudaGetDevice(&dev));
    PCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    R.sms = sms;
    void *p;
    PCK(cudaMallocFromPoolAsync(&p, sizeof(long long) * slot_base.size(), R.pool, R.st));
    R.slot_base = (long long *)p;
    PCK(cudaMallocFromPoolAsync(&p, sizeof(int) * (size_t)std::max(1LL, slots + 1), R.pool, R.st));
    R.rowcnt = (int *)p;
    PCK(cudaMallocFromPoolAsync(&p, sizeof(int) * 4, R.pool, R.st));
    R.status = (int *)p;
    double *d_inv;
    int *d_reach;
    PCK(cudaMallocFromPoolAsync(&p, sizeof(double) * (size_t)n, R.pool, R.st));
    d_inv = (double *)p;
    PCK(cudaMallocFromPoolAsync(&p, sizeof(int) * (size_t)n, R.pool, R.st));
    d_reach = (int *)p;
    PCK(cudaMemcpyAsync(R.slot_base, slot_base.data(), sizeof(long long) * slot_base.size(), cudaMemcpyHostToDevice,
                        R.st));
    PCK(cudaMemsetAsync(R.rowcnt, 0, sizeof(int) * (size_t)(slots + 1), R.st));
    PCK(cudaMemsetAsync(R.status, 0, sizeof(int) * 4, R.st));
    k_block_counts<<<grid_for_rows(n, sms), 256, 0, R.st>>>(R.frp, R.fcol, R.fval, n, T, s, R.slot_base, R.rowcnt,
                                                            d_inv, d_reach);
    PCK(cudaGetLastError());
    rowcnt.resize((size_t)slots);
    inv_diag.resize((size_t)n);
    reach.resize((size_t)n);
    PCK(cudaMemcpyAsync(rowcnt.data(), R.rowcnt, sizeof(int) * (size_t)slots, cudaMemcpyDeviceToHost, R.st));
    PCK(cudaMemcpyAsync(inv_diag.data(), d_inv, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, R.st));
    PCK(cudaMemcpyAsync(reach.data(), d_reach, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, R.st));
    PCK(cudaFreeAsync(d_inv, R.st));
    PCK(cudaFreeAsync(d_reach, R.st));
    PCK(cudaStreamSynchronize(R.st));
    return RBS_OK;
}

int dev_local_levels(DevRows &R, int T, int s, long long spin_limit, std::vector<int> &level, std::string &err) {
    const int n = R.n;
    void *p;
    int *d_level;
    PCK(cudaMallocFromPoolAsync(&p, sizeof(int) * (size_t)n, R.pool, R.st));
    d_level = (int *)p;
    PCK(cudaMemsetAsync(d_level, 0xff, sizeof(int) * (size_t)n, R.st));  // -1: not yet known
    PCK(cudaMemsetAsync(R.status, 0, sizeof(int) * 4, R.st));
    const int avg = (int)((long long)R.nnz / std::max(1, n));
    int per_sm = 1;
    const bool wide = avg >= 12;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wide ? k_local_levels<8> : k_local_levels<4>, 256, 0) !=
            cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int grid = per_sm * R.sms;  // resident groups only: every ticket is held by a running group
    if (wide)
        k_local_levels<8><<<grid, 256, 0, R.st>>>(R.frp, R.fcol, n, T, s, d_level, R.status + 1, R.status, spin_limit);
    else
        k_local_levels<4><<<grid, 256, 0, R.st>>>(R.frp, R.fcol, n, T, s, d_level, R.status + 1, R.status, spin_limit);
    PCK(cudaGetLastError());
    level.resize((size_t)n);
    int st_h = 0;
    PCK(cudaMemcpyAsync(level.data(), d_level, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, R.st));
    PCK(cudaMemcpyAsync(&st_h, R.status, sizeof(int), cudaMemcpyDeviceToHost, R.st));
    PCK(cudaFreeAsync(d_level, R.st));
    PCK(cudaStreamSynchronize(R.st));
    if (st_h & RBS_STATUS_TIMEOUT) {
        err = "device pools: a local-level wait exceeded its poll budget";
        return RBS_ERR_TIMEOUT;
    }
    return RBS_OK;
}

int dev_pool_fill(DevRows &R, int T, int s, long long slots, long long entries, bulk_vector<int> &col_pool,
                  bulk_vector<double> &val_pool, std::string &err) {
    const int n = R.n;
    void *p;
    int *rowstart, *d_col;
    double *d_val;
    PCK(cudaMallocFromPoolAsync(&p, sizeof(int) * (size_t)(slots + 1), R.pool, R.st));
    rowstart = (int *)p;
    size_t tmp = 0;
    PCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, R.rowcnt, rowstart, (int)(slots + 1), R.st));
    void *t;
    PCK(cudaMallocFromPoolAsync(&t, std::max<size_t>(tmp, 1), R.pool, R.st));
    PCK(cub::DeviceScan::ExclusiveSum(t, tmp, R.rowcnt, rowstart, (int)(slots + 1), R.st));
    PCK(cudaMallocFromPoolAsync(&p, sizeof(int) * (size_t)std::max(1LL, entries), R.pool, R.st));
    d_col = (int *)p;
    PCK(cudaMallocFromPoolAsync(&p, sizeof(double) * (size_t)std::max(1LL, entries), R.pool, R.st));
    d_val = (double *)p;
    k_pool_fill<<<grid_for_rows(n, R.sms), 256, 0, R.st>>>(R.frp, R.fcol, R.fval, n, T, s, R.slot_base, rowstart,
                                                            d_col, d_val);
    PCK(cudaGetLastError());
    col_pool.resize((size_t)entries);
    val_pool.resize((size_t)entries);
    if (entries > 0) {
        PCK(cudaMemcpyAsync(col_pool.data(), d_col, sizeof(int) * (size_t)entries, cudaMemcpyDeviceToHost, R.st));
        PCK(cudaMemcpyAsync(val_pool.data(), d_val, sizeof(double) * (size_t)entries, cudaMemcpyDeviceToHost, R.st));
    }
    for (void *q : {(void *)rowstart, t, (void *)d_col, (void *)d_val}) PCK(cudaFreeAsync(q, R.st));
    PCK(cudaStreamSynchronize(R.st));
    return RBS_OK;
}

}  // namespace rbs
