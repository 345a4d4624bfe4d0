// noalloc.cu -- a triangular solve that allocates no device memory.
//
// Some callers cannot call cudaMalloc/cudaFree on the path where they need a
// solve: a host framework whose caching allocator has already reserved the
// device's free memory (a raw cudaMalloc then fails, and cudaFree would
// synchronise the whole device), or a latency-critical loop whose rules
// forbid allocation after start-up.  rbs_sptrsv_csr_noalloc serves them: the
// caller passes the matrix, b and x; the only scratch the solve needs (a
// ticket counter, a status word and the sentinel-filled x work vector) lives
// in g_noalloc_scratch below, a static device array that every GPU loading
// this library holds until the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "kernels.cuh"
#include "rbs.h"
#include "rbs_internal.h"

namespace rbs {
namespace {

// 32 header doubles (256 bytes: ticket at int 0, status at int 1), then the
// x work vector of RBS_NOALLOC_MAX_ROWS doubles.
constexpr int kHeader = 32;
static __device__ __align__(256) double g_noalloc_scratch[kHeader + RBS_NOALLOC_MAX_ROWS];

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// The sync-free triangle kernel (k_tri_syncfree) on a caller's CSR with the
// diagonal stored inside each row: groups of G lanes own a row, find its
// diagonal among the entries, wait for every other column's x to leave the
// sentinel and publish x once.  Rows are ticketed in topological order
// (ascending for lower, descending for upper).  Columns outside [0, n) or
// on the wrong side of the diagonal, and rows without a diagonal, raise
// status bit 2 instead of being read.
__global__ void __launch_bounds__(256) k_noalloc_syncfree(const int *__restrict__ rp, const int *__restrict__ col,
                                                          const double *__restrict__ val, int n, int backward,
                                                          const double *__restrict__ b, double *xw, int *ticket,
                                                          int *status, int G, long long limit) {
    const int lane = threadIdx.x & 31;
    const int rows_per_warp = 32 / G;
    const int sub = lane / G, sl = lane % G;
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (sub * G));
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(ticket, rows_per_warp);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) return;
        const int t = base + sub;
        const bool active = t < n;
        const int row = backward ? n - 1 - t : t;
        double sum = 0, diag = 0;
        if (active) {
            const int s = rp[row], e = rp[row + 1];
            for (int k = s + sl; k < e; k += G) {
                const int c = col[k];
                if (c == row) {
                    diag += val[k];
                } else if (c < 0 || c >= n || (backward ? c < row : c > row)) {
                    atomicOr(status, 2);
                } else {
                    sum += val[k] * wait_value(xw + c, status, limit);
                }
            }
        }
        for (int off = G >> 1; off > 0; off >>= 1) {
            sum += __shfl_down_sync(gmask, sum, off, G);
            diag += __shfl_down_sync(gmask, diag, off, G);
        }
        if (active && sl == 0) {
            if (diag == 0.0) atomicOr(status, 2);
            st_relaxed(xw + row, finalize((b[row] - sum) / diag));
        }
        __syncwarp();
    }
}

__global__ void k_noalloc_prepare(double *scratch, int n) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < kHeader) scratch[t] = 0.0;  // ticket and status start at zero
    for (long long i = t; i < n; i += (long long)gridDim.x * blockDim.x)
        scratch[kHeader + i] = Sent<double>::value();
}

__global__ void k_noalloc_copy_out(const double *scratch, double *x, int n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        x[i] = scratch[kHeader + i];
}

// Device address of the scratch array for the current device.  The symbol
// name is only a host-side handle; kernels must be given this address.
int scratch_for_current_device(double *&ptr, std::string &err) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        err = std::string("rbs_sptrsv_csr_noalloc: cudaGetDevice: ") + cudaGetErrorString(e);
        return RBS_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        err = "rbs_sptrsv_csr_noalloc: device ordinal out of range";
        return RBS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            err = std::string("rbs_sptrsv_csr_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return RBS_ERR_CUDA;
        }
        g_scratch_addr[dev] = (double *)p;
    }
    ptr = g_scratch_addr[dev];
    return RBS_OK;
}

}  // namespace
}  // namespace rbs

extern "C" int rbs_sptrsv_csr_noalloc(const int *d_rowptr, const int *d_colidx, const double *d_val, int n,
                                      int substitution, const double *d_b, double *d_x, void *stream) {
    using namespace rbs;
    if (!d_rowptr || !d_colidx || !d_val || !d_b || !d_x || n <= 0) {
        set_error("rbs_sptrsv_csr_noalloc: null pointer or n <= 0");
        return RBS_ERR_ARG;
    }
    if (n > RBS_NOALLOC_MAX_ROWS) {
        set_error("rbs_sptrsv_csr_noalloc: n = " + std::to_string(n) + " exceeds the scratch limit of " +
                  std::to_string(RBS_NOALLOC_MAX_ROWS) + " rows; use rbs_analyse + rbs_solve");
        return RBS_ERR_ARG;
    }
    if (substitution != RBS_FORWARD && substitution != RBS_BACKWARD) {
        set_error("rbs_sptrsv_csr_noalloc: substitution must be RBS_FORWARD or RBS_BACKWARD");
        return RBS_ERR_ARG;
    }
    std::string err;
    double *scratch = nullptr;
    int rc = scratch_for_current_device(scratch, err);
    if (rc) {
        set_error(err);
        return rc;
    }
    cudaStream_t st = (cudaStream_t)stream;
    int nnz = 0;
    cudaError_t e = cudaMemcpyAsync(&nnz, d_rowptr + n, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(std::string("rbs_sptrsv_csr_noalloc: ") + cudaGetErrorString(e));
        return RBS_ERR_CUDA;
    }
    const double avg = (double)nnz / n;
    const int G = avg < 3 ? 1 : avg < 6 ? 2 : avg < 12 ? 4 : avg < 24 ? 8 : avg < 48 ? 16 : 32;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_noalloc_syncfree, 256, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const long long warps = ((long long)n * G + 31) / 32;
    const int grid = (int)std::max<long long>(1, std::min<long long>((long long)per_sm * sms, (warps + 7) / 8));
    const int vgrid = (int)std::max<long long>(1, std::min<long long>(((long long)n + 255) / 256, (long long)sms * 16));
    int *ticket = (int *)scratch;
    int *status = ticket + 1;
    k_noalloc_prepare<<<vgrid, 256, 0, st>>>(scratch, n);
    k_noalloc_syncfree<<<grid, 256, 0, st>>>(d_rowptr, d_colidx, d_val, n, substitution == RBS_BACKWARD, d_b,
                                             scratch + kHeader, ticket, status, G, 1LL << 22);
    k_noalloc_copy_out<<<vgrid, 256, 0, st>>>(scratch, d_x, n);
    e = cudaGetLastError();
    int h_status = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(std::string("rbs_sptrsv_csr_noalloc: ") + cudaGetErrorString(e));
        return RBS_ERR_CUDA;
    }
    if (h_status & 2) {
        set_error("rbs_sptrsv_csr_noalloc: column outside the triangle or missing/zero diagonal");
        return RBS_ERR_STRUCTURE;
    }
    if (h_status & RBS_STATUS_TIMEOUT) {
        set_error("rbs_sptrsv_csr_noalloc: a device wait exceeded its poll budget");
        return RBS_ERR_TIMEOUT;
    }
    set_error("");
    return RBS_OK;
}
