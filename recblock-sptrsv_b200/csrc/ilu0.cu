// ilu0.cu -- incomplete LU factorisation with zero fill (ILU(0)) on the
// device: the factor producer for this solver in preconditioned Krylov
// methods (no counterpart in the reference, which takes its factors as
// given).
//
// Row-wise IKJ order restricted to A's pattern: for row i and each k < i in
// the row (ascending), a_ik /= a_kk, then a_ij -= a_ik * a_kj for every j > k
// present in both rows i and k.  Row i needs rows k < i of its lower part to
// be final, so one warp takes one row at a time in ticket order -- rows
// sorted by dependency level (computed on the host from a copy of the
// pattern), so the rows in flight span whole levels; the earliest
// unfinished row always has a warp: no deadlock whatever the grid -- and
// waits, bounded, on each dependency's completion flag (release/acquire).
// Every product and difference is rounded separately (no contraction), and
// a row's updates happen in the serial order, so the factor is bit-identical
// to the serial IKJ algorithm.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "rbs.h"
#include "rbs_internal.h"

namespace rbs {

namespace {

constexpr int ILU_MISSING_DIAG = 2, ILU_UNSORTED = 4, ILU_ZERO_PIVOT = 8;

__device__ __forceinline__ int ld_acquire_int(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_int(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// diagonal position of every row; the row pointer must be valid and the
// columns in range and ascending (checked before any of them is used)
__global__ void k_ilu0_diag(const int *__restrict__ rp, const int *__restrict__ ci, int n, int nnz, int *diag,
                            int *status, int *bad_row) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int d = -1, flag = 0;
        const int b = rp[i], e = rp[i + 1];
        if (b < 0 || e < b || e > nnz) flag |= ILU_UNSORTED;
        else
            for (int p = b; p < e; ++p) {
                if (ci[p] < 0 || ci[p] >= n || (p + 1 < e && ci[p] >= ci[p + 1])) flag |= ILU_UNSORTED;
                if (ci[p] == i) d = p;
            }
        if (d < 0) flag |= ILU_MISSING_DIAG;
        diag[i] = d;
        if (flag) {
            atomicOr(status, flag);
            atomicMin(bad_row, i);
        }
    }
}

__global__ void k_ilu0(const int *__restrict__ rp, const int *__restrict__ ci, const int *__restrict__ diag,
                       const int *__restrict__ order, double *lu, int n, int *ticket, int *done, int *status,
                       int *bad_row, long long limit) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(ticket, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n) return;
        const int i = order[t];
        const int s = rp[i], d = diag[i], e = rp[i + 1];
        for (int p = s; p < d; ++p) {
            const int k = ci[p];
            if (lane == 0) {
                unsigned ns = 32;
                for (long long it = 0; ld_acquire_int(done + k) == 0; ++it) {
                    if (it >= limit) {
                        atomicOr(status, RBS_STATUS_TIMEOUT);
                        break;
                    }
                    if (it > 16) {
                        __nanosleep(ns);
                        if (ns < 1024) ns <<= 1;
                    }
                }
            }
            __syncwarp();
            const double piv = __ldcg(lu + diag[k]);
            const double a = __ddiv_rn(lu[p], piv);
            __syncwarp();
            if (lane == 0) lu[p] = a;
            const int kb = diag[k] + 1, ke = rp[k + 1];
            for (int q = p + 1 + lane; q < e; q += 32) {
                const int j = ci[q];
                int lo = kb, hi = ke;  // first column >= j in row k's upper part
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (ci[mid] < j) lo = mid + 1;
                    else hi = mid;
                }
                if (lo < ke && ci[lo] == j) lu[q] = __dsub_rn(lu[q], __dmul_rn(a, __ldcg(lu + lo)));
            }
            __syncwarp();
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) {
            if (lu[d] == 0.0) {
                atomicOr(status, ILU_ZERO_PIVOT);
                atomicMin(bad_row, i);
            }
            st_release_int(done + i, 1);
        }
    }
}

}  // namespace

int device_ilu0(const int *d_rp, const int *d_ci, const double *d_val, int n, int nnz, double *d_lu,
                const rbs_options &opt, std::string &err) {
    auto ck = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && err.empty()) err = std::string("rbs_ilu0_device: ") + what + ": " + cudaGetErrorString(e);
        return e == cudaSuccess;
    };
    if (opt.device >= 0 && !ck(cudaSetDevice(opt.device), "cudaSetDevice")) return RBS_ERR_CUDA;
    int dev = 0, sms = 148;
    if (!ck(cudaGetDevice(&dev), "cudaGetDevice") ||
        !ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute"))
        return RBS_ERR_CUDA;
    cudaStream_t st = nullptr;
    int *scratch = nullptr;  // diag[n], done[n], ticket, status, bad_row
    int rc = RBS_OK;
    if (!ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream") ||
        !ck(cudaMalloc(&scratch, sizeof(int) * (2 * (size_t)n + 4)), "cudaMalloc"))
        rc = RBS_ERR_CUDA;
    int *diag = scratch, *done = scratch + n, *ticket = scratch + 2 * (size_t)n, *status = ticket + 1,
        *bad = ticket + 2;
    int h[3] = {0, 0, 0};
    if (rc == RBS_OK) {
        const int bad0[3] = {0, 0, 0x7fffffff};
        bool ok = ck(cudaMemsetAsync(done, 0, sizeof(int) * (size_t)n, st), "memset") &&
                  ck(cudaMemcpyAsync(ticket, bad0, sizeof(bad0), cudaMemcpyHostToDevice, st), "memcpy") &&
                  ck(cudaMemcpyAsync(d_lu, d_val, sizeof(double) * (size_t)nnz, cudaMemcpyDeviceToDevice, st), "memcpy");
        if (ok) {
            k_ilu0_diag<<<(n + 255) / 256 < sms * 8 ? (n + 255) / 256 : sms * 8, 256, 0, st>>>(d_rp, d_ci, n, nnz, diag,
                                                                                          status, bad);
            ok = ck(cudaGetLastError(), "launch") &&
                 ck(cudaMemcpyAsync(h, ticket, sizeof(h), cudaMemcpyDeviceToHost, st), "memcpy") &&
                 ck(cudaStreamSynchronize(st), "sync");
        }
        if (!ok) rc = RBS_ERR_CUDA;
        else if (h[1] & (ILU_MISSING_DIAG | ILU_UNSORTED)) {
            err = "rbs_ilu0_device: row " + std::to_string(h[2]) +
                  ((h[1] & ILU_UNSORTED) ? " has columns out of order or out of range" : " has no diagonal");
            rc = RBS_ERR_STRUCTURE;
        }
    }
    // rows in dependency-level order (level of row i = 1 + the largest level
    // of the rows of its lower part; all of them precede i), ascending inside
    // a level: the rows in flight at a time span whole levels, and every
    // dependency of a row has an earlier ticket
    int *order = nullptr;
    if (rc == RBS_OK) {
        std::vector<int> hrp((size_t)n + 1), hci((size_t)nnz), lvl((size_t)n, 0), ord((size_t)n);
        bool ok = ck(cudaMemcpyAsync(hrp.data(), d_rp, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost, st), "memcpy") &&
                  ck(cudaMemcpyAsync(hci.data(), d_ci, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost, st), "memcpy") &&
                  ck(cudaStreamSynchronize(st), "sync");
        if (ok) {
            int nlev = 0;
            for (int i = 0; i < n; ++i) {
                int l = 0;
                for (int p = hrp[(size_t)i]; p < hrp[(size_t)i + 1] && hci[(size_t)p] < i; ++p) l = std::max(l, lvl[(size_t)hci[(size_t)p]] + 1);
                lvl[(size_t)i] = l;
                nlev = std::max(nlev, l + 1);
            }
            std::vector<int> start((size_t)nlev + 1, 0);
            for (int i = 0; i < n; ++i) start[(size_t)lvl[(size_t)i] + 1]++;
            for (int l = 0; l < nlev; ++l) start[(size_t)l + 1] += start[(size_t)l];
            for (int i = 0; i < n; ++i) ord[(size_t)start[(size_t)lvl[(size_t)i]]++] = i;
            ok = ck(cudaMalloc(&order, sizeof(int) * (size_t)n), "cudaMalloc") &&
                 ck(cudaMemcpyAsync(order, ord.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st), "memcpy");
        }
        if (!ok) rc = RBS_ERR_CUDA;
    }
    if (rc == RBS_OK) {
        k_ilu0<<<sms * 4, 256, 0, st>>>(d_rp, d_ci, diag, order, d_lu, n, ticket, done, status, bad, opt.spin_limit);
        if (!ck(cudaGetLastError(), "launch") ||
            !ck(cudaMemcpyAsync(h, ticket, sizeof(h), cudaMemcpyDeviceToHost, st), "memcpy") ||
            !ck(cudaStreamSynchronize(st), "sync"))
            rc = RBS_ERR_CUDA;
        else if (h[1] & RBS_STATUS_TIMEOUT) {
            err = "rbs_ilu0_device: a dependency wait exceeded its poll budget";
            rc = RBS_ERR_TIMEOUT;
        } else if (h[1] & ILU_ZERO_PIVOT) {
            err = "rbs_ilu0_device: zero pivot in row " + std::to_string(h[2]);
            rc = RBS_ERR_STRUCTURE;
        }
    }
    if (order) cudaFree(order);
    if (scratch) cudaFree(scratch);
    if (st) cudaStreamDestroy(st);
    return rc;
}

}  // namespace rbs
