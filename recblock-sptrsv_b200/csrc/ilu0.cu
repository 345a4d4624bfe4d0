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
//
// IC(0) (incomplete Cholesky, zero fill) of an SPD matrix given as its lower
// triangle uses the same scheme: row i computes l_ik = (a_ik - sum_{j<k}
// l_ij l_kj) / l_kk for its columns k in ascending order, the products over
// the columns it shares with row k found by the lanes (binary search) and
// subtracted in ascending column order through warp shuffles, then
// l_ii = sqrt(a_ii - sum_j l_ij^2) -- the serial row algorithm bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "rbs.h"
#include "rbs_internal.h"

namespace rbs {

namespace {

constexpr int ILU_MISSING_DIAG = 2, ILU_UNSORTED = 4, ILU_ZERO_PIVOT = 8, IC_NOT_LOWER = 16, IC_NOT_POSITIVE = 32;
constexpr unsigned FULL = 0xffffffffu;

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

// IC(0) input: every row ends with its diagonal, columns strictly
// ascending before it (so all of them are below the diagonal)
__global__ void k_ic0_check(const int *__restrict__ rp, const int *__restrict__ ci, int n, int nnz, int *diag,
                            int *status, int *bad_row) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int flag = 0;
        const int b = rp[i], e = rp[i + 1];
        if (b < 0 || e <= b || e > nnz) {
            flag |= ILU_UNSORTED;
        } else {
            const int last = ci[e - 1];
            if (last > i) flag |= IC_NOT_LOWER;
            else if (last < i) flag |= ILU_MISSING_DIAG;
            for (int p = b; p + 1 < e; ++p)
                if (ci[p] < 0 || ci[p] >= ci[p + 1]) flag |= ILU_UNSORTED;
        }
        diag[i] = e - 1;
        if (flag) {
            atomicOr(status, flag);
            atomicMin(bad_row, i);
        }
    }
}

__global__ void k_ic0(const int *__restrict__ rp, const int *__restrict__ ci, const int *__restrict__ order,
                      double *l, int n, int *ticket, int *done, int *status, int *bad_row, long long limit) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(ticket, 1);
        t = __shfl_sync(FULL, t, 0);
        if (t >= n) return;
        const int i = order[t];
        const int b = rp[i], d = rp[i + 1] - 1;
        for (int p = b; p < d; ++p) {
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
            const int kb = rp[k], kd = rp[k + 1] - 1;
            double s = l[p];  // a_ik
            for (int base = b; base < p; base += 32) {
                const int q = base + lane;
                double prod = 0.0;
                int hit = 0;
                if (q < p) {
                    const int j = ci[q];
                    int lo = kb, hi = kd;  // column j in row k's strict part
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (ci[mid] < j) lo = mid + 1;
                        else hi = mid;
                    }
                    if (lo < kd && ci[lo] == j) {
                        prod = __dmul_rn(l[q], __ldcg(l + lo));
                        hit = 1;
                    }
                }
                const int cnt = p - base < 32 ? p - base : 32;
                for (int u = 0; u < cnt; ++u) {
                    const double pu = __shfl_sync(FULL, prod, u);
                    if (__shfl_sync(FULL, hit, u)) s = __dsub_rn(s, pu);
                }
            }
            s = __ddiv_rn(s, __ldcg(l + kd));
            __syncwarp();
            if (lane == 0) l[p] = s;
            __syncwarp();
        }
        double s = l[d];  // a_ii
        for (int base = b; base < d; base += 32) {
            const int q = base + lane;
            const double prod = q < d ? __dmul_rn(l[q], l[q]) : 0.0;
            const int cnt = d - base < 32 ? d - base : 32;
            for (int u = 0; u < cnt; ++u) s = __dsub_rn(s, __shfl_sync(FULL, prod, u));
        }
        __syncwarp();
        if (lane == 0) {
            if (s > 0.0) {
                l[d] = __dsqrt_rn(s);
            } else {
                l[d] = s;
                atomicOr(status, IC_NOT_POSITIVE);
                atomicMin(bad_row, i);
            }
            st_release_int(done + i, 1);
        }
    }
}

}  // namespace

// ILU(0) (ic == false) or IC(0) (ic == true) of a device CSR matrix
static int device_factor(bool ic, const int *d_rp, const int *d_ci, const double *d_val, int n, int nnz,
                         double *d_lu, const rbs_options &opt, std::string &err) {
    const char *who = ic ? "rbs_ic0_device" : "rbs_ilu0_device";
    auto ck = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && err.empty()) err = std::string(who) + ": " + what + ": " + cudaGetErrorString(e);
        return e == cudaSuccess;
    };
    if (opt.device >= 0 && !ck(cudaSetDevice(opt.device), "cudaSetDevice")) return RBS_ERR_CUDA;
    int dev = 0, sms = 148;
    if (!ck(cudaGetDevice(&dev), "cudaGetDevice") ||
        !ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute"))
        return RBS_ERR_CUDA;
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;  // the per-device stream-ordered pool (allocations on st)
    int *scratch = nullptr;  // diag[n], done[n], ticket, status, bad_row
    int rc = RBS_OK;
    if (!ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream") ||
        !ck(device_mem_pool(dev, pool), "memory pool") ||
        !ck(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&scratch), sizeof(int) * (2 * (size_t)n + 4), pool, st),
            "cudaMallocFromPoolAsync"))
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
            const int g = (n + 255) / 256 < sms * 8 ? (n + 255) / 256 : sms * 8;
            if (ic) k_ic0_check<<<g, 256, 0, st>>>(d_rp, d_ci, n, nnz, diag, status, bad);
            else k_ilu0_diag<<<g, 256, 0, st>>>(d_rp, d_ci, n, nnz, diag, status, bad);
            ok = ck(cudaGetLastError(), "launch") &&
                 ck(cudaMemcpyAsync(h, ticket, sizeof(h), cudaMemcpyDeviceToHost, st), "memcpy") &&
                 ck(cudaStreamSynchronize(st), "sync");
        }
        if (!ok) rc = RBS_ERR_CUDA;
        else if (h[1] & (ILU_MISSING_DIAG | ILU_UNSORTED | IC_NOT_LOWER)) {
            err = std::string(who) + ": row " + std::to_string(h[2]) +
                  ((h[1] & ILU_UNSORTED)   ? " has columns out of order or out of range"
                   : (h[1] & IC_NOT_LOWER) ? " has entries above the diagonal (IC(0) takes the lower triangle)"
                   : ic                    ? " does not end with its diagonal"
                                           : " has no diagonal");
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
            ok = ck(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&order), sizeof(int) * (size_t)n, pool, st),
                    "cudaMallocFromPoolAsync") &&
                 ck(cudaMemcpyAsync(order, ord.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st), "memcpy");
        }
        if (!ok) rc = RBS_ERR_CUDA;
    }
    if (rc == RBS_OK) {
        if (ic) k_ic0<<<sms * 4, 256, 0, st>>>(d_rp, d_ci, order, d_lu, n, ticket, done, status, bad, opt.spin_limit);
        else k_ilu0<<<sms * 4, 256, 0, st>>>(d_rp, d_ci, diag, order, d_lu, n, ticket, done, status, bad, opt.spin_limit);
        if (!ck(cudaGetLastError(), "launch") ||
            !ck(cudaMemcpyAsync(h, ticket, sizeof(h), cudaMemcpyDeviceToHost, st), "memcpy") ||
            !ck(cudaStreamSynchronize(st), "sync"))
            rc = RBS_ERR_CUDA;
        else if (h[1] & RBS_STATUS_TIMEOUT) {
            err = std::string(who) + ": a dependency wait exceeded its poll budget";
            rc = RBS_ERR_TIMEOUT;
        } else if (h[1] & ILU_ZERO_PIVOT) {
            err = std::string(who) + ": zero pivot in row " + std::to_string(h[2]);
            rc = RBS_ERR_STRUCTURE;
        } else if (h[1] & IC_NOT_POSITIVE) {
            err = std::string(who) + ": pivot <= 0 in row " + std::to_string(h[2]) +
                  " (not positive definite on the pattern)";
            rc = RBS_ERR_STRUCTURE;
        }
    }
    if (order) cudaFreeAsync(order, st);
    if (scratch) cudaFreeAsync(scratch, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    return rc;
}

int device_ilu0(const int *d_rp, const int *d_ci, const double *d_val, int n, int nnz, double *d_lu,
                const rbs_options &opt, std::string &err) {
    return device_factor(false, d_rp, d_ci, d_val, n, nnz, d_lu, opt, err);
}

int device_ic0(const int *d_rp, const int *d_ci, const double *d_val, int n, int nnz, double *d_l,
               const rbs_options &opt, std::string &err) {
    return device_factor(true, d_rp, d_ci, d_val, n, nnz, d_l, opt, err);
}

}  // namespace rbs
