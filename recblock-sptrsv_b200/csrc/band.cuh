// band.cuh -- parallel affine scan for deep, narrow-band triangles.
//
// Replaces the reference's method 1 (cuSPARSE csrsv2 for blocks with more
// than 20000 levels, recblocking_preprocess.h:518-623) when every row's
// entries lie within W positions of the diagonal.  Such a block is a chain:
// with the state s_p = (x_p, x_{p-1}, ..., x_{p-W+1}), row p is the affine
// map  s_p = M_p s_{p-1} + c_p,  M_p a companion matrix whose first row is
// -a_p / l_pp and whose other rows shift the state.  Maps compose
// associatively, so a chain of m rows is solved in one launch instead of m
// dependent steps (k_band_onepass): each thread composes the maps of C
// consecutive rows (a chunk); a CTA scans its BAND_T chunk maps in shared
// memory (Kogge-Stone) and publishes their total; the state entering the
// CTA is its predecessors' totals applied in order to the zero state (one
// W x W matrix-vector product each, no scan of maps needed); each thread
// applies the composition of its CTA's earlier chunks to that state and
// replays its rows from there.  CTAs take their place in the chain from a
// ticket, so every predecessor a CTA waits for is already running and
// publishes without waiting on anyone: no deadlock, whatever the residency.
// The first form ran three launches per triangle and scanned the chunk maps
// in one CTA: 122 us of a 155 us triangle on the banded chain, then 31 us in
// three launches once the CTAs scanned their own chunks.
// Band coefficients are stored chunk-interleaved (row i of chunk j at
// [(i*nch + j)*W]) so the threads of a warp read consecutive addresses.
// For diagonally dominant rows every ||M_p||_inf <= 1, so composed maps stay
// bounded and the scan is as stable as substitution.
#pragma once

#include "kernels.cuh"

namespace rbs {

template <typename VT, int W>
__device__ __forceinline__ void band_step_M(VT (&M)[W][W], VT (&c)[W], const VT *a, VT iv, VT bp) {
    VT r[W];
#pragma unroll
    for (int q = 0; q < W; ++q) {
        VT s = 0;
#pragma unroll
        for (int d = 0; d < W; ++d) s += a[d] * M[d][q];
        r[q] = -iv * s;
    }
    VT c0 = 0;
#pragma unroll
    for (int d = 0; d < W; ++d) c0 += a[d] * c[d];
    c0 = iv * (bp - c0);
#pragma unroll
    for (int d = W - 1; d > 0; --d) {
#pragma unroll
        for (int q = 0; q < W; ++q) M[d][q] = M[d - 1][q];
        c[d] = c[d - 1];
    }
#pragma unroll
    for (int q = 0; q < W; ++q) M[0][q] = r[q];
    c[0] = c0;
}

// Chunks per CTA of the maps and replay passes (the CTA-level scan's width).
constexpr int BAND_T = 256;

__host__ __device__ constexpr int band_blocks(int nch) { return (nch + BAND_T - 1) / BAND_T; }

// A thread's (M, c) into, and another thread's out of, shared memory laid
// out element-major (element k of thread t at sm[k * T + t]), so a warp's
// accesses are consecutive words.  Thread-major records (stride W*W+W)
// put 8 threads of a warp on each bank.
template <typename VT, int W>
__device__ __forceinline__ void band_put(VT *sm, int T, int t, const VT (&M)[W][W], const VT (&c)[W]) {
#pragma unroll
    for (int r = 0; r < W; ++r) {
#pragma unroll
        for (int q = 0; q < W; ++q) sm[(r * W + q) * T + t] = M[r][q];
        sm[(W * W + r) * T + t] = c[r];
    }
}
template <typename VT, int W>
__device__ __forceinline__ void band_get(const VT *sm, int T, int t, VT (&M)[W][W], VT (&c)[W]) {
#pragma unroll
    for (int r = 0; r < W; ++r) {
#pragma unroll
        for (int q = 0; q < W; ++q) M[r][q] = sm[(r * W + q) * T + t];
        c[r] = sm[(W * W + r) * T + t];
    }
}

// Inclusive Kogge-Stone scan of one (M, c) per thread over the CTA, through
// sm (blockDim.x * (W*W + W) values): thread t ends with map_t o ... o map_0.
template <typename VT, int W>
__device__ __forceinline__ void band_cta_scan(VT (&M)[W][W], VT (&c)[W], VT *sm) {
    const int tid = threadIdx.x, T = blockDim.x;
    for (int off = 1; off < T; off <<= 1) {
        band_put<VT, W>(sm, T, tid, M, c);
        __syncthreads();
        if (tid >= off) {
            VT Me[W][W], ce[W];
            band_get<VT, W>(sm, T, tid - off, Me, ce);
            // (M, c) <- (M, c) o (Me, ce):  M = M Me,  c = M ce + c
            VT nM[W][W], nc[W];
#pragma unroll
            for (int r = 0; r < W; ++r) {
                VT v = c[r];
#pragma unroll
                for (int k = 0; k < W; ++k) v += M[r][k] * ce[k];
                nc[r] = v;
#pragma unroll
                for (int q = 0; q < W; ++q) {
                    VT t = 0;
#pragma unroll
                    for (int k = 0; k < W; ++k) t += M[r][k] * Me[k][q];
                    nM[r][q] = t;
                }
            }
#pragma unroll
            for (int r = 0; r < W; ++r) {
                c[r] = nc[r];
#pragma unroll
                for (int q = 0; q < W; ++q) M[r][q] = nM[r][q];
            }
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int band_ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void band_st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// One launch per triangle.  Several right-hand sides run side by side:
// column c = blockIdx.y, with its own CTA totals at agg + c * nblk * (W*W+W)
// and its own ticket and ready flags (flags: c * (nblk + 1), the ticket
// first, then one flag per CTA; zeroed before the launch).  Waits are
// bounded: after `limit` polls a CTA raises RBS_STATUS_TIMEOUT and goes on.
template <typename VT, int W>
__global__ void __launch_bounds__(BAND_T) k_band_onepass(const VT *__restrict__ coef, const VT *__restrict__ inv,
                                                         const VT *__restrict__ b, int K, int m, int C, int nch,
                                                         VT *__restrict__ agg, int *flags, VT *x, int *status,
                                                         long long limit) {
    extern __shared__ unsigned char smem_raw[];
    VT *sm = reinterpret_cast<VT *>(smem_raw);
    __shared__ VT s_state[W];
    __shared__ int s_o;
    constexpr int E = W * W + W;
    const int tid = threadIdx.x, colk = blockIdx.y;
    const int nblk = band_blocks(nch);
    agg += (long long)colk * nblk * E;
    flags += (long long)colk * (nblk + 1);
    if (tid == 0) s_o = atomicAdd(flags, 1);  // this CTA's place in the chain
    __syncthreads();
    const int o = s_o;
    const int j = o * BAND_T + tid;
    const int rows = j < nch ? min(C, m - j * C) : 0;

    // 1. the chunk's map, scanned over the CTA's chunks
    VT M[W][W], c[W];
#pragma unroll
    for (int r = 0; r < W; ++r) {
#pragma unroll
        for (int q = 0; q < W; ++q) M[r][q] = r == q ? VT(1) : VT(0);
        c[r] = 0;
    }
#pragma unroll 4
    for (int i = 0; i < rows; ++i) {
        const long long oi = (long long)i * nch + j;
        VT a[W];
#pragma unroll
        for (int d = 0; d < W; ++d) a[d] = coef[oi * W + d];
        band_step_M<VT, W>(M, c, a, inv[oi], b[(long long)(j * C + i) * K + colk]);
    }
    band_cta_scan<VT, W>(M, c, sm);

    // 2. publish the CTA's total (the last thread's inclusive composition)
    if (tid == BAND_T - 1) {
        VT *out = agg + (long long)o * E;
#pragma unroll
        for (int r = 0; r < W; ++r) {
#pragma unroll
            for (int q = 0; q < W; ++q) out[r * W + q] = M[r][q];
            out[W * W + r] = c[r];
        }
        __threadfence();
        band_st_release(flags + 1 + o, 1);
    }
    // the composition of this CTA's chunks before this one (thread tid - 1's)
    band_put<VT, W>(sm, BAND_T, tid, M, c);
    __syncthreads();
    if (tid > 0) band_get<VT, W>(sm, BAND_T, tid - 1, M, c);
    __syncthreads();  // sm is reused below

    // 3. the state entering this CTA: predecessors' totals applied in order
    VT s0[W];
#pragma unroll
    for (int r = 0; r < W; ++r) s0[r] = 0;
    for (int base = 0; base < o; base += BAND_T) {
        const int cnt = min(BAND_T, o - base);
        if (tid < cnt) {
            const int *f = flags + 1 + base + tid;
            for (long long it = 0; band_ld_acquire(f) == 0; ++it) {
                if (it >= limit) {
                    atomicOr(status, RBS_STATUS_TIMEOUT);
                    break;
                }
                if (it > 16) __nanosleep(64);
            }
        }
        __syncthreads();
        for (int i = tid; i < cnt * E; i += BAND_T) sm[i] = __ldcg(agg + (long long)base * E + i);
        __syncthreads();
        if (tid == 0) {
            for (int q = 0; q < cnt; ++q) {
                const VT *t = sm + (long long)q * E;
                VT ns[W];
#pragma unroll
                for (int r = 0; r < W; ++r) {
                    VT v = t[W * W + r];
#pragma unroll
                    for (int k = 0; k < W; ++k) v += t[r * W + k] * s0[k];
                    ns[r] = v;
                }
#pragma unroll
                for (int r = 0; r < W; ++r) s0[r] = ns[r];
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
#pragma unroll
        for (int r = 0; r < W; ++r) s_state[r] = s0[r];
    }
    __syncthreads();

    // 4. the state entering this thread's chunk, then its rows replayed
    VT s[W];
#pragma unroll
    for (int r = 0; r < W; ++r) s0[r] = s_state[r];
    if (tid == 0) {
#pragma unroll
        for (int r = 0; r < W; ++r) s[r] = s0[r];
    } else {
#pragma unroll
        for (int r = 0; r < W; ++r) {
            VT v = c[r];
#pragma unroll
            for (int k = 0; k < W; ++k) v += M[r][k] * s0[k];
            s[r] = v;
        }
    }
#pragma unroll 4
    for (int i = 0; i < rows; ++i) {
        const long long oi = (long long)i * nch + j;
        const int p = j * C + i;
        VT acc = 0;
#pragma unroll
        for (int d = 0; d < W; ++d) acc += coef[oi * W + d] * s[d];
        const VT xp = inv[oi] * (b[(long long)p * K + colk] - acc);
#pragma unroll
        for (int d = W - 1; d > 0; --d) s[d] = s[d - 1];
        s[0] = xp;
        x[(long long)p * K + colk] = finalize(xp);
    }
}

}  // namespace rbs
