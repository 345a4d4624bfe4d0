// band.cuh -- parallel affine scan for deep, narrow-band triangles.
//
// Replaces the reference's method 1 (cuSPARSE csrsv2 for blocks with more
// than 20000 levels, recblocking_preprocess.h:518-623) when every row's
// entries lie within W positions of the diagonal.  Such a block is a chain:
// with the state s_p = (x_p, x_{p-1}, ..., x_{p-W+1}), row p is the affine
// map  s_p = M_p s_{p-1} + c_p,  M_p a companion matrix whose first row is
// -a_p / l_pp and whose other rows shift the state.  Maps compose
// associatively, so a chain of m rows is solved in three passes instead of
// m dependent steps:
//   1. k_band_maps   : each thread composes the maps of C consecutive rows;
//   2. k_band_scan   : one CTA scans the chunk maps (sequential per thread,
//                      Kogge-Stone across threads) into each chunk's
//                      entering state;
//   3. k_band_replay : each thread replays its rows from that state.
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

// Several right-hand sides run side by side in one launch of each pass:
// column c = blockIdx.y of the maps and replay passes (blockIdx.x of the
// scan), with its own maps and states at c * nch * (W*W + W) and c * nch * W.
//
// Pass 1: maps[j] = composition of the row maps of chunk j.
template <typename VT, int W>
__global__ void __launch_bounds__(256) k_band_maps(const VT *__restrict__ coef, const VT *__restrict__ inv,
                                                   const VT *__restrict__ b, int K, int m, int C, int nch,
                                                   VT *__restrict__ maps) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int colk = blockIdx.y;
    maps += (long long)colk * nch * (W * W + W);
    if (j >= nch) return;
    VT M[W][W], c[W];
#pragma unroll
    for (int r = 0; r < W; ++r) {
#pragma unroll
        for (int q = 0; q < W; ++q) M[r][q] = r == q ? VT(1) : VT(0);
        c[r] = 0;
    }
    const int rows = min(C, m - j * C);
#pragma unroll 4
    for (int i = 0; i < rows; ++i) {
        const long long o = (long long)i * nch + j;
        VT a[W];
#pragma unroll
        for (int d = 0; d < W; ++d) a[d] = coef[o * W + d];
        const int p = j * C + i;
        band_step_M<VT, W>(M, c, a, inv[o], b[(long long)p * K + colk]);
    }
    VT *out = maps + (long long)j * (W * W + W);
#pragma unroll
    for (int r = 0; r < W; ++r) {
#pragma unroll
        for (int q = 0; q < W; ++q) out[r * W + q] = M[r][q];
        out[W * W + r] = c[r];
    }
}

// (M, c) <- (Mo, co) o (M, c):  M = Mo M,  c = Mo c + co
template <typename VT, int W>
__device__ __forceinline__ void band_compose_after(VT (&M)[W][W], VT (&c)[W], const VT *o) {
    VT nM[W][W], nc[W];
#pragma unroll
    for (int r = 0; r < W; ++r) {
        VT s = o[W * W + r];
#pragma unroll
        for (int k = 0; k < W; ++k) s += o[r * W + k] * c[k];
        nc[r] = s;
#pragma unroll
        for (int q = 0; q < W; ++q) {
            VT t = 0;
#pragma unroll
            for (int k = 0; k < W; ++k) t += o[r * W + k] * M[k][q];
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

// Pass 2: one CTA of 256 threads.  Thread t composes chunks [t*Q, t*Q+Q),
// the CTA scans the per-thread maps, and each thread then walks its chunks
// to write the state entering each of them (the block starts from s = 0).
template <typename VT, int W>
__global__ void __launch_bounds__(256) k_band_scan(const VT *__restrict__ maps, int nch, VT *__restrict__ states) {
    extern __shared__ unsigned char smem_raw[];
    maps += (long long)blockIdx.x * nch * (W * W + W);
    states += (long long)blockIdx.x * nch * W;
    VT *sm = reinterpret_cast<VT *>(smem_raw);
    constexpr int E = W * W + W;
    const int tid = threadIdx.x, T = blockDim.x;
    const int Q = (nch + T - 1) / T;
    const int j0 = min(nch, tid * Q), j1 = min(nch, j0 + Q);
    VT M[W][W], c[W];
#pragma unroll
    for (int r = 0; r < W; ++r) {
#pragma unroll
        for (int q = 0; q < W; ++q) M[r][q] = r == q ? VT(1) : VT(0);
        c[r] = 0;
    }
    for (int j = j0; j < j1; ++j) band_compose_after<VT, W>(M, c, maps + (long long)j * E);
    // inclusive Kogge-Stone over the T per-thread maps
    for (int off = 1; off < T; off <<= 1) {
        VT *mine = sm + (long long)tid * E;
#pragma unroll
        for (int r = 0; r < W; ++r) {
#pragma unroll
            for (int q = 0; q < W; ++q) mine[r * W + q] = M[r][q];
            mine[W * W + r] = c[r];
        }
        __syncthreads();
        if (tid >= off) {
            // this <- this o earlier:  M = M_this M_earlier,  c = M_this c_earlier + c_this
            const VT *e = sm + (long long)(tid - off) * E;
            VT nM[W][W], nc[W];
#pragma unroll
            for (int r = 0; r < W; ++r) {
                VT s = c[r];
#pragma unroll
                for (int k = 0; k < W; ++k) s += M[r][k] * e[W * W + k];
                nc[r] = s;
#pragma unroll
                for (int q = 0; q < W; ++q) {
                    VT t = 0;
#pragma unroll
                    for (int k = 0; k < W; ++k) t += M[r][k] * e[k * W + q];
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
    // state entering this thread's first chunk = exclusive prefix applied to 0
    VT *mine = sm + (long long)tid * E;
#pragma unroll
    for (int r = 0; r < W; ++r) mine[W * W + r] = c[r];
    __syncthreads();
    VT s[W];
#pragma unroll
    for (int r = 0; r < W; ++r) s[r] = tid == 0 ? VT(0) : sm[(long long)(tid - 1) * E + W * W + r];
    for (int j = j0; j < j1; ++j) {
#pragma unroll
        for (int r = 0; r < W; ++r) states[(long long)j * W + r] = s[r];
        const VT *f = maps + (long long)j * E;
        VT ns[W];
#pragma unroll
        for (int r = 0; r < W; ++r) {
            VT t = f[W * W + r];
#pragma unroll
            for (int k = 0; k < W; ++k) t += f[r * W + k] * s[k];
            ns[r] = t;
        }
#pragma unroll
        for (int r = 0; r < W; ++r) s[r] = ns[r];
    }
}

// Pass 3: replay chunk j from its entering state and write x.
template <typename VT, int W>
__global__ void __launch_bounds__(256) k_band_replay(const VT *__restrict__ coef, const VT *__restrict__ inv,
                                                     const VT *__restrict__ b, int K, int m, int C, int nch,
                                                     const VT *__restrict__ states, VT *x) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int colk = blockIdx.y;
    states += (long long)colk * nch * W;
    if (j >= nch) return;
    VT s[W];
#pragma unroll
    for (int r = 0; r < W; ++r) s[r] = states[(long long)j * W + r];
    const int rows = min(C, m - j * C);
#pragma unroll 4
    for (int i = 0; i < rows; ++i) {
        const long long o = (long long)i * nch + j;
        const int p = j * C + i;
        VT acc = 0;
#pragma unroll
        for (int d = 0; d < W; ++d) acc += coef[o * W + d] * s[d];
        const VT xp = inv[o] * (b[(long long)p * K + colk] - acc);
#pragma unroll
        for (int d = W - 1; d > 0; --d) s[d] = s[d - 1];
        s[0] = xp;
        x[(long long)p * K + colk] = finalize(xp);
    }
}

}  // namespace rbs
