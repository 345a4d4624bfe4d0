// level_ca.cuh -- single-CTA level-synchronous triangle with per-thread
// asynchronous staging (cp.async) of the row data several levels ahead.
//
// For deep triangles whose levels are narrow (<= 1024 rows) and whose rows
// are short (ELL width <= 4), e.g. grid-like factors in level order.  The
// critical path of a level is: read the dependencies' x from the shared-
// memory window, multiply-add, write x, one CTA barrier.  Everything that
// does not depend on x -- columns, values, inverse diagonal, right-hand side
// -- is copied by each thread for its own row of level l+S-1 with cp.async
// while level l is being solved, into an S-stage shared-memory ring, so it
// is on chip when the level comes up.  A thread only reads what it copied
// itself (cp.async.wait_group), so staging needs no extra synchronisation.
//
// Layout (host-built, per level l): rows [lo_l, lo_l + w_l), ELL width W_l,
// entries column-major at off_l: column of entry j of row lo_l+i at
// col[off_l + j*w_l + i] (padding -1), so a level's loads are coalesced.
// Dependencies within the last XW rows come from the window; older ones
// from x in global memory (written by this CTA before an earlier barrier).
#pragma once

#include "kernels.cuh"

namespace rbs {

constexpr int CA_ROWS = 1024;  // rows per level (= threads)
constexpr int CA_XW = 4096;    // x window (rows)
constexpr int CA_TAB = 6144;   // ints of the level table staged in shared memory (3 per level)

struct CaDesc {
    const int *col;   // level-ELL columns (block-local), padding -1
    const void *val;  // level-ELL values
    const void *inv;  // inverse diagonal of the block's rows
    const void *b;    // right-hand side of the block's rows
    void *x;          // solution of the block's rows
    const int *lvl;   // per level: lo, W, off  (3 ints), plus lo of the end (nlv*3 + 1 ints)
    int m, nlv, pad0, pad1;
};

template <typename VT, int W, int S>
struct CaLayout {
    static constexpr size_t col_bytes = (size_t)W * CA_ROWS * 4;
    static constexpr size_t val_bytes = (size_t)W * CA_ROWS * sizeof(VT);
    static constexpr size_t stage_bytes = col_bytes + val_bytes + 2 * CA_ROWS * sizeof(VT);
    static constexpr size_t xw_off = S * stage_bytes;
    static constexpr size_t tab_off = xw_off + CA_XW * sizeof(VT);
    static constexpr size_t total = tab_off + CA_TAB * 4;
};

__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
template <typename VT>
__device__ __forceinline__ void cp_async_v(VT *dst, const VT *src) {
    if (sizeof(VT) == 8) cp_async8(dst, src);
    else cp_async4(dst, src);
}

template <typename VT, int W, int S>
__global__ void __launch_bounds__(1024) k_tri_level_ca(const CaDesc *__restrict__ descs) {
    using Lay = CaLayout<VT, W, S>;
    extern __shared__ __align__(128) unsigned char sm[];
    const CaDesc d = descs[blockIdx.x];
    const VT *__restrict__ valp = (const VT *)d.val;
    const VT *__restrict__ invp = (const VT *)d.inv;
    const VT *__restrict__ bp = (const VT *)d.b;
    VT *x = (VT *)d.x;
    VT *xs = reinterpret_cast<VT *>(sm + Lay::xw_off);
    int *tab = reinterpret_cast<int *>(sm + Lay::tab_off);
    const int tid = threadIdx.x;
    const int ntab = 3 * d.nlv + 1;
    const bool in_smem = ntab <= CA_TAB;
    if (in_smem)
        for (int i = tid; i < ntab; i += blockDim.x) tab[i] = d.lvl[i];
    __syncthreads();
    const int *lt = in_smem ? tab : d.lvl;

    // stage the row data of level l for this thread (one commit group per level)
    auto stage = [&](int l) {
        if (l < d.nlv) {
            const int lo = lt[3 * l], wl = lt[3 * l + 1], off = lt[3 * l + 2];
            const int w = lt[3 * l + 3] - lo;  // rows of the level
            if (tid < w) {
                unsigned char *st = sm + (size_t)(l % S) * Lay::stage_bytes;
                int *cs = reinterpret_cast<int *>(st);
                VT *vs = reinterpret_cast<VT *>(st + Lay::col_bytes);
                VT *is = reinterpret_cast<VT *>(st + Lay::col_bytes + Lay::val_bytes);
                VT *bs = is + CA_ROWS;
                for (int j = 0; j < wl; ++j) {
                    cp_async4(cs + j * CA_ROWS + tid, d.col + off + (long long)j * w + tid);
                    cp_async_v<VT>(vs + j * CA_ROWS + tid, valp + off + (long long)j * w + tid);
                }
                cp_async_v<VT>(is + tid, invp + lo + tid);
                cp_async_v<VT>(bs + tid, bp + lo + tid);
            }
        }
        cp_async_commit();
    };

#pragma unroll 1
    for (int l = 0; l < S - 1; ++l) stage(l);
#pragma unroll 1
    for (int l = 0; l < d.nlv; ++l) {
        stage(l + S - 1);             // its stage held level l-1, finished at the last barrier
        cp_async_wait<S - 1>();       // this thread's copies of level l have landed
        const int lo = lt[3 * l], wl = lt[3 * l + 1];
        const int hi = lt[3 * l + 3];
        if (tid < hi - lo) {
            const unsigned char *st = sm + (size_t)(l % S) * Lay::stage_bytes;
            const int *cs = reinterpret_cast<const int *>(st);
            const VT *vs = reinterpret_cast<const VT *>(st + Lay::col_bytes);
            const VT *is = reinterpret_cast<const VT *>(st + Lay::col_bytes + Lay::val_bytes);
            const VT *bs = is + CA_ROWS;
            VT sum = 0;
#pragma unroll
            for (int j = 0; j < W; ++j) {
                if (j < wl) {
                    const int c = cs[j * CA_ROWS + tid];
                    if (c >= 0) {
                        const VT xv = c >= hi - CA_XW ? xs[c & (CA_XW - 1)] : x[c];
                        sum += vs[j * CA_ROWS + tid] * xv;
                    }
                }
            }
            const int r = lo + tid;
            const VT xv = finalize((bs[tid] - sum) * is[tid]);
            xs[r & (CA_XW - 1)] = xv;
            x[r] = xv;
        }
        __syncthreads();
    }
    cp_async_wait<0>();
}

}  // namespace rbs
