// level_lc.cuh -- single-CTA level-chunk triangle: bulk-copied (TMA) chunk
// records, a gather of the long-settled dependencies a few chunks ahead,
// and a shared-memory window for the recent ones.
//
// A triangle (or every independent segment of one, e.g. the systems of a
// batch) is cut by the host into chunks: consecutive rows of one level, at
// most LC_RMAX rows, with a footprint of at most LC_FMAX bytes.  Rows of a
// chunk are independent, so a CTA solves the chunks in order with one CTA
// barrier between them.  For chunk j the host splits every row's entries
// into
//   old    -- dependencies in chunks < j - LC_D, final when chunk j - LC_D
//             starts; their x values are copied (cp.async) into the chunk's
//             shared-memory record LC_D chunks ahead, off the critical path;
//   recent -- dependencies in chunks j - LC_D .. j - 1, read from the
//             shared-memory window of the last LC_XW rows (slot = virtual row
//             index mod LC_XW; the host keeps the rows of LC_D + 1
//             consecutive chunks within LC_XW so no slot is reused early).
// The static part of a record (row map, row pointers, inverse diagonal,
// columns, values) is one contiguous 16-byte-aligned piece of global memory
// copied by one bulk copy into a shared-memory ring; the host places every
// record in the ring and precomputes the chunk iteration at which its copy
// may be issued (the ring bytes and mbarrier slot it needs are free by
// then), always at least LC_D chunks before it is used.
//
// Record layout (sections 16-byte aligned, element type VT):
//   int hdr[8]: nrows, ne_old, ne_rec, vbase, ring offset of the next chunk (16-byte units)
//   int dest[nrows]          block row of each chunk row
//   int rpo[nrows+1]         old-entry pointer
//   int rpr[nrows+1]         recent-entry pointer
//   VT  inv[nrows]           inverse diagonal
//   int colo[ne_old]         block row of the dependency
//   VT  valo[ne_old]
//   int colr[ne_rec]         window slot of the dependency
//   VT  valr[ne_rec]
//   -- end of the copied part; the ring also reserves --
//   VT  gx[ne_old]           gathered x of the old entries
//   VT  bs[nrows]            gathered right-hand side
#pragma once

#include "lc_layout.h"
#include "level_ca.cuh"
#include "tma.cuh"

namespace rbs {

struct LcSeg {
    const LcChunk *tab;
    int nch;
    int ring0;  // ring offset of chunk 0
};

template <typename VT>
struct LcView {
    const int *dest, *rpo, *rpr, *colo, *colr;
    const VT *inv, *valo, *valr;
    VT *gx, *bs;
    __device__ __forceinline__ LcView(unsigned char *rb, int nrows, int ne_old, int ne_rec) {
        constexpr int vq = 16 / sizeof(VT);  // VTs per 16 bytes
        auto padv = [](int n) { return (n + vq - 1) / vq * vq; };
        int *ip = reinterpret_cast<int *>(rb) + LC_HDR_INTS;
        dest = ip;
        ip += lc_pad4(nrows);
        rpo = ip;
        ip += lc_pad4(nrows + 1);
        rpr = ip;
        ip += lc_pad4(nrows + 1);
        VT *vp = reinterpret_cast<VT *>(ip);
        inv = vp;
        vp += padv(nrows);
        ip = reinterpret_cast<int *>(vp);
        colo = ip;
        ip += lc_pad4(ne_old);
        vp = reinterpret_cast<VT *>(ip);
        valo = vp;
        vp += padv(ne_old);
        ip = reinterpret_cast<int *>(vp);
        colr = ip;
        ip += lc_pad4(ne_rec);
        vp = reinterpret_cast<VT *>(ip);
        valr = vp;
        vp += padv(ne_rec);
        gx = vp;
        vp += padv(ne_old);
        bs = vp;
    }
};

__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity, long long limit) {
    for (long long it = 0;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it >= limit) return false;
    }
}
__device__ __forceinline__ void mbar_inval(unsigned long long *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One CTA per segment at a time; CTAs take segments from `queue` (reset to
// 0 before the launch) in the order the host listed them (largest first).
template <typename VT>
__global__ void __launch_bounds__(LC_T, 1)
    k_tri_lc(const LcSeg *__restrict__ segs, int nseg, const unsigned char *__restrict__ rec, int layout32,
             const VT *__restrict__ b, VT *__restrict__ x, int *queue, int *status, long long limit) {
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char *ring = sm;
    VT *xs = reinterpret_cast<VT *>(sm + LC_RING);
    unsigned long long *mbar = reinterpret_cast<unsigned long long *>(sm + LC_RING + LC_XW * sizeof(VT));
    __shared__ int s_seg;
    const int tid = threadIdx.x;
    bool inited = false;
    for (;;) {
        __syncthreads();  // the previous segment is finished by every thread
        if (tid == 0) {
            s_seg = atomicAdd(queue, 1);
            if (s_seg < nseg) {
                for (int i = 0; i < LC_NB; ++i) {
                    if (inited) mbar_inval(mbar + i);
                    mbar_init(mbar + i, 1);
                }
                fence_mbar_init();
            }
        }
        __syncthreads();
        const int sg = s_seg;
        if (sg >= nseg) break;
        inited = true;
        const LcSeg sd = segs[sg];
        const int nch = sd.nch;
        const LcChunk *tab = sd.tab;

        // producer (thread 0): issue every chunk whose issue iteration has come
        int nxt = 0;
        LcChunk ck{};
        if (tid == 0 && nch > 0) ck = tab[0];
        auto issue = [&](int it) {
            while (nxt < nch && ck.issue <= it) {
                const int src = layout32 ? ck.src32 : ck.src64;
                const unsigned by = (unsigned)(layout32 ? ck.bytes32 : ck.bytes64) * 16u;
                unsigned long long *mb = mbar + (nxt % LC_NB);
                mbar_arrive_expect_tx(mb, by);
                bulk_g2s(ring + (size_t)ck.ring * 16, rec + (size_t)src * 16, by, mb);
                if (++nxt < nch) ck = tab[nxt];
            }
        };
        int waited = 0;  // chunks whose copy this thread has seen land
        // wait for chunk j's record, then copy the x of its old entries and
        // its right-hand side into the record (thread-per-row, the mapping
        // the compute step uses, so each thread reads only its own copies)
        auto gather = [&](int j, int rj, int &rnext) -> bool {
            if (!mbar_wait_bounded(mbar + (j % LC_NB), (unsigned)((j / LC_NB) & 1), limit)) return false;
            waited = j + 1;
            unsigned char *rb = ring + (size_t)rj * 16;
            const int4 h = *reinterpret_cast<const int4 *>(rb);
            rnext = reinterpret_cast<const int *>(rb)[4];
            LcView<VT> v(rb, h.x, h.y, h.z);
            for (int r = tid; r < h.x; r += LC_T) {
                const int s0 = v.rpo[r], s1 = v.rpo[r + 1];
                for (int e = s0; e < s1; ++e) cp_async_v<VT>(v.gx + e, x + v.colo[e]);
                cp_async_v<VT>(v.bs + r, b + v.dest[r]);
            }
            return true;
        };

        bool abort = false;
        int roff[LC_D + 1];
        if (tid == 0) issue(0);
        int rcur = sd.ring0;
#pragma unroll
        for (int j = 0; j < LC_D; ++j) {
            roff[j] = rcur;
            if (j < nch && !abort) {
                int rn = 0;
                if (gather(j, rcur, rn)) rcur = rn;
                else abort = true;
            }
            cp_async_commit();
        }
        roff[LC_D] = rcur;
#pragma unroll 1
        for (int c = 0; c < nch; ++c) {
            if (tid == 0) issue(c);
            const int j = c + LC_D;
            int rn = 0;
            if (j < nch && !abort && !gather(j, roff[LC_D], rn)) abort = true;
            cp_async_commit();
            cp_async_wait<LC_D>();  // this thread's copies for chunk c have landed
            if (!abort) {
                unsigned char *rb = ring + (size_t)roff[0] * 16;
                const int4 h = *reinterpret_cast<const int4 *>(rb);
                LcView<VT> v(rb, h.x, h.y, h.z);
                for (int r = tid; r < h.x; r += LC_T) {
                    VT sum = 0;
                    const int o0 = v.rpo[r], o1 = v.rpo[r + 1];
                    for (int e = o0; e < o1; ++e) sum += v.valo[e] * v.gx[e];
                    const int q0 = v.rpr[r], q1 = v.rpr[r + 1];
                    for (int e = q0; e < q1; ++e) sum += v.valr[e] * xs[v.colr[e]];
                    const VT xv = finalize((v.bs[r] - sum) * v.inv[r]);
                    xs[(h.w + r) & (LC_XW - 1)] = xv;
                    x[v.dest[r]] = xv;
                }
            }
#pragma unroll
            for (int q = 0; q < LC_D; ++q) roff[q] = roff[q + 1];
            roff[LC_D] = rn;
            if (__syncthreads_or(abort)) {
                abort = true;
                break;
            }
        }
        cp_async_wait<0>();
        if (abort) {
            // drain: every copy issued must land before the CTA exits
            if (tid == 0) {
                atomicOr(status, RBS_STATUS_TIMEOUT);
                for (int j = waited; j < nxt; ++j)
                    mbar_wait_bounded(mbar + (j % LC_NB), (unsigned)((j / LC_NB) & 1), limit);
            }
            __syncthreads();
            return;
        }
    }
}

}  // namespace rbs
