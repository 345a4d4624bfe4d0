// level_lc.cuh -- single-CTA level-chunk triangle: bulk-copied (TMA) chunk
// records, a shared-memory window of the last LC_XW solved rows, and a
// gather of the few dependencies that lie further back.
//
// A triangle (or every independent segment of one, e.g. the systems of a
// batch) is cut by the host into chunks: rows of one level, at most LC_RMAX
// rows and LC_FMAX bytes of ring footprint.  Rows of a chunk are
// independent, so a CTA solves the chunks in order with one CTA barrier
// between them.  Rows are numbered by their position in the segment's chunk
// sequence ("virtual row"); the window keeps x of virtual row v in slot
// v mod LC_XW.  For chunk j the host splits every row's entries into
//   recent -- the dependency is still in the window when chunk j is solved
//             (virtual row >= end of chunk j - LC_XW): read from the window;
//   old    -- further back, so final since before chunk j - LC_D started:
//             its x is copied (cp.async) into the chunk's shared-memory
//             record LC_D chunks ahead, off the critical path.
// Recent entries are stored as jagged columns (rows sorted by their recent
// count, entry k of row t at cs[k] + t), so a warp's loads of one column are
// consecutive words: no bank conflicts.
//
// The copied part of a record is one contiguous 16-byte-aligned piece of
// global memory moved by one bulk copy into a shared-memory ring; the host
// places every record in the ring and precomputes the chunk iteration at
// which its copy may be issued (the ring bytes and mbarrier slot it reuses
// are free by then), always at least LC_D chunks before it is used.  The
// last warp (rows are sorted longest first, so its rows are the shortest)
// issues the copies: lane l holds entry base + l of a 32-entry window of the
// chunk table (the next window is loaded 32 chunks ahead) and issues that
// chunk's copies itself once it is due.
//
// Record layout (sections 16-byte aligned, element type VT):
//   int hdr[8]: nrows, ne_old, ne_rec, vbase, ring offset of the next chunk
//               (16-byte units), jagged columns, longest row, blo (first block
//               row when the rows are contiguous, else -1)
//   int dest[nrows]          block row of each chunk row
//   int rlen[nrows]          recent entries of each row (non-increasing)
//   int rpo[nrows+1]         old-entry pointer
//   int cs[ncols+1]          start of each jagged column
//   VT  inv[nrows]           inverse diagonal
//   int colr[ne_rec]         window slot of the dependency
//   VT  valr[ne_rec]
//   int colo[ne_old]         block row of the dependency
//   VT  valo[ne_old]
//   -- end of the copied part; the ring also reserves --
//   VT  gx[ne_old]           gathered x of the old entries
//   VT  bs[...]              right-hand side: gathered per row (bs[r]), or, when the
//                            chunk's rows are contiguous block rows [blo, blo+nrows),
//                            bulk-copied with the record from the 16-byte boundary
//                            at or below b + blo
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
    const int *dest, *rlen, *rpo, *cs, *colr, *colo;
    const VT *inv, *valr, *valo;
    VT *gx, *bs;
    __device__ __forceinline__ LcView(unsigned char *rb, int nrows, int ne_old, int ne_rec, int ncols) {
        constexpr int vq = 16 / sizeof(VT);  // VTs per 16 bytes
        auto padv = [](int n) { return (n + vq - 1) / vq * vq; };
        int *ip = reinterpret_cast<int *>(rb) + LC_HDR_INTS;
        dest = ip;
        ip += lc_pad4(nrows);
        rlen = ip;
        ip += lc_pad4(nrows);
        rpo = ip;
        ip += lc_pad4(nrows + 1);
        cs = ip;
        ip += lc_pad4(ncols + 1);
        VT *vp = reinterpret_cast<VT *>(ip);
        inv = vp;
        vp += padv(nrows);
        ip = reinterpret_cast<int *>(vp);
        colr = ip;
        ip += lc_pad4(ne_rec);
        vp = reinterpret_cast<VT *>(ip);
        valr = vp;
        vp += padv(ne_rec);
        ip = reinterpret_cast<int *>(vp);
        colo = ip;
        ip += lc_pad4(ne_old);
        vp = reinterpret_cast<VT *>(ip);
        valo = vp;
        vp += padv(ne_old);
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
    __shared__ int s_seg, s_roff[4];
    const int tid = threadIdx.x, lane = tid & 31;
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

        // producer (the last warp, whose rows are the shortest): lane l holds
        // table entries base + l (cur) and base + 32 + l (nxw); copies are
        // issued in chunk order
        int nxt = 0, base = 0;
        LcChunk cur{}, nxw{};
        const LcChunk none{0, 0, 0, 0, 0, 0x7fffffff, -1, 0, 0, 0};
        const bool producer = tid >= LC_T - 32;
        if (producer) {
            cur = lane < nch ? tab[lane] : none;
            nxw = 32 + lane < nch ? tab[32 + lane] : none;
        }
        auto issue = [&](int it) {  // producer warp, converged
            for (;;) {
                if (nxt >= nch) break;
                if (nxt - base >= 32) {
                    base += 32;
                    cur = nxw;
                    nxw = base + 32 + lane < nch ? tab[base + 32 + lane] : none;
                }
                // chunks due now form a run starting at nxt: each lane issues its own
                const bool ready = base + lane >= nxt && cur.issue <= it;
                const unsigned due = __ballot_sync(0xffffffffu, ready);
                if (ready) {
                    const int j = base + lane;
                    unsigned long long *mb = mbar + (j % LC_NB);
                    const int by = (layout32 ? cur.bytes32 : cur.bytes64) * 16;
                    unsigned bb = 0;
                    const void *bsrc = nullptr;
                    if (cur.blo >= 0) {  // contiguous rows: their right-hand side in the same transaction
                        int delta;
                        bb = bulk_window(b + cur.blo, cur.bn, (int)sizeof(VT), bsrc, delta);
                    }
                    mbar_arrive_expect_tx(mb, (unsigned)by + bb);
                    bulk_g2s(ring + (size_t)cur.ring * 16, rec + (size_t)(layout32 ? cur.src32 : cur.src64) * 16,
                             (unsigned)by, mb);
                    if (bb) bulk_g2s(ring + (size_t)(cur.ring + (layout32 ? cur.bs32 : cur.bs64)) * 16, bsrc, bb, mb);
                }
                nxt += __popc(due);
                if (nxt - base < 32) break;  // the run ended inside this window
            }
        };
        int waited = 0;  // chunks whose copy the producer has seen land
        // producer: wait for chunk j's record, then copy the x of its old
        // entries and its right-hand side into the record
        auto gather = [&](int j, int rj, int &rnext) -> bool {
            if (!mbar_wait_bounded(mbar + (j % LC_NB), (unsigned)((j / LC_NB) & 1), limit)) return false;
            waited = j + 1;
            unsigned char *rb = ring + (size_t)rj * 16;
            const int4 h = *reinterpret_cast<const int4 *>(rb);
            const int4 h2 = *reinterpret_cast<const int4 *>(rb + 16);
            rnext = h2.x;
            LcView<VT> v(rb, h.x, h.y, h.z, h2.y);
            const int blo = h2.w;
            if (h.y > 0 || blo < 0)
                for (int r = lane; r < h.x; r += 32) {
                    const int s0 = v.rpo[r], s1 = v.rpo[r + 1];
                    for (int e = s0; e < s1; ++e) cp_async_v<VT>(v.gx + e, x + v.colo[e]);
                    if (blo < 0) cp_async_v<VT>(v.bs + r, b + v.dest[r]);
                }
            return true;
        };

        // The producer runs LC_D chunks ahead: in iteration c it issues the
        // copies due, gathers chunk c + LC_D and waits for its own gathers
        // of chunk c + 1, so after the iteration's barrier every thread may
        // read chunk c + 1's record (ring offset in s_roff).
        bool abort = false;
        int roff[LC_D + 1];
        if (producer) {
            issue(0);
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
            cp_async_wait<LC_D - 1>();  // chunk 0's gathers
            if (lane == 0) s_roff[0] = roff[0];
        }
        if (__syncthreads_or(abort)) abort = true;
#pragma unroll 1
        for (int c = 0; c < nch && !abort; ++c) {
            if (producer) {
                issue(c);
                const int j = c + LC_D;
                int rn = 0;
                if (j < nch && !abort && !gather(j, roff[LC_D], rn)) abort = true;
                cp_async_commit();
                cp_async_wait<LC_D - 1>();  // chunk c + 1's gathers have landed
#pragma unroll
                for (int q = 0; q < LC_D; ++q) roff[q] = roff[q + 1];
                roff[LC_D] = rn;
                if (lane == 0) s_roff[(c + 1) & 3] = roff[0];
            }
            {
                unsigned char *rb = ring + (size_t)s_roff[c & 3] * 16;
                const int4 h = *reinterpret_cast<const int4 *>(rb);
                const int4 h2 = *reinterpret_cast<const int4 *>(rb + 16);
                LcView<VT> v(rb, h.x, h.y, h.z, h2.y);
                const int blo = h2.w;
                // contiguous rows: bs holds b[blo - delta, ...) from a 16-byte boundary
                const int bshift = blo >= 0 ? (int)(((unsigned long long)(b + blo) & 15ull) / sizeof(VT)) - blo : 0;
                for (int r = tid; r < h.x; r += LC_T) {
                    VT sum = 0;
                    const int L = v.rlen[r];
#pragma unroll 4
                    for (int k = 0; k < L; ++k) {
                        const int e = v.cs[k] + r;
                        sum += v.valr[e] * xs[v.colr[e]];
                    }
                    const int o0 = v.rpo[r], o1 = v.rpo[r + 1];
                    for (int e = o0; e < o1; ++e) sum += v.valo[e] * v.gx[e];
                    const int d = v.dest[r];
                    const VT xv = finalize((v.bs[blo >= 0 ? d + bshift : r] - sum) * v.inv[r]);
                    xs[(h.w + r) & (LC_XW - 1)] = xv;
                    x[d] = xv;
                }
            }
            if (__syncthreads_or(abort)) abort = true;
        }
        cp_async_wait<0>();
        if (abort) {
            // drain: every copy issued must land before the CTA exits
            if (tid == LC_T - 32) {  // the producer's lane 0
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
