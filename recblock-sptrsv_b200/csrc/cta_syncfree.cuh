// cta_syncfree.cuh -- one CTA solves a deep triangle without CTA barriers.
//
// Level-synchronous execution pays a CTA barrier plus the slowest warp's
// whole row on every level.  Here the rows of the triangle are dealt
// round-robin to the CTA's consumer threads in processing (topological)
// order and every dependency is waited on individually, inside the SM:
//   * x of the last XW rows lives in a shared-memory window; each window
//     slot carries the index of the row whose value it holds (-1 while
//     being rewritten).  A writer marks the slot busy, fences, stores x,
//     fences, then publishes its row index; a reader polls the tag until it
//     reaches its column, reads x, and re-reads the tag (seqlock) -- if the
//     slot was recycled meanwhile, or the column is older than the window,
//     x comes from global memory (polled for the NaN sentinel, as in the
//     multi-CTA sync-free kernel);
//   * the block's ELL chunks (<= CSF_RMAX rows, <= CSF_EMAX slots, column
//     indices, padding = column -1) stream through an NS-slot shared-memory
//     ring with 1D bulk copies; a producer warp refills a slot once the
//     per-slot counter says every row of its chunk is finished, waits on the
//     slot's mbarrier in phase order and publishes the landed chunk index;
//   * a thread handles rows t, t+T, t+2T, ... in order; a chunk is loaded
//     before any later chunk and every dependency is an earlier row, so the
//     rows a waiting thread needs are always reachable: no deadlock;
//   * consumers write x only to the window; the producer warp copies each
//     finished chunk to global memory.  The ring holds at most NS chunks of
//     <= RMAX rows (2560 rows) ahead of the oldest unfinished chunk, less
//     than the window (4096 rows), so a slot is never recycled before the
//     row it held is finished and stored.
// All waits are bounded; on expiry the CTA raises the status, stops
// waiting, finishes with NaN, and drains its copies before exiting.
#pragma once

#include "tma.cuh"

namespace rbs {

struct EllChunk {
    int R0, R1, W, off;  // rows [R0,R1) (block-local), ELL width, offset in the ELL pools (elements)
};

constexpr int CSF_RMAX = 512;
constexpr int CSF_EMAX = 2048;
constexpr int CSF_NS = 5;
constexpr int CSF_XW = 4096;
constexpr int CSF_TAB = 2048;  // ints of the chunk table staged in shared memory

struct CsfDesc {
    const int *col;          // ELL columns (block-local), column-major per chunk, -1 = padding
    const void *val;         // ELL values
    const void *inv;         // inverse diagonal of the block's rows
    const void *b;           // right-hand side of the block's rows
    void *x;                 // solution of the block's rows (pre-filled with the sentinel)
    const EllChunk *chunks;  // nchunks entries
    int m, nchunks, G, pad;
};

template <typename VT>
struct CsfLayout {
    static constexpr size_t col_off = 0;
    static constexpr size_t val_off = col_off + ((CSF_EMAX * 4 + 16 + 127) / 128) * 128;
    static constexpr size_t inv_off = val_off + ((CSF_EMAX * sizeof(VT) + 16 + 127) / 128) * 128;
    static constexpr size_t b_off = inv_off + ((CSF_RMAX * sizeof(VT) + 16 + 127) / 128) * 128;
    static constexpr size_t slot_bytes = b_off + ((CSF_RMAX * sizeof(VT) + 16 + 127) / 128) * 128;
    static constexpr size_t xw_off = CSF_NS * slot_bytes;
    static constexpr size_t tag_off = xw_off + ((CSF_XW * sizeof(VT) + 127) / 128) * 128;
    static constexpr size_t bar_off = tag_off + CSF_XW * 4;
    static constexpr size_t hdr_off = bar_off + 128;            // per slot: 4 element deltas
    static constexpr size_t cnt_off = hdr_off + CSF_NS * 16;    // per slot: finished rows
    static constexpr size_t ld_off = cnt_off + 64;               // per slot: chunk index resident (-1 none)
    static constexpr size_t tab_off = ld_off + 64;
    static constexpr size_t total = tab_off + CSF_TAB * 4;
};

__device__ __forceinline__ int lds_volatile(const int *p) {
    int v;
    asm volatile("ld.volatile.shared.s32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}
__device__ __forceinline__ void sts_volatile(int *p, int v) {
    asm volatile("st.volatile.shared.s32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}

template <typename VT>
__global__ void __launch_bounds__(1024) k_tri_cta_syncfree(const CsfDesc *__restrict__ descs, int *status,
                                                           long long limit) {
    using Lay = CsfLayout<VT>;
    extern __shared__ __align__(128) unsigned char sm[];
    const CsfDesc d = descs[blockIdx.x];
    unsigned long long *full = reinterpret_cast<unsigned long long *>(sm + Lay::bar_off);
    int *hdr = reinterpret_cast<int *>(sm + Lay::hdr_off);
    int *cnt = reinterpret_cast<int *>(sm + Lay::cnt_off);
    int *loaded = reinterpret_cast<int *>(sm + Lay::ld_off);
    int *tag = reinterpret_cast<int *>(sm + Lay::tag_off);
    VT *xs = reinterpret_cast<VT *>(sm + Lay::xw_off);
    int *tab = reinterpret_cast<int *>(sm + Lay::tab_off);
    const VT *__restrict__ valp = (const VT *)d.val;
    const VT *__restrict__ invp = (const VT *)d.inv;
    const VT *__restrict__ bp = (const VT *)d.b;
    VT *x = (VT *)d.x;
    __shared__ int s_abort;
    const int tid = threadIdx.x;
    const int nwarps = blockDim.x >> 5;
    const int producer_warp = nwarps - 1;
    const bool tab_c = 4 * d.nchunks <= CSF_TAB;
    if (tab_c)
        for (int i = tid; i < 4 * d.nchunks; i += blockDim.x) tab[i] = reinterpret_cast<const int *>(d.chunks)[i];
    for (int i = tid; i < CSF_XW; i += blockDim.x) tag[i] = -1;
    if (tid < CSF_NS) {
        mbar_init(&full[tid], 1);
        cnt[tid] = 0;
        loaded[tid] = -1;
    }
    if (tid == 0) {
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
    const EllChunk *ch = tab_c ? reinterpret_cast<const EllChunk *>(tab) : d.chunks;
    const long long wlimit = limit;

    if ((tid >> 5) == producer_warp) {
        // ---------------- producer warp ----------------
        // Lane 0 alone waits on the slot mbarriers, always for the phase
        // right after the last one it observed, and publishes each landed
        // chunk in `loaded` (a consumer waiting on a parity two phases ahead
        // of the barrier would be told the phase had completed).  When a
        // chunk's rows are all finished the whole warp copies their x from
        // the window to global memory, so consumers never touch global
        // memory (a CTA fence behind a global store would cost an L2 round
        // trip per row).  A slot is refilled only after its chunk is stored.
        const int lane = tid & 31;
        int issued = 0, published = 0, stored = 0;
        long long idle = 0;
        bool stop = false;
        while (stored < d.nchunks && !stop) {
            int progress = 0;
            if (lane == 0) {
                while (published < issued &&
                       mbar_try_wait(&full[published % CSF_NS], (unsigned)((published / CSF_NS) & 1))) {
                    __threadfence_block();
                    sts_volatile(&loaded[published % CSF_NS], published);
                    ++published;
                    progress = 1;
                }
            }
            int do_store = 0;
            if (lane == 0 && stored < published) {
                const EllChunk c = ch[stored];
                do_store = lds_volatile(&cnt[stored % CSF_NS]) >= c.R1 - c.R0;
            }
            do_store = __shfl_sync(0xffffffffu, do_store, 0);
            if (do_store) {
                __threadfence_block();
                const EllChunk c = ch[stored];
                for (int r = c.R0 + lane; r < c.R1; r += 32) st_relaxed(x + r, xs[r & (CSF_XW - 1)]);
                ++stored;
                progress = 1;
            }
            if (lane == 0 && issued < d.nchunks && (issued < CSF_NS || stored > issued - CSF_NS)) {
                const int s = issued % CSF_NS;
                cnt[s] = 0;
                const EllChunk c = ch[issued];
                unsigned char *slot = sm + (size_t)s * Lay::slot_bytes;
                const int R = c.R1 - c.R0, E = R * c.W;
                const void *src[4];
                int dl[4];
                unsigned nb[4];
                nb[0] = bulk_window(d.col + c.off, E, 4, src[0], dl[0]);
                nb[1] = bulk_window(valp + c.off, E, sizeof(VT), src[1], dl[1]);
                nb[2] = bulk_window(invp + c.R0, R, sizeof(VT), src[2], dl[2]);
                nb[3] = bulk_window(bp + c.R0, R, sizeof(VT), src[3], dl[3]);
                hdr[s * 4 + 0] = dl[0];
                hdr[s * 4 + 1] = dl[1];
                hdr[s * 4 + 2] = dl[2];
                hdr[s * 4 + 3] = dl[3];
                fence_proxy_async();
                mbar_arrive_expect_tx(&full[s], nb[0] + nb[1] + nb[2] + nb[3]);
                if (nb[0]) bulk_g2s(slot + Lay::col_off, src[0], nb[0], &full[s]);
                if (nb[1]) bulk_g2s(slot + Lay::val_off, src[1], nb[1], &full[s]);
                bulk_g2s(slot + Lay::inv_off, src[2], nb[2], &full[s]);
                bulk_g2s(slot + Lay::b_off, src[3], nb[3], &full[s]);
                ++issued;
                progress = 1;
            }
            progress = __shfl_sync(0xffffffffu, progress, 0);
            if (progress) {
                idle = 0;
            } else {
                int ab = lane == 0 ? lds_volatile(&s_abort) : 0;
                if (lane == 0 && !ab && ++idle > wlimit) {
                    atomicOr(status, RBS_STATUS_TIMEOUT);
                    sts_volatile(&s_abort, 1);
                    ab = 1;
                }
                stop = __shfl_sync(0xffffffffu, ab, 0) != 0;
                __nanosleep(32);
            }
        }
        if (lane == 0) {
            // drain copies still in flight (bounded; only after an abort)
            for (int q = published; q < issued; ++q) {
                long long it = 0;
                while (!mbar_try_wait(&full[q % CSF_NS], (unsigned)((q / CSF_NS) & 1)) && ++it <= wlimit) {
                }
            }
        }
        if (stop) {
            // an aborted block still leaves every row written (NaN) for the host check
            for (int r = lane; r < d.m; r += 32) st_relaxed(x + r, Sent<VT>::nan());
        }
        return;
    }

    // ---------------- consumers: groups of G lanes, rows round-robin ----------------
    const int G = d.G;
    const int ngroups = (producer_warp * 32) / G;
    const int grp = tid / G, sl = (tid & 31) % G;
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((tid & 31) / G * G));
    int q = 0, ready_q = -1;
    bool aborted = false;
    for (int r = grp; r < d.m; r += ngroups) {
        while (ch[q].R1 <= r) ++q;
        const int s = q % CSF_NS;
        if (q > ready_q) {
            long long it = 0;
            while (lds_volatile(&loaded[s]) != q) {
                if (it > 8) __nanosleep(32);
                if (aborted || lds_volatile(&s_abort) || ++it > wlimit) {
                    aborted = true;
                    break;
                }
            }
            __threadfence_block();
            if (aborted) {
                atomicOr(status, RBS_STATUS_TIMEOUT);
                sts_volatile(&s_abort, 1);
            } else {
                ready_q = q;
            }
        }
        const EllChunk c = ch[q];
        const int R = c.R1 - c.R0, i = r - c.R0;
        VT sum = 0;
        VT bv = Sent<VT>::nan(), iv = 0;
        if (!aborted) {
            const unsigned char *slot = sm + (size_t)s * Lay::slot_bytes;
            const int *cols = reinterpret_cast<const int *>(slot + Lay::col_off) + hdr[s * 4];
            const VT *vals = reinterpret_cast<const VT *>(slot + Lay::val_off) + hdr[s * 4 + 1];
            iv = reinterpret_cast<const VT *>(slot + Lay::inv_off)[hdr[s * 4 + 2] + i];
            bv = reinterpret_cast<const VT *>(slot + Lay::b_off)[hdr[s * 4 + 3] + i];
            for (int j = sl; j < c.W; j += G) {
                const int cc = cols[j * R + i];
                if (cc < 0) continue;
                const VT v = vals[j * R + i];
                VT xv;
                bool have = false;
                if (r - cc < CSF_XW) {
                    int *tp = &tag[cc & (CSF_XW - 1)];
                    int t = lds_volatile(tp);
                    long long it = 0;
                    while (t < cc) {
                        if (it > 8) __nanosleep(20);
                        if (++it > wlimit || lds_volatile(&s_abort)) {
                            atomicOr(status, RBS_STATUS_TIMEOUT);
                            sts_volatile(&s_abort, 1);
                            aborted = true;
                            break;
                        }
                        t = lds_volatile(tp);
                    }
                    if (!aborted && t == cc) {
                        __threadfence_block();
                        xv = *(volatile VT *)&xs[cc & (CSF_XW - 1)];
                        __threadfence_block();
                        have = lds_volatile(tp) == cc;  // not recycled while reading
                    }
                }
                if (aborted) break;
                if (!have) xv = wait_value(x + cc, status, wlimit);
                sum += v * xv;
            }
        }
        if (G > 1)
            for (int off = G >> 1; off > 0; off >>= 1) sum += __shfl_down_sync(gmask, sum, off, G);
        if (sl == 0) {
            // window slot under a seqlock: mark busy, write, publish the row
            // index (the producer warp copies finished chunks to global)
            const VT xv = aborted ? Sent<VT>::nan() : finalize((bv - sum) * iv);
            int *tp = &tag[r & (CSF_XW - 1)];
            sts_volatile(tp, -1);
            __threadfence_block();
            *(volatile VT *)&xs[r & (CSF_XW - 1)] = xv;
            __threadfence_block();
            sts_volatile(tp, r);
            atomicAdd(&cnt[s], 1);
        }
    }
}

}  // namespace rbs
