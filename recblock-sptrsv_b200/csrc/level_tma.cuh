// level_tma.cuh -- single-CTA level-synchronous triangle with TMA staging.
//
// The plain level kernel (k_tri_level) spends most of each level waiting on
// a chain of dependent global loads (row pointer -> column -> x).  Only the
// x values are on the dependency chain; everything else of a row (row
// pointer, columns, values, inverse diagonal, right-hand side) is known
// before the solve reaches it.  This kernel therefore
//   * streams the block in row chunks (host-chosen: <= RMAX rows and <= EMAX
//     entries each) into an NS-slot shared-memory ring with 1D bulk copies
//     (cp.async.bulk, completion on one mbarrier per slot), NS-1 chunks
//     ahead of the rows being solved;
//   * keeps the x values of the last XW rows in a shared-memory window, so a
//     dependency in a recent level costs a shared-memory load;
//   * walks the local levels (contiguous row ranges) with one CTA barrier per
//     pass (a pass = the rows of one level that fit in the CTA and in the
//     resident chunks).
// Bulk copies need 16-byte aligned addresses and sizes: every copy starts at
// the 16-byte boundary below its first element and is rounded up, and each
// slot records where its first element landed.  Device pools are padded so
// the rounded-up tail never leaves the allocation.
#pragma once

#include "kernels.cuh"

namespace rbs {

constexpr int TMA_RMAX = 512;   // rows per chunk
constexpr int TMA_EMAX = 2048;  // entries per chunk
constexpr int TMA_NS = 5;       // ring slots
constexpr int TMA_XW = 2048;    // x window (rows)
constexpr int TMA_TAB = 6144;   // ints of chunk/level tables staged in shared memory

struct TmaSlotHdr {
    int R0, R1, E0, E1;                   // rows / entries of the chunk (block-local rows, absolute entries)
    int d_rp, d_inv, d_b, d_col, d_val;   // element offset of the first wanted element inside each array
    int pad[3];
};

template <typename VT>
struct TmaLayout {
    static constexpr int RP_CAP = TMA_RMAX + 16;
    static constexpr int V_CAP = TMA_RMAX + 16 / (int)sizeof(VT) + 2;
    static constexpr int COL_CAP = TMA_EMAX + 8;
    static constexpr int VAL_CAP = TMA_EMAX + 16 / (int)sizeof(VT) + 2;
    static constexpr size_t rp_off = 0;
    static constexpr size_t inv_off = rp_off + ((RP_CAP * 4 + 127) / 128) * 128;
    static constexpr size_t b_off = inv_off + ((V_CAP * sizeof(VT) + 127) / 128) * 128;
    static constexpr size_t col_off = b_off + ((V_CAP * sizeof(VT) + 127) / 128) * 128;
    static constexpr size_t val_off = col_off + ((COL_CAP * 4 + 127) / 128) * 128;
    static constexpr size_t slot_bytes = val_off + ((VAL_CAP * sizeof(VT) + 127) / 128) * 128;
    static constexpr size_t ring_off = 0;
    static constexpr size_t xw_off = ring_off + TMA_NS * slot_bytes;
    static constexpr size_t hdr_off = xw_off + TMA_XW * sizeof(VT);
    static constexpr size_t bar_off = hdr_off + TMA_NS * sizeof(TmaSlotHdr);
    static constexpr size_t tab_off = bar_off + TMA_NS * 8;
    static constexpr size_t total = tab_off + TMA_TAB * 4;
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Rounded 16-byte copy window of `count` elements of size `es` starting at
// `src`: returns bytes to copy, sets the aligned source and the element
// offset of src inside the window.
__device__ __forceinline__ unsigned bulk_window(const void *src, int count, int es, const void *&asrc, int &delta) {
    const unsigned long long a = (unsigned long long)src;
    const unsigned long long a0 = a & ~15ull;
    const unsigned long long a1 = (a + (unsigned long long)count * es + 15ull) & ~15ull;
    asrc = (const void *)a0;
    delta = (int)((a - a0) / es);
    return (unsigned)(a1 - a0);
}

struct TmaDesc {
    const int *rp;        // block row pointer (m+1, absolute entry offsets)
    const int *col;       // column pool (block-local columns)
    const void *val;      // value pool
    const void *inv;      // inverse diagonal of the block's rows
    const void *b;        // right-hand side of the block's rows
    void *x;              // solution of the block's rows
    const int *lvl;       // local level pointers (nlv+1)
    const int *chunks;    // chunk row boundaries (nchunks+1), then their entry offsets rp[row] (nchunks+1)
    int m, nlv, nchunks, G;
};

template <typename VT>
__global__ void __launch_bounds__(1024) k_tri_level_tma(const TmaDesc *__restrict__ descs, int *status, long long limit) {
    using Lay = TmaLayout<VT>;
    extern __shared__ __align__(128) unsigned char sm[];
    const TmaDesc d = descs[blockIdx.x];
    TmaSlotHdr *hdr = reinterpret_cast<TmaSlotHdr *>(sm + Lay::hdr_off);
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(sm + Lay::bar_off);
    VT *xs = reinterpret_cast<VT *>(sm + Lay::xw_off);
    const VT *__restrict__ valp = (const VT *)d.val;
    const VT *__restrict__ invp = (const VT *)d.inv;
    const VT *__restrict__ bp = (const VT *)d.b;
    VT *x = (VT *)d.x;
    const int tid = threadIdx.x;
    const int G = d.G;
    const int lane = tid & 31, sl = lane % G, gslot = tid / G, nslots = blockDim.x / G;
    __shared__ int s_abort;
    if (tid < TMA_NS) mbar_init(&bar[tid], 1);
    if (tid == 0) {
        fence_mbar_init();
        s_abort = 0;
    }
    // chunk boundaries (rows, entries) and level pointers in shared memory
    // when they fit: the pass loop reads them on every level
    int *tab = reinterpret_cast<int *>(sm + Lay::tab_off);
    const int nct = d.nchunks + 1;
    const bool tab_chunks = 2 * nct <= TMA_TAB;
    const bool tab_lvl = tab_chunks && 2 * nct + d.nlv + 1 <= TMA_TAB;
    if (tab_chunks)
        for (int i = tid; i < 2 * nct; i += blockDim.x) tab[i] = d.chunks[i];
    if (tab_lvl)
        for (int i = tid; i <= d.nlv; i += blockDim.x) tab[2 * nct + i] = d.lvl[i];
    const int *cR = tab_chunks ? tab : d.chunks;
    const int *cE = cR + nct;
    const int *lv = tab_lvl ? tab + 2 * nct : d.lvl;
    __syncthreads();
    // a bulk copy completes in microseconds; waits give up after `wlimit`
    // polls, raise the status and make every later wait of the CTA skip
    const long long wlimit = limit < (1ll << 20) ? limit : (1ll << 20);

    int q_issue = 0;  // next chunk to load (thread 0 only)
    int q_a = 0;      // chunk holding the first row of the current pass (all threads)
    bool timed_out = false;
    for (int l = 0; l < d.nlv; ++l) {
        const int lo = lv[l], hi = lv[l + 1];
        for (int ra = lo; ra < hi;) {
            while (cR[q_a + 1] <= ra) ++q_a;
            const int qlim = min(q_a + TMA_NS - 1, d.nchunks);
            const int rb = min(min(hi, ra + nslots), cR[qlim]);
            if (tid == 0 && !s_abort) {
                // refill every slot whose chunk lies entirely before this pass
                while (q_issue < d.nchunks && (q_issue < TMA_NS || cR[q_issue - TMA_NS + 1] <= ra)) {
                    const int s = q_issue % TMA_NS;
                    unsigned char *slot = sm + Lay::ring_off + (size_t)s * Lay::slot_bytes;
                    TmaSlotHdr h;
                    h.R0 = cR[q_issue];
                    h.R1 = cR[q_issue + 1];
                    h.E0 = cE[q_issue];
                    h.E1 = cE[q_issue + 1];
                    const void *src[5];
                    unsigned nb[5];
                    nb[0] = bulk_window(d.rp + h.R0, h.R1 - h.R0 + 1, 4, src[0], h.d_rp);
                    nb[1] = bulk_window(invp + h.R0, h.R1 - h.R0, sizeof(VT), src[1], h.d_inv);
                    nb[2] = bulk_window(bp + h.R0, h.R1 - h.R0, sizeof(VT), src[2], h.d_b);
                    nb[3] = bulk_window(d.col + h.E0, h.E1 - h.E0, 4, src[3], h.d_col);
                    nb[4] = bulk_window(valp + h.E0, h.E1 - h.E0, sizeof(VT), src[4], h.d_val);
                    hdr[s] = h;
                    fence_proxy_async();
                    unsigned total = 0;
                    for (int i = 0; i < 5; ++i) total += nb[i];
                    mbar_arrive_expect_tx(&bar[s], total);
                    bulk_g2s(slot + Lay::rp_off, src[0], nb[0], &bar[s]);
                    bulk_g2s(slot + Lay::inv_off, src[1], nb[1], &bar[s]);
                    bulk_g2s(slot + Lay::b_off, src[2], nb[2], &bar[s]);
                    if (nb[3]) bulk_g2s(slot + Lay::col_off, src[3], nb[3], &bar[s]);
                    if (nb[4]) bulk_g2s(slot + Lay::val_off, src[4], nb[4], &bar[s]);
                    ++q_issue;
                }
            }
            const int row = ra + gslot;
            const bool active = row < rb;
            VT sum = 0;
            int q = q_a;
            if (active) {
                while (cR[q + 1] <= row) ++q;
                const int s = q % TMA_NS;
                const unsigned parity = (unsigned)((q / TMA_NS) & 1);
                long long it = 0;
                bool ready = !s_abort;
                while (ready && !mbar_try_wait(&bar[s], parity)) {
                    if (++it > wlimit) {
                        timed_out = true;
                        ready = false;
                        s_abort = 1;
                    }
                }
                if (ready) {
                    const TmaSlotHdr &h = hdr[s];
                    const unsigned char *slot = sm + Lay::ring_off + (size_t)s * Lay::slot_bytes;
                    const int *rps = reinterpret_cast<const int *>(slot + Lay::rp_off) + h.d_rp;
                    const int *cols = reinterpret_cast<const int *>(slot + Lay::col_off) + h.d_col - h.E0;
                    const VT *vals = reinterpret_cast<const VT *>(slot + Lay::val_off) + h.d_val - h.E0;
                    const int e0 = max(rps[row - h.R0], h.E0), e1 = min(rps[row - h.R0 + 1], h.E1);
                    for (int k = e0 + sl; k < e1; k += G) {
                        const int c = cols[k];
                        if ((unsigned)c >= (unsigned)lo) continue;  // only earlier levels (guards corrupt data)
                        const VT xv = c >= hi - TMA_XW ? xs[c & (TMA_XW - 1)] : x[c];
                        sum += vals[k] * xv;
                    }
                } else {
                    sum = Sent<VT>::nan();
                }
            }
            for (int off = G >> 1; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off, G);
            if (active && sl == 0) {
                const int s = q % TMA_NS;
                const TmaSlotHdr &h = hdr[s];
                const unsigned char *slot = sm + Lay::ring_off + (size_t)s * Lay::slot_bytes;
                const VT iv = reinterpret_cast<const VT *>(slot + Lay::inv_off)[h.d_inv + row - h.R0];
                const VT bv = reinterpret_cast<const VT *>(slot + Lay::b_off)[h.d_b + row - h.R0];
                const VT xv = finalize((bv - sum) * iv);
                xs[row & (TMA_XW - 1)] = xv;
                x[row] = xv;
            }
            __syncthreads();
            ra = rb;
        }
    }
    if (timed_out) atomicOr(status, RBS_STATUS_TIMEOUT);
    __syncthreads();
    if (s_abort && tid == 0) {
        // drain: wait (bounded) for the copies still in flight before exiting
        for (int q = max(0, q_issue - TMA_NS); q < q_issue; ++q) {
            long long it = 0;
            while (!mbar_try_wait(&bar[q % TMA_NS], (unsigned)((q / TMA_NS) & 1)) && ++it <= wlimit) {
            }
        }
    }
}

}  // namespace rbs
