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
// itself (cp.async.wait_group), so staging needs no extra synchronisation;
// in triangles of wide levels it reads the next level's row into registers
// before the barrier that ends a level.
//
// Layout (host-built): per level l a table entry {lo, off, w, 0}: rows
// [lo, lo + w) of the block; the block's ELL width W (1, 2 or 4) is fixed,
// entry j of row lo+i at col/val[off + i*W + j] (row-major, padding column
// -1), so a thread stages its row's columns and values with one or two
// 4-16 byte copies and the level's loads are coalesced.
// Dependencies within the last XW rows come from the window; older ones
// from x in global memory (written by this CTA before an earlier barrier).
// When every dependency lies in the window (WIN) and W >= 2, the columns are
// window slots (0..XW, XW the zero slot) held as 16-bit integers: a row's
// columns are one 4- or 8-byte copy, and the level's column reads take half
// the shared-memory wavefronts of 32-bit columns.  Wide levels are bound by
// the shared-memory pipe, which carries every staged byte twice.
//
// Several right-hand sides: CTA y of the launch's second grid dimension
// solves the G consecutive columns [y*G, y*G+G) on its own, with no
// synchronisation between CTAs: every column group walks the same levels
// with its own window (G values per slot), and the rows' columns, values and
// inverse diagonal, which all groups share, come through L2.  One dependency
// walk per group serves G columns; the groups run side by side on separate
// SMs.  The work vectors are either row-interleaved (entry (row, c) at
// row*K + c: ld = K, groups G apart) or grouped (each group's rows
// contiguous, G values per row: ld = G, groups n*G apart), where a thread's
// G values sit next to its neighbours' and a warp's copies coalesce.  No L2
// prefetch runs ahead of the staging: with grouped vectors the copies S-1
// levels ahead already hide the latency, and a prefetch of each row 12
// levels ahead measured 8-23 % slower at 8 to 128 columns (its instructions
// sit in every level of every CTA).
#pragma once

#include <type_traits>

#include "kernels.cuh"
#include "rbs_internal.h"

namespace rbs {

constexpr int CA_ROWS = 1024;            // rows per level (= threads)
constexpr int CA_XW = CA_WINDOW_ROWS;    // x window (rows), plus one always-zero slot
constexpr int CA_TAB = 6144;   // ints of the level table staged in shared memory (4 per level)

struct CaDesc {
    const void *col;  // row-major level-ELL columns: block-local rows (int, padding -1), or
                      // window slots (short, padding the zero slot) for WIN blocks with W >= 2
    const void *val;  // level-ELL values
    const void *inv;  // inverse diagonal of the block's rows
    const void *b;    // right-hand side of the block's rows, column group 0 (row stride ld)
    void *x;          // solution of the block's rows, column group 0 (row stride ld)
    const int *lvl;   // per level: lo, off, w, 0 (4 ints), then {m, 0, 0, 0}
    int m, nlv, ld, pad1;
    long long gstride;  // elements from one column group to the next
};

// CB: bytes per column (4, or 2 for window slots)
template <typename VT, int W, int S, int G = 1, int CB = 4>
struct CaLayout {
    static constexpr size_t col_bytes = (size_t)W * CA_ROWS * CB;
    static constexpr size_t val_bytes = (size_t)W * CA_ROWS * sizeof(VT);
    static constexpr size_t inv_bytes = (size_t)CA_ROWS * sizeof(VT);
    static constexpr size_t b_bytes = (size_t)G * CA_ROWS * sizeof(VT);
    static constexpr size_t stage_bytes = col_bytes + val_bytes + inv_bytes + b_bytes;
    static constexpr size_t xw_off = S * stage_bytes;
    static constexpr size_t tab_off = xw_off + (CA_XW + 16) * G * sizeof(VT);
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
__device__ __forceinline__ void cp_async_s4(unsigned dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_s8(unsigned dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_s16(unsigned dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
// `BYTES` (4, 8, 16 or 32) contiguous bytes to a shared-memory address
template <int BYTES>
__device__ __forceinline__ void cp_async_sn(unsigned dst, const void *src) {
    if constexpr (BYTES == 4) cp_async_s4(dst, src);
    else if constexpr (BYTES == 8) cp_async_s8(dst, src);
    else if constexpr (BYTES == 16) cp_async_s16(dst, src);
    else {
        static_assert(BYTES == 32, "row segment of 4, 8, 16 or 32 bytes");
        cp_async_s16(dst, src);
        cp_async_s16(dst + 16, static_cast<const char *>(src) + 16);
    }
}


// The level loop is unrolled by the stage count S, so every stage address
// is a compile-time offset from per-thread bases computed once.
// WIN: the block's columns are window slots (every dependency within the
// window; padding reads the zero slot), so a dependency is one shared-memory
// load and an unconditional multiply-add.
// G: right-hand sides per CTA (blockIdx.y selects the column group).
// MC: a multi-column launch; without it the row stride is 1 and there is
// one group (the single right-hand-side solve, with no stride arithmetic).
template <int W, bool WIN>
constexpr int ca_col_bytes() {
    return WIN && W >= 2 ? 2 : 4;
}

// Dynamic shared memory of one instance of k_tri_level_ca.
template <typename VT, int W, int S, bool WIN, int G>
constexpr size_t ca_smem_total() {
    return CaLayout<VT, W, S, G, ca_col_bytes<W, WIN>()>::total;
}

// LATE (with S = 4): the late copies and register read-ahead below, for
// triangles of wide levels.
template <typename VT, int W, int S, bool WIN, int G = 1, bool MC = false, bool LATE = false>
__global__ void __launch_bounds__(1024) k_tri_level_ca(const CaDesc *__restrict__ descs) {
    constexpr int CB = ca_col_bytes<W, WIN>();
    using CT = std::conditional_t<CB == 2, short, int>;
    using Lay = CaLayout<VT, W, S, G, CB>;
    using VG = Vec<VT, G>;
    static_assert(S == 2 || S == 4, "stage count 2 or 4");
    static_assert(G == 1 || G == 2 || G == 4, "1, 2 or 4 right-hand sides per CTA");
    extern __shared__ __align__(128) unsigned char sm[];
    const CaDesc d = descs[blockIdx.x];
    static_assert(MC || G == 1, "one column per CTA without a multi-column launch");
    const int ld = MC ? d.ld : 1;
    const long long goff = MC ? (long long)blockIdx.y * d.gstride : 0;
    VT *x = (VT *)d.x + goff;
    VG *xs = reinterpret_cast<VG *>(sm + Lay::xw_off);
    int *tab = reinterpret_cast<int *>(sm + Lay::tab_off);
    const int tid = threadIdx.x;
    const int nlv = d.nlv;
    const int ntab = 4 * (nlv + 1);
    const bool in_smem = ntab <= CA_TAB;
    if (in_smem)
        for (int i = tid; i < ntab; i += blockDim.x) tab[i] = d.lvl[i];
    if (tid == 0) {
        VG z;
#pragma unroll
        for (int g = 0; g < G; ++g) z.v[g] = VT(0);
        xs[CA_XW] = z;
    }
    __syncthreads();
    const int4 *lt = reinterpret_cast<const int4 *>(in_smem ? tab : d.lvl);

    // this thread's source rows and stage-0 slots
    const CT *colp = static_cast<const CT *>(d.col) + tid * W;
    const VT *valp = (const VT *)d.val + tid * W;
    const VT *inv_t = (const VT *)d.inv + tid;
    const VT *b_t = (const VT *)d.b + goff + (size_t)tid * ld;
    const unsigned s0 = (unsigned)__cvta_generic_to_shared(sm);
    const unsigned s_col = s0 + tid * W * CB;
    const unsigned s_val = s0 + (unsigned)Lay::col_bytes + tid * W * (unsigned)sizeof(VT);
    const unsigned s_inv = s0 + (unsigned)(Lay::col_bytes + Lay::val_bytes) + tid * (unsigned)sizeof(VT);
    const unsigned s_b = s0 + (unsigned)(Lay::col_bytes + Lay::val_bytes + Lay::inv_bytes) +
                         tid * G * (unsigned)sizeof(VT);

    // stage the row data of level l into slot U (= l % S) for this thread,
    // one commit group per level
    // e: the level's table entry {lo, off, w}
    auto stage = [&](int l, const int4 &e, auto slot) {
        constexpr unsigned off = decltype(slot)::value * (unsigned)Lay::stage_bytes;
        if (l < nlv && tid < e.z) {
            cp_async_sn<CB * W>(s_col + off, colp + e.y);
            cp_async_sn<(int)sizeof(VT) * W>(s_val + off, valp + e.y);
            cp_async_sn<(int)sizeof(VT)>(s_inv + off, inv_t + e.x);
            cp_async_sn<(int)sizeof(VT) * G>(s_b + off, b_t + (size_t)e.x * ld);
        }
        cp_async_commit();
    };
    // table entries of levels l .. l+S-1 in registers, entry of level l' in
    // ent[l' % S] (compile-time indices in the unrolled loop)
    int4 ent[S];
#pragma unroll
    for (int k = 0; k < S; ++k) ent[k] = lt[k < nlv ? k : nlv];
    // solve level l: read the entry of level l+S a level early.  Late (S = 4,
    // triangles of wide levels): after the level's work, stage level l+S-1
    // into the slot freed at the last barrier, wait for this thread's copies
    // of level l+1 (two groups may stay in flight) and read them into
    // registers, all before the barrier; copies issued at the start of a
    // wide level queue ahead of its dependency reads (c1a's wide triangles
    // 108-111 -> 103-107 us).  Otherwise stage at the start of the level and
    // wait for level l's own copies: a narrow level is bound by its barrier
    // chain, which the read-ahead lengthens (c1a's narrow triangles 148-150
    // -> 154-155 us with it); with S = 2 a later issue would leave no level
    // between copy and use.
    constexpr bool late = S == 4 && LATE;
    // late: this thread's staged row of the next level, read into registers
    // before the barrier that starts it (a thread reads only its own copies,
    // so only the window reads must wait for the barrier)
    Vec<CT, W> ncs{};
    Vec<VT, W> nvs{};
    VT niv{};
    VG nbv{};
    auto load_staged = [&](int w, auto slot) {
        constexpr int U = decltype(slot)::value;
        if (tid < w) {
            const unsigned char *st = sm + (size_t)U * Lay::stage_bytes;
            ncs = reinterpret_cast<const Vec<CT, W> *>(st)[tid];
            nvs = reinterpret_cast<const Vec<VT, W> *>(st + Lay::col_bytes)[tid];
            niv = reinterpret_cast<const VT *>(st + Lay::col_bytes + Lay::val_bytes)[tid];
            nbv = reinterpret_cast<const VG *>(st + Lay::col_bytes + Lay::val_bytes + Lay::inv_bytes)[tid];
        }
    };
    auto level = [&](int l, int &lo, auto slot) {
        constexpr int U = decltype(slot)::value;
        const int hi = ent[(U + 1) % S].x;
        const int4 e_stage = ent[(U + S - 1) % S];
        if (l + S <= nlv) ent[U] = lt[l + S];  // level l's own entry is no longer needed
        if constexpr (!late) {
            stage(l + S - 1, e_stage, std::integral_constant<int, (U + S - 1) % S>{});
            cp_async_wait<S - 1>();
        }
        if (tid < hi - lo) {
            Vec<CT, W> cs;
            Vec<VT, W> vs;
            VT iv;
            VG bv;
            if constexpr (late) {
                cs = ncs;
                vs = nvs;
                iv = niv;
                bv = nbv;
            } else {
                const unsigned char *st = sm + (size_t)U * Lay::stage_bytes;
                cs = reinterpret_cast<const Vec<CT, W> *>(st)[tid];
                vs = reinterpret_cast<const Vec<VT, W> *>(st + Lay::col_bytes)[tid];
                iv = reinterpret_cast<const VT *>(st + Lay::col_bytes + Lay::val_bytes)[tid];
                bv = reinterpret_cast<const VG *>(st + Lay::col_bytes + Lay::val_bytes + Lay::inv_bytes)[tid];
            }
            VT sum[G];
#pragma unroll
            for (int g = 0; g < G; ++g) sum[g] = 0;
#pragma unroll
            for (int j = 0; j < W; ++j) {
                const int c = cs.v[j];
                if constexpr (WIN) {
                    const VG xv = xs[c];
#pragma unroll
                    for (int g = 0; g < G; ++g) sum[g] += vs.v[j] * xv.v[g];
                } else if (c >= 0) {
                    VG xv;
                    if (c >= hi - CA_XW) xv = xs[c & (CA_XW - 1)];
                    else if constexpr (G == 1) xv.v[0] = x[(size_t)c * ld];
                    else xv = *reinterpret_cast<const VG *>(x + (size_t)c * ld);
#pragma unroll
                    for (int g = 0; g < G; ++g) sum[g] += vs.v[j] * xv.v[g];
                }
            }
            const int r = lo + tid;
            VG xv;
#pragma unroll
            for (int g = 0; g < G; ++g) xv.v[g] = finalize((bv.v[g] - sum[g]) * iv);
            xs[r & (CA_XW - 1)] = xv;
            if constexpr (G == 1) x[(size_t)r * ld] = xv.v[0];
            else *reinterpret_cast<VG *>(x + (size_t)r * ld) = xv;
        }
        if constexpr (late) {
            stage(l + S - 1, e_stage, std::integral_constant<int, (U + S - 1) % S>{});
            cp_async_wait<S - 2>();
            load_staged(ent[(U + 2) % S].x - hi, std::integral_constant<int, (U + 1) % S>{});
        }
        lo = hi;
        __syncthreads();
    };

    stage(0, ent[0], std::integral_constant<int, 0>{});
    if constexpr (S == 4) {
        stage(1, ent[1], std::integral_constant<int, 1>{});
        stage(2, ent[2], std::integral_constant<int, 2>{});
    }
    if constexpr (late) {
        cp_async_wait<S - 2>();
        load_staged(ent[1].x, std::integral_constant<int, 0>{});
    }
    int lo = 0;
#pragma unroll 1
    for (int l = 0; l < nlv; l += S) {
        level(l, lo, std::integral_constant<int, 0>{});
        if (l + 1 >= nlv) break;
        level(l + 1, lo, std::integral_constant<int, 1>{});
        if constexpr (S == 4) {
            if (l + 2 >= nlv) break;
            level(l + 2, lo, std::integral_constant<int, 2>{});
            if (l + 3 >= nlv) break;
            level(l + 3, lo, std::integral_constant<int, 3>{});
        }
    }
    cp_async_wait<0>();
}

}  // namespace rbs
