// kernels.cuh -- sm_100a kernels of the recursive-block triangular solve.
//
// All triangles are solved in processing order (lower triangular, see
// rbs_internal.h).  Work vectors are row-interleaved: entry (row p, rhs c)
// of a K-wide vector lives at v[p*K + c], so the K values one row produces
// or consumes are contiguous.
//
// Readiness of x: the solution work vector is filled with a NaN sentinel
// before a solve; a value is ready when it no longer carries the sentinel
// bit pattern.  Arithmetic never produces that pattern (the hardware's NaN
// is canonical and results equal to it are replaced), so one relaxed load
// both polls and fetches the value: no separate flag array, no fence.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rbs {

#define RBS_SENT64 0xFFF8DEADBEEFCAFEull
#define RBS_SENT32 0xFFC0DEADu
#define RBS_STATUS_TIMEOUT 1
#define RBS_LONGROW 2048
#define RBS_MEDROW 8  // squares, single RHS, lane group < 32: longer rows take a warp each

template <typename VT> struct Sent;
template <> struct Sent<double> {
    __device__ __forceinline__ static double value() { return __longlong_as_double((long long)RBS_SENT64); }
    __device__ __forceinline__ static bool is(double v) {
        return (unsigned long long)__double_as_longlong(v) == RBS_SENT64;
    }
    __device__ __forceinline__ static double nan() { return __longlong_as_double(0x7FF8000000000000ll); }
};
template <> struct Sent<float> {
    __device__ __forceinline__ static float value() { return __uint_as_float(RBS_SENT32); }
    __device__ __forceinline__ static bool is(float v) { return __float_as_uint(v) == RBS_SENT32; }
    __device__ __forceinline__ static float nan() { return __uint_as_float(0x7FC00000u); }
};

__device__ __forceinline__ double ld_relaxed(const double *p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ float ld_relaxed(const float *p) {
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(double *p, double v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(float *p, float v) {
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

// Wait until x[i] is produced.  Bounded: after `limit` polls the wait gives
// up, raises RBS_STATUS_TIMEOUT and returns NaN so dependants still finish.
// Polls back off to at most 128 ns apart: a backoff growing to 1 us added up
// to a microsecond to every dependency hop of narrow levels (the power-law
// factor's first triangle spent most of its 67 us asleep).
template <typename VT>
__device__ __forceinline__ VT wait_value(const VT *p, int *status, long long limit) {
    VT v = ld_relaxed(p);
    if (!Sent<VT>::is(v)) return v;
    unsigned ns = 32;
    for (long long it = 0; it < limit; ++it) {
        if (it > 16) {
            __nanosleep(ns);
            if (ns < 128) ns <<= 1;
        }
        v = ld_relaxed(p);
        if (!Sent<VT>::is(v)) return v;
    }
    atomicOr(status, RBS_STATUS_TIMEOUT);
    return Sent<VT>::nan();
}

template <typename VT>
__device__ __forceinline__ VT finalize(VT v) {
    return Sent<VT>::is(v) ? Sent<VT>::nan() : v;
}

// N values of type T moved as one aligned access
template <typename T, int N>
struct alignas(sizeof(T) * N) Vec {
    T v[N];
};

// ---------------------------------------------------------------------------
// Vector permutations (utils_cuda.h:858-876 levelset_reordering_vecb/vecx,
// fused with the RHS interleave, the precision cast and the sentinel reset).
// ---------------------------------------------------------------------------
template <typename VT, int K>
__global__ void k_gather(const double *__restrict__ b, int ld, int k, const int *__restrict__ perm, int n,
                         VT *__restrict__ out) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)n * K;
    for (; t < total; t += (long long)gridDim.x * blockDim.x) {
        int p = (int)(t / K), c = (int)(t % K);
        double v = c < k ? b[(long long)c * ld + perm[p]] : 0.0;
        out[t] = (VT)v;
    }
}

// x[perm[p] + c*ld] = xw[p*K + c]; xw reset to the sentinel for the next solve.
template <typename VT, int K>
__global__ void k_scatter_reset(VT *__restrict__ xw, const int *__restrict__ perm, int n, int k, double *x,
                                int ld) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)n * K;
    for (; t < total; t += (long long)gridDim.x * blockDim.x) {
        int p = (int)(t / K), c = (int)(t % K);
        VT v = xw[t];
        if (c < k) x[(long long)c * ld + perm[p]] = (double)v;
        xw[t] = Sent<VT>::value();
    }
}

// The same from a table of column pointers (one device pointer per
// right-hand side, e.g. the columns of several requests batched together):
// out[p*K + c] = cols[c][perm[p]], 0 for c >= k.
template <typename VT, int K>
__global__ void k_gather_cols(const double *const *__restrict__ cols, int k, const int *__restrict__ perm, int n,
                              VT *__restrict__ out) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)n * K;
    for (; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(t / K), c = (int)(t % K);
        out[t] = c < k ? (VT)cols[c][perm[p]] : VT(0);
    }
}

// cols[c][perm[p]] = xw[p*K + c] for c < k; xw reset to the sentinel.
template <typename VT, int K>
__global__ void k_scatter_cols(VT *__restrict__ xw, const int *__restrict__ perm, int n, int k,
                               double *const *__restrict__ cols) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)n * K;
    for (; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(t / K), c = (int)(t % K);
        const VT v = xw[t];
        if (c < k) cols[c][perm[p]] = (double)v;
        xw[t] = Sent<VT>::value();
    }
}

// Transposing forms of the gather and scatter for many right-hand sides
// with the row-interleaved work vector (entry (p, c) at p*K + c): a CTA takes
// a tile of 32 original rows, reads it column by column (32 consecutive
// values of a column: coalesced), and writes every row at its processing
// position (K consecutive values: coalesced), through a shared-memory tile;
// the scatter runs the other way.  Columns come from b + c*ld, or from the
// table cols[c] when cols is not NULL.  ipos[i] is the processing position
// of original row i.
constexpr int TP_ROWS = 32;

// Columns of several independent systems solved as one block-diagonal plan
// (a server group): column c of system f comes from tab[c*F + f] (NULL: no
// request there, zeros in, nothing out); seg[i] is the system of original
// row i, off[f] its first row.
struct GroupCols {
    const double *const *tab;
    const int *seg, *off;
    int F;
};

__device__ __forceinline__ const double *group_src(const GroupCols &g, int c, long long i, long long &r) {
    const int f = g.seg[i];
    r = i - g.off[f];
    return g.tab[(long long)c * g.F + f];
}

template <typename VT, typename VT2, int K>
__global__ void __launch_bounds__(256) k_gather_t(const double *__restrict__ b, int ld,
                                                  const double *const *__restrict__ cols, int k,
                                                  const int *__restrict__ ipos, int n, VT *__restrict__ out,
                                                  VT2 *__restrict__ out2, GroupCols grp) {
    __shared__ double tile[K][TP_ROWS + 1];
    for (long long i0 = (long long)blockIdx.x * TP_ROWS; i0 < n; i0 += (long long)gridDim.x * TP_ROWS) {
        const int rows = (int)min((long long)TP_ROWS, n - i0);
        for (int e = threadIdx.x; e < K * TP_ROWS; e += blockDim.x) {
            const int c = e / TP_ROWS, t = e % TP_ROWS;
            double v = 0.0;
            if (c < k && t < rows) {
                if (grp.tab) {
                    long long r;
                    const double *src = group_src(grp, c, i0 + t, r);
                    if (src) v = src[r];
                } else {
                    v = cols ? cols[c][i0 + t] : b[(long long)c * ld + i0 + t];
                }
            }
            tile[c][t] = v;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < K * TP_ROWS; e += blockDim.x) {
            const int t = e / K, c = e % K;
            if (t < rows) {
                const long long o = (long long)ipos[i0 + t] * K + c;
                out[o] = (VT)tile[c][t];
                if (out2) out2[o] = (VT2)tile[c][t];
            }
        }
        __syncthreads();
    }
}

// RESET: the work vector is set back to the sentinel as it is read.
template <typename VT, int K, bool RESET>
__global__ void __launch_bounds__(256) k_scatter_t(VT *__restrict__ xw, const int *__restrict__ ipos, int n, int k,
                                                   double *__restrict__ x, int ld, double *const *__restrict__ cols,
                                                   GroupCols grp) {
    __shared__ double tile[K][TP_ROWS + 1];
    for (long long i0 = (long long)blockIdx.x * TP_ROWS; i0 < n; i0 += (long long)gridDim.x * TP_ROWS) {
        const int rows = (int)min((long long)TP_ROWS, n - i0);
        for (int e = threadIdx.x; e < K * TP_ROWS; e += blockDim.x) {
            const int t = e / K, c = e % K;
            if (t < rows) {
                const long long o = (long long)ipos[i0 + t] * K + c;
                tile[c][t] = (double)xw[o];
                if (RESET) xw[o] = Sent<VT>::value();
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < K * TP_ROWS; e += blockDim.x) {
            const int c = e / TP_ROWS, t = e % TP_ROWS;
            if (c < k && t < rows) {
                if (grp.tab) {
                    long long r;
                    double *dst = const_cast<double *>(group_src(grp, c, i0 + t, r));
                    if (dst) dst[r] = tile[c][t];
                } else if (cols) {
                    cols[c][i0 + t] = tile[c][t];
                } else {
                    x[(long long)c * ld + i0 + t] = tile[c][t];
                }
            }
        }
        __syncthreads();
    }
}

// Gather and scatter for the grouped work vector (column group g = c / GL
// holds its rows contiguously, GL values per row: entry (p, c) at
// g*n*GL + p*GL + c % GL).  One thread per processing position p and GT
// column groups: the work-vector side is one GL-wide vector access per
// group (consecutive threads, consecutive positions: coalesced), the
// caller's side GL single values at the original row perm[p].  Grid x runs
// over positions, grid y over chunks of GT groups, so the CTAs resident at
// one time work on one chunk of columns and the rows they touch out of order
// (GT*GL columns of n values) stay in L2 until every value of a sector has
// been used.  Only positions [pa, pb) are moved (a range of triangles when
// the moves overlap the block walk).  Columns c in [k, K), and columns whose
// table entry cols[c] is NULL, get zeros on the way in and are not written
// out.
template <int K, int GL>
struct GroupTile {
    static_assert(GL > 0 && K % GL == 0, "grouped layout");
    static constexpr int NG = K / GL;              // column groups
    static constexpr int GT = NG < 4 ? NG : 4;     // groups per thread
    static constexpr int CHUNKS = (NG + GT - 1) / GT;
};

template <typename VT, typename VT2, int K, int GL>
__global__ void __launch_bounds__(256) k_gather_grp(const double *__restrict__ b, int ld,
                                                    const double *const *__restrict__ cols, int k,
                                                    const int *__restrict__ perm, int n, int pa, int pb,
                                                    VT *__restrict__ out, VT2 *__restrict__ out2, GroupCols grp) {
    using T = GroupTile<K, GL>;
    const long long p = pa + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pb) return;
    const int g0 = blockIdx.y * T::GT;
    const long long i = perm[p];
    long long r = i;
    int f = 0;
    if (grp.tab) {
        f = grp.seg[i];
        r = i - grp.off[f];
    }
    double v[T::GT][GL];
#pragma unroll
    for (int a = 0; a < T::GT; ++a)
#pragma unroll
        for (int j = 0; j < GL; ++j) {
            const int c = (g0 + a) * GL + j;
            double t = 0.0;
            if (c < k) {
                if (grp.tab) {
                    const double *src = grp.tab[(long long)c * grp.F + f];
                    if (src) t = src[r];
                } else if (cols) {
                    const double *src = cols[c];
                    if (src) t = src[i];
                } else {
                    t = b[(long long)c * ld + i];
                }
            }
            v[a][j] = t;
        }
#pragma unroll
    for (int a = 0; a < T::GT; ++a) {
        const int g = g0 + a;
        if (T::NG % T::GT != 0 && g >= T::NG) break;
        const long long o = (long long)g * n * GL + p * GL;
        Vec<VT, GL> w;
#pragma unroll
        for (int j = 0; j < GL; ++j) w.v[j] = (VT)v[a][j];
        *reinterpret_cast<Vec<VT, GL> *>(out + o) = w;
        if (out2) {
            Vec<VT2, GL> w2;
#pragma unroll
            for (int j = 0; j < GL; ++j) w2.v[j] = (VT2)v[a][j];
            *reinterpret_cast<Vec<VT2, GL> *>(out2 + o) = w2;
        }
    }
}

// RESET: the work vector is set back to the sentinel as it is read (every
// one of the K columns, as the solve expects).
template <typename VT, int K, int GL, bool RESET>
__global__ void __launch_bounds__(256) k_scatter_grp(VT *__restrict__ xw, const int *__restrict__ perm, int n, int k,
                                                     int pa, int pb, double *__restrict__ x, int ld,
                                                     double *const *__restrict__ cols, GroupCols grp) {
    using T = GroupTile<K, GL>;
    const long long p = pa + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pb) return;
    const int g0 = blockIdx.y * T::GT;
    const long long i = perm[p];
    long long r = i;
    int f = 0;
    if (grp.tab) {
        f = grp.seg[i];
        r = i - grp.off[f];
    }
    Vec<VT, GL> w[T::GT];
#pragma unroll
    for (int a = 0; a < T::GT; ++a) {
        const int g = g0 + a;
        if (T::NG % T::GT != 0 && g >= T::NG) break;
        VT *src = xw + (long long)g * n * GL + p * GL;
        w[a] = *reinterpret_cast<const Vec<VT, GL> *>(src);
        if (RESET) {
            Vec<VT, GL> s;
#pragma unroll
            for (int j = 0; j < GL; ++j) s.v[j] = Sent<VT>::value();
            *reinterpret_cast<Vec<VT, GL> *>(src) = s;
        }
    }
#pragma unroll
    for (int a = 0; a < T::GT; ++a)
#pragma unroll
        for (int j = 0; j < GL; ++j) {
            const int c = (g0 + a) * GL + j;
            if (c >= k) continue;
            const double t = (double)w[a].v[j];
            if (grp.tab) {
                double *dst = const_cast<double *>(grp.tab[(long long)c * grp.F + f]);
                if (dst) dst[r] = t;
            } else if (cols) {
                if (cols[c]) cols[c][i] = t;
            } else {
                x[(long long)c * ld + i] = t;
            }
        }
}

// Grouped scatter of one triangle's solutions in ORIGINAL row order: rows[q]
// for q in [qa, qb) lists the triangle's original rows ascending, so a
// warp's writes to a caller's column fall on neighbouring rows (whole
// sectors), while the work vector is read out of order at each row's
// processing position ipos[i], one GL-wide vector per group (reads out of
// order are what L2 absorbs; writes out of order of 8 bytes are not).  A CTA
// takes TR rows and a chunk of GT column groups through a shared-memory
// tile.  Columns whose table entry is NULL are not written.
// The work vector keeps its values (no sentinel reset).
template <typename VT, int K, int GL>
__global__ void __launch_bounds__(256) k_scatter_rows(const VT *__restrict__ xw, const int *__restrict__ rows,
                                                     const int *__restrict__ ipos, int n, int qa, int qb,
                                                     double *const *__restrict__ cols) {
    using T = GroupTile<K, GL>;
    static_assert(T::NG % T::GT == 0 && 256 % T::GT == 0, "whole chunks");
    constexpr int CC = T::GT * GL;  // columns per chunk
    constexpr int TR = 256 / T::GT;  // rows per tile
    __shared__ double tile[CC][TR + 1];
    __shared__ int trow[TR];
    const int g0 = blockIdx.y * T::GT;
    const long long q0 = qa + (long long)blockIdx.x * TR;
    {
        const int t = threadIdx.x % TR, a = threadIdx.x / TR;
        const long long q = q0 + t;
        if (q < qb) {
            const int i = rows[q];
            if (a == 0) trow[t] = i;
            const Vec<VT, GL> w =
                *reinterpret_cast<const Vec<VT, GL> *>(xw + (long long)(g0 + a) * n * GL + (long long)ipos[i] * GL);
#pragma unroll
            for (int j = 0; j < GL; ++j) tile[a * GL + j][t] = (double)w.v[j];
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < CC * TR; e += blockDim.x) {
        const int cl = e / TR, t = e % TR;
        if (q0 + t < qb) {
            double *dst = cols[g0 * GL + cl];
            if (dst) dst[trow[t]] = tile[cl][t];
        }
    }
}

// The caller's columns as a device table for the block walk that moves them
// itself (a graph replayed for every solve reads the columns through it):
// tab[c] = b + c*ld and tab[RBS_IO_COLS + c] = x + c*ld for c < k, NULL
// for the rest.
constexpr int RBS_IO_COLS = 128;
static __global__ void k_set_io(double **tab, const double *b, double *x, int ld, int k) {
    const int c = threadIdx.x;
    if (c >= RBS_IO_COLS) return;
    tab[c] = c < k ? const_cast<double *>(b) + (long long)c * ld : nullptr;
    tab[RBS_IO_COLS + c] = c < k ? x + (long long)c * ld : nullptr;
}

template <typename VT>
__global__ void k_fill(VT *__restrict__ v, long long count, VT value) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; t < count; t += (long long)gridDim.x * blockDim.x) v[t] = value;
}

// ---------------------------------------------------------------------------
// Diagonal-only triangle (reference method 0, utils_sptrsv_cuda.h:202-216).
// ---------------------------------------------------------------------------
template <typename VT, int K>
__global__ void k_tri_diag(const VT *__restrict__ inv, const VT *__restrict__ b, VT *x, int m) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)m * K;
    for (; t < total; t += (long long)gridDim.x * blockDim.x) {
        int p = (int)(t / K);
        st_relaxed(x + t, finalize(b[t] * inv[p]));
    }
}

// ---------------------------------------------------------------------------
// Sync-free triangle (replaces reference method 3, utils_sptrsv_cuda.h:53-114).
// Pull-style over CSR: a group of lanes owns a row, gathers its dependencies
// as they become ready and publishes x_p once.  Rows are handed out by a
// ticket counter in processing (topological) order, so every row a waiting
// group depends on is owned by a group that is already running: no
// deadlock for any grid size.  No atomics on values: results are
// deterministic.
//   K == 1: G lanes share the entries of a row (G in {1,..,32}).
//   K  > 1: R = min(K,32) lanes per row, each owns K/R right-hand sides.
// ---------------------------------------------------------------------------
template <typename VT, int K>
__global__ void __launch_bounds__(256) k_tri_syncfree(const int *__restrict__ rp, const int *__restrict__ col,
                                                      const VT *__restrict__ val, const VT *__restrict__ inv,
                                                      const VT *__restrict__ b, VT *x, int m, int G,
                                                      int *ticket, int *status, long long limit) {
    const int lane = threadIdx.x & 31;
    constexpr int R = K < 32 ? K : 32;
    constexpr int RPL = K / R;
    const int g = K == 1 ? G : R;
    const int rows_per_warp = 32 / g;
    const int sub = lane / g, sl = lane % g;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(ticket, rows_per_warp);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= m) return;
        const int row = base + sub;
        const bool active = row < m;
        if (K == 1) {
            // Reduce inside the row group only: a later group of this warp may
            // be spinning on the row this group is about to publish.
            const unsigned gmask = g == 32 ? 0xffffffffu : (((1u << g) - 1u) << (sub * g));
            VT sum = 0, bi = 0, iv = 0;
            if (active) {
                // the row's entries in aligned pairs, one vector load of two
                // values (16 bytes in FP64) and one of two columns per pair
                // and lane; an odd first entry and an odd last one alone.
                // b and the inverse diagonal are read with the row pointers:
                // after the polls (whose loads order every memory access)
                // they would add a round trip to each row
                const int s = rp[row], e = rp[row + 1];
                if (sl == 0) {
                    bi = b[row];
                    iv = inv[row];
                }
                const int p0 = s + (s & 1);
                if (sl == 0 && p0 > s && s < e) sum += val[s] * wait_value(x + col[s], status, limit);
                using V2 = Vec<VT, 2>;
                const int npair = (e - p0) / 2;
                // Two pairs per iteration: the four dependencies' first loads
                // are issued together and only a value still carrying the
                // sentinel is polled again, so a row's ready dependencies cost
                // one L2 round trip instead of one each (same summation order
                // as one pair at a time).
                int q = sl;
                for (; q + g < npair; q += 2 * g) {
                    const int k0 = p0 + 2 * q, k1 = k0 + 2 * g;
                    const int2 ca = *reinterpret_cast<const int2 *>(col + k0);
                    const int2 cb = *reinterpret_cast<const int2 *>(col + k1);
                    const V2 va = *reinterpret_cast<const V2 *>(val + k0);
                    const V2 vb = *reinterpret_cast<const V2 *>(val + k1);
                    VT xa0 = ld_relaxed(x + ca.x), xa1 = ld_relaxed(x + ca.y);
                    VT xb0 = ld_relaxed(x + cb.x), xb1 = ld_relaxed(x + cb.y);
                    if (Sent<VT>::is(xa0)) xa0 = wait_value(x + ca.x, status, limit);
                    if (Sent<VT>::is(xa1)) xa1 = wait_value(x + ca.y, status, limit);
                    if (Sent<VT>::is(xb0)) xb0 = wait_value(x + cb.x, status, limit);
                    if (Sent<VT>::is(xb1)) xb1 = wait_value(x + cb.y, status, limit);
                    sum += va.v[0] * xa0;
                    sum += va.v[1] * xa1;
                    sum += vb.v[0] * xb0;
                    sum += vb.v[1] * xb1;
                }
                if (q < npair) {
                    const int k = p0 + 2 * q;
                    const int2 c2 = *reinterpret_cast<const int2 *>(col + k);
                    const V2 v2 = *reinterpret_cast<const V2 *>(val + k);
                    VT x0 = ld_relaxed(x + c2.x), x1 = ld_relaxed(x + c2.y);
                    if (Sent<VT>::is(x0)) x0 = wait_value(x + c2.x, status, limit);
                    if (Sent<VT>::is(x1)) x1 = wait_value(x + c2.y, status, limit);
                    sum += v2.v[0] * x0;
                    sum += v2.v[1] * x1;
                }
                const int last = p0 + 2 * npair;
                if (last < e && sl == (npair % g)) sum += val[last] * wait_value(x + col[last], status, limit);
            }
            for (int off = g >> 1; off > 0; off >>= 1) sum += __shfl_down_sync(gmask, sum, off, g);
            if (active && sl == 0) st_relaxed(x + row, finalize((bi - sum) * iv));
            __syncwarp();
        } else {
            if (active) {
                VT acc[RPL], bo[RPL];
                const long long o = (long long)row * K + sl * RPL;
                const VT d = inv[row];  // read ahead of the polls, as for one column
#pragma unroll
                for (int r = 0; r < RPL; ++r) {
                    acc[r] = 0;
                    bo[r] = b[o + r];
                }
                const int s = rp[row], e = rp[row + 1];
                for (int k = s; k < e; ++k) {
                    const VT v = val[k];
                    const VT *xs = x + (long long)col[k] * K + sl * RPL;
#pragma unroll
                    for (int r = 0; r < RPL; ++r) acc[r] += v * wait_value(xs + r, status, limit);
                }
#pragma unroll
                for (int r = 0; r < RPL; ++r) st_relaxed(x + o + r, finalize((bo[r] - acc[r]) * d));
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------
// Single-CTA level-synchronous triangle (replaces reference method 2,
// utils_sptrsv_cuda.h:116-200 + the per-level launches of
// recblocking_calculate.h:68-94): one launch walks all local levels with a
// CTA barrier between levels instead of a kernel boundary.  Level l is the
// row range [lvl[l], lvl[l+1]) (or rows map[lvl[l]..lvl[l+1]) when the local
// levels are not contiguous).  gridDim.x > 1 solves independent systems
// described by `desc` (batched mode).
// ---------------------------------------------------------------------------
struct LevelDesc {
    const int *rp, *col, *lvl, *map;
    const void *val, *inv, *b;
    void *x;
    int m, nlv, G, pad;
};

template <typename VT, int K>
__global__ void __launch_bounds__(1024) k_tri_level(const LevelDesc *__restrict__ descs) {
    const LevelDesc d = descs[blockIdx.x];
    const int *__restrict__ rp = d.rp;
    const int *__restrict__ col = d.col;
    const VT *__restrict__ val = (const VT *)d.val;
    const VT *__restrict__ inv = (const VT *)d.inv;
    const VT *__restrict__ b = (const VT *)d.b;
    VT *x = (VT *)d.x;
    constexpr int R = K < 32 ? K : 32;
    constexpr int RPL = K / R;
    const int g = K == 1 ? d.G : R;
    const int lane = threadIdx.x & 31;
    const int sl = lane % g;
    const int slot = threadIdx.x / g, nslots = blockDim.x / g;
    for (int l = 0; l < d.nlv; ++l) {
        const int lo = d.lvl[l], hi = d.lvl[l + 1];
        // all lanes of a group stay together; groups never straddle warps
        for (int base = lo; base < hi; base += nslots) {
            const int idx = base + slot;
            const bool active = idx < hi;
            const int row = active ? (d.map ? d.map[idx] : idx) : 0;
            if (K == 1) {
                VT sum = 0;
                if (active) {
                    const int s = rp[row], e = rp[row + 1];
                    for (int k = s + sl; k < e; k += g) sum += val[k] * x[col[k]];
                }
                for (int off = g >> 1; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off, g);
                if (active && sl == 0) x[row] = finalize((b[row] - sum) * inv[row]);
            } else if (active) {
                VT acc[RPL];
#pragma unroll
                for (int r = 0; r < RPL; ++r) acc[r] = 0;
                const int s = rp[row], e = rp[row + 1];
                for (int k = s; k < e; ++k) {
                    const VT v = val[k];
                    const VT *xs = x + (long long)col[k] * K + sl * RPL;
#pragma unroll
                    for (int r = 0; r < RPL; ++r) acc[r] += v * xs[r];
                }
                const VT dv = inv[row];
                const long long o = (long long)row * K + sl * RPL;
#pragma unroll
                for (int r = 0; r < RPL; ++r) x[o + r] = finalize((b[o + r] - acc[r]) * dv);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Sequential triangle for deep, narrow blocks without a small bandwidth: one
// warp walks the rows in order, lanes split a row's entries; x of recent
// rows is kept in a shared-memory ring.
// ---------------------------------------------------------------------------
template <typename VT, int K>
__global__ void __launch_bounds__(32) k_tri_seq(const int *__restrict__ rp, const int *__restrict__ col,
                                                const VT *__restrict__ val, const VT *__restrict__ inv,
                                                const VT *__restrict__ b, VT *x, int m) {
    constexpr int RING = 4096 / K;
    __shared__ VT ring[RING * K];
    const int lane = threadIdx.x;
    for (int row = 0; row < m; ++row) {
        const int s = rp[row], e = rp[row + 1];
        for (int c = 0; c < K; ++c) {
            VT sum = 0;
            for (int k = s + lane; k < e; k += 32) {
                const int q = col[k];
                const VT xv = q >= row - RING ? ring[(q % RING) * K + c] : x[(long long)q * K + c];
                sum += val[k] * xv;
            }
            for (int off = 16; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off);
            if (lane == 0) {
                const VT v = finalize((b[(long long)row * K + c] - sum) * inv[row]);
                ring[(row % RING) * K + c] = v;
                x[(long long)row * K + c] = v;
            }
        }
        __syncwarp();
    }
}

// Medium rows of a square whose lane group is narrow (single RHS): rows of
// more than RBS_MEDROW entries, up to RBS_LONGROW, one warp each, summed in
// a fixed shuffle order (deterministic) -- so a few long rows no longer
// hold a narrow group for hundreds of serial steps.  `pos` lists positions
// in the row pointer (the row for CSR, the list index for DCSR).  Run by
// the first `nblk` CTAs of the square's k_spmv_sub launch (block index
// `blk`), beside the CTAs of its other rows: one launch per square, and the
// longest rows start first.
template <typename VT>
__device__ __forceinline__ void spmv_rows_warps(const int *__restrict__ rp, const int *__restrict__ col,
                                                const VT *__restrict__ val, const int *__restrict__ rows,
                                                const int *__restrict__ pos, int npos, const VT *__restrict__ x,
                                                VT *b, int blk, int nblk) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blk * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)nblk * blockDim.x) >> 5;
    for (long long t = warp; t < npos; t += nwarps) {
        const int i = pos[t];
        const int s = rp[i], e = rp[i + 1];
        VT sum = 0;
        // unrolled 16 deep: a row of up to 2048 entries has its column and
        // x loads in flight together instead of in a chain of dependent pairs
#pragma unroll 16
        for (int k = s + lane; k < e; k += 32) sum += val[k] * x[col[k]];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
        if (lane == 0) b[rows ? rows[i] : i] -= sum;
    }
}

// ---------------------------------------------------------------------------
// Square block: b[rows] -= S * x[cols]  (reference mv methods 0..3,
// utils_spmv_cuda.h:60-203, with subKernel :205-212 fused).  `rows` lists
// the rows for the DCSR form, NULL for plain CSR.  Rows longer than maxlen
// are skipped by the lane groups: those of up to 2048 entries (single RHS,
// narrow group; listed in `med`) are taken by the launch's first medctas
// CTAs, a warp each; longer ones by k_spmv_long (utils_spmv_cuda.h:30-58).
// ---------------------------------------------------------------------------
template <typename VT, int K>
__global__ void __launch_bounds__(256) k_spmv_sub(const int *__restrict__ rp, const int *__restrict__ col,
                                                  const VT *__restrict__ val, const int *__restrict__ rows,
                                                  int nrows, int G, const VT *__restrict__ x, VT *b,
                                                  int maxlen, const int *__restrict__ med, int nmed,
                                                  int medctas, int pairs) {
    if (K == 1 && (int)blockIdx.x < medctas) {  // the square's medium rows, in the same launch
        spmv_rows_warps<VT>(rp, col, val, rows, med, nmed, x, b, blockIdx.x, medctas);
        return;
    }
    constexpr int R = K < 32 ? K : 32;
    constexpr int RPL = K / R;
    const int g = K == 1 ? G : R;
    const int lane = threadIdx.x & 31;
    const int sl = lane % g, rpw = 32 / g;
    const long long bx = (long long)blockIdx.x - medctas, gx = (long long)gridDim.x - medctas;
    const long long warp = (bx * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = (gx * blockDim.x) >> 5;
    if constexpr (K == 1) {
        if (pairs) {
            // Two row groups per lane group and iteration (rows base + t and
            // base + rpw + t), their loads interleaved, so the chains of row
            // pointer, column, x and b round trips of the two rows overlap:
            // for squares whose grid is capped, where every warp loops (the
            // power-law factor's big square: 61 -> 46 us).  Each row keeps its
            // summation order (lane sl: entries sl, sl+g, ...).
            for (long long base = warp * rpw * 2; base < nrows; base += nwarps * rpw * 2) {
                const long long i0 = base + lane / g, i1 = i0 + rpw;
                int s0 = 0, e0 = 0, r0 = 0, s1 = 0, e1 = 0, r1 = 0;
                if (i0 < nrows) {
                    s0 = rp[i0];
                    e0 = rp[i0 + 1];
                    r0 = rows ? rows[i0] : (int)i0;
                    if (e0 - s0 > maxlen) e0 = s0;  // a longer row is the medium or long rows' work
                }
                if (i1 < nrows) {
                    s1 = rp[i1];
                    e1 = rp[i1 + 1];
                    r1 = rows ? rows[i1] : (int)i1;
                    if (e1 - s1 > maxlen) e1 = s1;
                }
                const int n0 = e0 - s0, n1 = e1 - s1;
                VT sum0 = 0, sum1 = 0;
#pragma unroll 4
                for (int q = sl; q < max(n0, n1); q += g) {
                    if (q < n0) sum0 += val[s0 + q] * x[col[s0 + q]];
                    if (q < n1) sum1 += val[s1 + q] * x[col[s1 + q]];
                }
                for (int off = g >> 1; off > 0; off >>= 1) {
                    sum0 += __shfl_down_sync(0xffffffffu, sum0, off, g);
                    sum1 += __shfl_down_sync(0xffffffffu, sum1, off, g);
                }
                if (sl == 0) {
                    if (n0 > 0) b[r0] -= sum0;
                    if (n1 > 0) b[r1] -= sum1;
                }
            }
        } else {
            for (long long base = warp * rpw; base < nrows; base += nwarps * rpw) {
                const long long i = base + lane / g;
                int s = 0, e = 0, row = 0;
                if (i < nrows) {
                    s = rp[i];
                    e = rp[i + 1];
                    row = rows ? rows[i] : (int)i;
                    if (e - s > maxlen) e = s;
                }
                VT sum = 0;
                // unrolled: several column loads issue before their x gathers
                // (same summation order).  Aligned pairs of entries per lane (one
                // 16-byte value load) measured no faster on the power-law factor:
                // its short rows left half of each lane group idle.
#pragma unroll 4
                for (int k = s + sl; k < e; k += g) sum += val[k] * x[col[k]];
                for (int off = g >> 1; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off, g);
                if (sl == 0 && e > s) b[row] -= sum;
            }
        }
    } else {
        for (long long base = warp * rpw; base < nrows; base += nwarps * rpw) {
            const long long i = base + lane / g;
            const bool active = i < nrows;
            int s = 0, e = 0, row = 0;
            if (active) {
                s = rp[i];
                e = rp[i + 1];
                row = rows ? rows[i] : (int)i;
                if (e - s > maxlen) e = s;  // a longer row is another kernel's
            }
            if (active && e > s) {
                VT acc[RPL];
#pragma unroll
                for (int r = 0; r < RPL; ++r) acc[r] = 0;
                for (int k = s; k < e; ++k) {
                    const VT v = val[k];
                    const VT *xs = x + (long long)col[k] * K + sl * RPL;
#pragma unroll
                    for (int r = 0; r < RPL; ++r) acc[r] += v * xs[r];
                }
                const long long o = (long long)row * K + sl * RPL;
#pragma unroll
                for (int r = 0; r < RPL; ++r) b[o + r] -= acc[r];
            }
        }
    }
}

// Long rows: each warp takes a 32*8-entry slice of one long row and
// accumulates into b with atomics (the only atomics of the solve; their
// order varies, so long-row results can differ in the last bits between
// runs).
template <typename VT, int K>
__global__ void __launch_bounds__(256) k_spmv_long(const int *__restrict__ rp, const int *__restrict__ col,
                                                   const VT *__restrict__ val, const int *__restrict__ rows,
                                                   const int *__restrict__ longpos, int nlong,
                                                   const VT *__restrict__ x, VT *b) {
    constexpr int SLICE = 256;
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (int li = 0; li < nlong; ++li) {
        const int pos = longpos[li];  // index into rp (the row itself for plain CSR)
        const int row = rows ? rows[pos] : pos;
        const int s = rp[pos], e = rp[pos + 1];
        const long long nslices = (e - s + SLICE - 1) / SLICE;
        for (long long w = warp; w < nslices; w += nwarps) {
            const int ss = s + (int)w * SLICE, se = min(e, ss + SLICE);
            for (int c = 0; c < K; ++c) {
                VT sum = 0;
                for (int k = ss + lane; k < se; k += 32) sum += val[k] * x[(long long)col[k] * K + c];
                for (int off = 16; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off);
                if (lane == 0) atomicAdd(b + (long long)row * K + c, -sum);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Mixed precision: r32 = (float)(b - A x) with FP64 A, x, b (full
// processing-order CSR including the diagonal).
// ---------------------------------------------------------------------------
template <int K>
__global__ void __launch_bounds__(256) k_residual(const int *__restrict__ rp, const int *__restrict__ col,
                                                  const double *__restrict__ val, const double *__restrict__ x,
                                                  const double *__restrict__ b, float *__restrict__ r32, int n,
                                                  int G) {
    constexpr int R = K < 32 ? K : 32;
    constexpr int RPL = K / R;
    const int g = K == 1 ? G : R;
    const int lane = threadIdx.x & 31;
    const int sl = lane % g, rpw = 32 / g;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * rpw; base < n; base += nwarps * rpw) {
        const long long row = base + lane / g;
        const bool active = row < n;
        if (K == 1) {
            double sum = 0;
            if (active)
                for (int k = rp[row] + sl; k < rp[row + 1]; k += g) sum += val[k] * x[col[k]];
            for (int off = g >> 1; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off, g);
            if (active && sl == 0) r32[row] = (float)(b[row] - sum);
        } else if (active) {
            double acc[RPL];
#pragma unroll
            for (int r = 0; r < RPL; ++r) acc[r] = 0;
            for (int k = rp[row]; k < rp[row + 1]; ++k) {
                const double v = val[k];
                const double *xs = x + (long long)col[k] * K + sl * RPL;
#pragma unroll
                for (int r = 0; r < RPL; ++r) acc[r] += v * xs[r];
            }
            const long long o = row * K + sl * RPL;
#pragma unroll
            for (int r = 0; r < RPL; ++r) r32[o + r] = (float)(b[o + r] - acc[r]);
        }
    }
}

// x64 (+)= d32; d32 reset to the sentinel; per-column sums of squares of the
// correction and of the updated solution accumulated into norms[2*K].
template <int K>
__global__ void __launch_bounds__(256) k_update(double *__restrict__ x64, float *__restrict__ d32, int n, int first,
                                                double *__restrict__ norms) {
    // blockDim (256) and the grid stride are multiples of K, so a thread
    // always works on the same right-hand side c.
    __shared__ double sd[2 * K];
    for (int i = threadIdx.x; i < 2 * K; i += blockDim.x) sd[i] = 0;
    __syncthreads();
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)n * K;
    const int c = (int)(t % K);
    double dd = 0, xx = 0;
    for (; t < total; t += (long long)gridDim.x * blockDim.x) {
        const double d = (double)d32[t];
        const double xn = first ? d : x64[t] + d;
        x64[t] = xn;
        d32[t] = __uint_as_float(RBS_SENT32);
        dd += d * d;
        xx += xn * xn;
    }
    atomicAdd(&sd[c], dd);
    atomicAdd(&sd[K + c], xx);
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * K; i += blockDim.x) atomicAdd(&norms[i], sd[i]);
}

// x[perm[p] + c*ld] = x64[p*K + c]
template <int K>
__global__ void k_scatter64(const double *__restrict__ x64, const int *__restrict__ perm, int n, int k, double *x,
                            int ld) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)n * K;
    for (; t < total; t += (long long)gridDim.x * blockDim.x) {
        int p = (int)(t / K), c = (int)(t % K);
        if (c < k) x[(long long)c * ld + perm[p]] = x64[t];
    }
}

// cols[c][perm[p]] = x64[p*K + c] for c < k (column-pointer table form)
template <int K>
__global__ void k_scatter64_cols(const double *__restrict__ x64, const int *__restrict__ perm, int n, int k,
                                 double *const *__restrict__ cols) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)n * K;
    for (; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(t / K), c = (int)(t % K);
        if (c < k) cols[c][perm[p]] = x64[t];
    }
}

// ---------------------------------------------------------------------------
// Grouped work vectors (column group g of G columns: its rows contiguous, G
// values each; groups gstride elements apart).  Pointers are those of group
// 0 at the block's first row (or column).
// ---------------------------------------------------------------------------
template <typename VT, int G>
__global__ void k_tri_diag_grp(const VT *__restrict__ inv, const VT *__restrict__ b, VT *x, int m, int ngroups,
                               long long gstride) {
    const long long per = (long long)m * G, total = per * ngroups;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long g = t / per, rest = t - g * per;
        const long long o = g * gstride + rest;
        x[o] = finalize(b[o] * inv[rest / G]);
    }
}

// b[rows] -= S x[cols]: one thread per (row, group), consecutive threads on
// consecutive rows of one group.
template <typename VT, int G>
__global__ void __launch_bounds__(256) k_spmv_sub_grp(const int *__restrict__ rp, const int *__restrict__ col,
                                                      const VT *__restrict__ val, const int *__restrict__ rows,
                                                      int nrows, int ngroups, long long gstride,
                                                      const VT *__restrict__ x, VT *b) {
    using VG = Vec<VT, G>;
    const long long total = (long long)nrows * ngroups;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long g = t / nrows;
        const int i = (int)(t - g * nrows);
        const int s = rp[i], e = rp[i + 1];
        if (e == s) continue;
        const int row = rows ? rows[i] : i;
        const VT *xg = x + g * gstride;
        VT acc[G];
#pragma unroll
        for (int j = 0; j < G; ++j) acc[j] = 0;
        for (int k = s; k < e; ++k) {
            const VT v = val[k];
            const VG xv = *reinterpret_cast<const VG *>(xg + (long long)col[k] * G);
#pragma unroll
            for (int j = 0; j < G; ++j) acc[j] += v * xv.v[j];
        }
        VG *bp = reinterpret_cast<VG *>(b + g * gstride + (long long)row * G);
        VG bv = *bp;
#pragma unroll
        for (int j = 0; j < G; ++j) bv.v[j] -= acc[j];
        *bp = bv;
    }
}

// Mixed precision, grouped: r32 = (float)(b - A x), one thread per (row, group).
template <int G>
__global__ void __launch_bounds__(256) k_residual_grp(const int *__restrict__ rp, const int *__restrict__ col,
                                                      const double *__restrict__ val, const double *__restrict__ x,
                                                      const double *__restrict__ b, float *__restrict__ r32, int n,
                                                      int ngroups, long long gstride) {
    using VG = Vec<double, G>;
    const long long total = (long long)n * ngroups;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long g = t / n;
        const int row = (int)(t - g * n);
        const double *xg = x + g * gstride;
        double acc[G];
#pragma unroll
        for (int j = 0; j < G; ++j) acc[j] = 0;
        for (int k = rp[row]; k < rp[row + 1]; ++k) {
            const double v = val[k];
            const VG xv = *reinterpret_cast<const VG *>(xg + (long long)col[k] * G);
#pragma unroll
            for (int j = 0; j < G; ++j) acc[j] += v * xv.v[j];
        }
        const long long o = g * gstride + (long long)row * G;
        const VG bv = *reinterpret_cast<const VG *>(b + o);
#pragma unroll
        for (int j = 0; j < G; ++j) r32[o + j] = (float)(bv.v[j] - acc[j]);
    }
}

// Mixed precision, grouped: x64 (+)= d32, d32 reset to the sentinel, per-column
// sums of squares into norms[2*K].  Column c = blockIdx.y.
template <int K, int G>
__global__ void __launch_bounds__(256) k_update_grp(double *__restrict__ x64, float *__restrict__ d32, int n,
                                                    int first, double *__restrict__ norms) {
    __shared__ double red[2][8];
    const int c = blockIdx.y;
    const long long base = (long long)(c / G) * n * G + (c % G);
    double dd = 0, xx = 0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const long long o = base + p * G;
        const double d = (double)d32[o];
        const double xn = first ? d : x64[o] + d;
        x64[o] = xn;
        d32[o] = __uint_as_float(RBS_SENT32);
        dd += d * d;
        xx += xn * xn;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        dd += __shfl_down_sync(0xffffffffu, dd, off);
        xx += __shfl_down_sync(0xffffffffu, xx, off);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = dd;
        red[1][w] = xx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, z = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            a += red[0][q];
            z += red[1][q];
        }
        atomicAdd(&norms[c], a);
        atomicAdd(&norms[K + c], z);
    }
}

}  // namespace rbs
