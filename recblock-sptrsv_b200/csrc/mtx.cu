// mtx.cu -- Matrix Market coordinate files read onto the device: the
// reference's mmio_info / mmio_data (mmio_highlevel.h:7-296) and the
// driver's triangle extraction and CSR->CSC transposition (main.cu:151-236,
// tranpose.h:7-54), with the per-entry work on the GPU.
//
// The host parses the banner and the size line (mm_read_banner,
// mm_read_mtx_crd_size: mmio.h:254-367) and streams the entry bytes to HBM
// through a ring of pinned buffers.  On the device:
//   tokens   each 8 KB tile counts its token starts (a non-space byte after a
//            space), a scan over tiles numbers them, and every entry records
//            the byte offset of its first token -- fscanf's whitespace-
//            separated reading, independent of line structure;
//   entries  one thread per entry converts its tokens (indices as C ints,
//            values correctly rounded, mtx_parse.cuh); values outside the
//            exact window go to strtod on the host and are scattered back;
//   CSR      symmetric and Hermitian files emit the mirrored entry right
//            after the entry (diagonal once), and a stable radix sort of the
//            expanded sequence by row gives mmio_data's layout exactly:
//            rows ascending, file order inside a row;
//   triangle a scan of the strictly-lower (upper) flags places every entry
//            and the unit diagonal of main.cu:157-198's triangle, and a
//            stable sort by column gives tranpose.h's CSC.
// Integer results are bit-identical to the reference's; values are the
// bits fscanf("%lg") produces.
#include <cuda_runtime.h>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "mtx_parse.cuh"
#include "rbs.h"
#include "rbs_internal.h"

namespace rbs {

namespace {

#define MCK(call)                                                                       \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            err = std::string("Matrix Market reader: ") + #call + ": " + cudaGetErrorString(e_); \
            return RBS_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

constexpr int TOK_T = 256;                       // threads per tile
constexpr int TOK_B = 32;                        // bytes per thread
constexpr long long TOK_TILE = TOK_T * TOK_B;    // bytes per tile
constexpr long long CHUNK = 32LL << 20;          // host read / copy granule
constexpr int NRING = 3;                         // pinned staging buffers
constexpr int SLOT = 64;                         // bytes per value token handed to the host
constexpr int SLOT_TEXT = SLOT - 2;              // token characters held in a slot

enum { MTX_BAD_TOKEN = 1, MTX_OUT_OF_RANGE = 2 };

cudaError_t pool_for(int dev, cudaMemPool_t &pool) { return device_mem_pool(dev, pool); }

struct Buf {  // temporaries of one call, stream-ordered on st
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;
    std::vector<void *> ptrs;
    ~Buf() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
    }
    template <typename T>
    cudaError_t get(T *&p, size_t count) {
        void *q = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&q, std::max<size_t>(count, 1) * sizeof(T), pool, st);
        if (e == cudaSuccess) {
            ptrs.push_back(q);
            p = static_cast<T *>(q);
        }
        return e;
    }
};

int bits_for(long long n) {
    int b = 1;
    while (b < 31 && (1LL << b) < n) ++b;
    return b;
}

int grid_for(long long n, int threads, int sms) {
    const long long g = (n + threads - 1) / threads;
    return (int)std::max<long long>(1, std::min<long long>(g, (long long)sms * 16));
}

// ---------------------------------------------------------------- kernels

// bit j of the result: byte j of w is a C-locale space (' ', \t..\r)
__device__ __forceinline__ unsigned space4(unsigned w) {
    const unsigned sp = __vcmpeq4(w, 0x20202020u) | __vcmpltu4(__vsub4(w, 0x09090909u), 0x05050505u);
    // 0x00/0xFF bytes -> 4 bits: the top bit of byte j lands on bit 28 + j
    return ((sp & 0x80808080u) * 0x00204081u) >> 28;
}

// bit j set: byte p0 + j starts a token.  The buffer is padded with spaces
// to whole tiles, so bytes at or beyond len are spaces already.
__device__ __forceinline__ unsigned start_mask(const unsigned char *__restrict__ s, long long len, long long p0) {
    if (p0 >= len) return 0;
    const unsigned prev_space = (p0 == 0 || mtxp::is_space(s[p0 - 1])) ? 1u : 0u;
    const uint4 a = *reinterpret_cast<const uint4 *>(s + p0);
    const uint4 b = *reinterpret_cast<const uint4 *>(s + p0 + 16);
    const unsigned sp = space4(a.x) | space4(a.y) << 4 | space4(a.z) << 8 | space4(a.w) << 12 | space4(b.x) << 16 |
                        space4(b.y) << 20 | space4(b.z) << 24 | space4(b.w) << 28;
    return ~sp & ((sp << 1) | prev_space);
}

__global__ void __launch_bounds__(TOK_T) k_tok_count(const unsigned char *__restrict__ s, long long len,
                                                      long long *tile_cnt) {
    const long long p0 = (long long)blockIdx.x * TOK_TILE + (long long)threadIdx.x * TOK_B;
    typedef cub::BlockReduce<int, TOK_T> R;
    __shared__ typename R::TempStorage tmp;
    const int tot = R(tmp).Sum(__popc(start_mask(s, len, p0)));
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

// offset of the first token of every entry (tokens_per_entry tokens each)
__global__ void __launch_bounds__(TOK_T) k_tok_mark(const unsigned char *__restrict__ s, long long len,
                                                     const long long *__restrict__ tile_off, int tpe, long long nz,
                                                     long long *entry_pos) {
    const long long p0 = (long long)blockIdx.x * TOK_TILE + (long long)threadIdx.x * TOK_B;
    unsigned mask = start_mask(s, len, p0);
    typedef cub::BlockScan<int, TOK_T> S;
    __shared__ typename S::TempStorage tmp;
    int before = 0;
    S(tmp).ExclusiveSum(__popc(mask), before);
    if (!mask) return;
    const long long t = tile_off[blockIdx.x] + before;
    long long q = t / tpe;  // entry of this thread's first token
    int r = (int)(t - q * tpe);  // its place inside the entry
    while (mask && q < nz) {
        const int j = __ffs(mask) - 1;
        mask &= mask - 1;
        if (r == 0) entry_pos[q] = p0 + j;
        if (++r == tpe) {
            r = 0;
            ++q;
        }
    }
}

__device__ __forceinline__ long long skip_space(const unsigned char *s, long long len, long long p) {
    while (p < len && mtxp::is_space(s[p])) ++p;
    return p;
}

constexpr int ENT_T = 256;          // entries per CTA
constexpr int ENT_SMEM = 24576;     // bytes of their text staged in shared memory

// One entry per thread: 0-based row and column, value, the mirror flag of
// symmetric files, and the value token's offset when the host converts it.
// A CTA's 256 consecutive entries occupy one contiguous stretch of text,
// loaded into shared memory with 16-byte coalesced loads (parsed from global
// memory instead when the stretch is longer than the buffer).
__global__ void __launch_bounds__(ENT_T) k_entries(const unsigned char *__restrict__ s, long long len,
                                                   const long long *__restrict__ entry_pos, long long nz, int field,
                                                   int symmetric, int m, int n, int *row, int *col, double *val,
                                                   int *mirror, unsigned char *host_flag, long long *vpos,
                                                   int *status, unsigned long long *bad_entry) {
    __shared__ __align__(16) unsigned char text[ENT_SMEM];
    const long long e0 = (long long)blockIdx.x * ENT_T;
    const long long e = e0 + threadIdx.x;
    const long long last = e0 + ENT_T < nz ? e0 + ENT_T : nz;
    const long long start = entry_pos[e0] & ~15LL;  // the buffer base is 256-byte aligned
    const long long stop = last < nz ? entry_pos[last] : len;
    const long long wlen = stop - start;
    const bool staged = wlen <= ENT_SMEM;
    if (staged) {
        // up to 15 bytes past stop: inside the tile-padded buffer
        const int nvec = (int)((wlen + 15) >> 4);
        const uint4 *src = reinterpret_cast<const uint4 *>(s + start);
        for (int i = threadIdx.x; i < nvec; i += ENT_T) reinterpret_cast<uint4 *>(text)[i] = src[i];
    }
    __syncthreads();
    if (e >= nz) return;
    const unsigned char *b = staged ? text : s + start;
    const long long blen = staged ? wlen : len - start;
    long long p = entry_pos[e] - start, end = p;
    int r = 0, c = 0, fl = 0, hf = 0;
    double v = 1.0;
    if (mtxp::parse_int(b, blen, p, r, end) != mtxp::PARSE_OK) {
        fl = MTX_BAD_TOKEN;
    } else {
        p = skip_space(b, blen, end);
        if (mtxp::parse_int(b, blen, p, c, end) != mtxp::PARSE_OK) {
            fl = MTX_BAD_TOKEN;
        } else if (field == RBS_MTX_REAL || field == RBS_MTX_COMPLEX) {
            p = skip_space(b, blen, end);
            if (mtxp::parse_real(b, blen, p, v, end) != mtxp::PARSE_OK) {
                hf = 1;
                vpos[e] = start + p;
                v = 0.0;
            }
        } else if (field == RBS_MTX_INTEGER) {
            p = skip_space(b, blen, end);
            int iv = 0;
            if (mtxp::parse_int(b, blen, p, iv, end) != mtxp::PARSE_OK) fl = MTX_BAD_TOKEN;
            v = (double)iv;
        }
    }
    if (!fl && (r < 1 || r > m || c < 1 || c > n)) fl = MTX_OUT_OF_RANGE;
    if (fl) {
        atomicOr(status, fl);
        atomicMin(bad_entry, (unsigned long long)e);
    }
    row[e] = r - 1;
    col[e] = c - 1;
    val[e] = v;
    mirror[e] = (symmetric && r != c) ? 1 : 0;
    host_flag[e] = (unsigned char)hf;
}

// the value tokens the host converts, one slot each: text (NUL-terminated,
// at most SLOT_TEXT characters) and, in the last byte, 1 when the token is
// longer than that
__global__ void k_gather_tokens(const unsigned char *__restrict__ s, long long len, const int *__restrict__ fidx,
                                int h, const long long *__restrict__ vpos, unsigned char *slots) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < h; i += gridDim.x * blockDim.x) {
        const long long p = vpos[fidx[i]];
        unsigned char *o = slots + (size_t)i * SLOT;
        int k = 0;
        while (k < SLOT_TEXT && p + k < len && !mtxp::is_space(s[p + k])) {
            o[k] = s[p + k];
            ++k;
        }
        o[k] = 0;
        o[SLOT - 1] = (p + k < len && !mtxp::is_space(s[p + k])) ? 1 : 0;
    }
}

__global__ void k_scatter_values(const int *__restrict__ fidx, int h, const double *__restrict__ hv, double *val) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < h; i += gridDim.x * blockDim.x) val[fidx[i]] = hv[i];
}

// expanded sequence: entry e at e + mirrors before it, its mirror right after
__global__ void k_expand(const int *__restrict__ row, const int *__restrict__ col, const int *__restrict__ moff,
                         long long nz, int *keys, unsigned *codes) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nz;
         e += (long long)gridDim.x * blockDim.x) {
        const long long b = e + moff[e];
        keys[b] = row[e];
        codes[b] = (unsigned)(2 * e);
        if (moff[e + 1] != moff[e]) {
            keys[b + 1] = col[e];
            codes[b + 1] = (unsigned)(2 * e + 1);
        }
    }
}

// CSR columns and values from the sorted codes; counts of strictly lower
// and strictly upper entries
__global__ void k_fill(const unsigned *__restrict__ codes, const int *__restrict__ rowof, const int *__restrict__ row,
                       const int *__restrict__ col, const double *__restrict__ v, long long cnt, int *colidx,
                       double *val, unsigned long long *lower_upper) {
    unsigned long long lo = 0, up = 0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < cnt;
         p += (long long)gridDim.x * blockDim.x) {
        const unsigned code = codes[p];
        const unsigned e = code >> 1;
        const int c = (code & 1) ? row[e] : col[e];
        colidx[p] = c;
        val[p] = v[e];
        lo += c < rowof[p];
        up += c > rowof[p];
    }
    typedef cub::BlockReduce<unsigned long long, 256> R;
    __shared__ typename R::TempStorage t1, t2;
    lo = R(t1).Sum(lo);
    up = R(t2).Sum(up);
    if (threadIdx.x == 0) {
        atomicAdd(lower_upper, lo);
        atomicAdd(lower_upper + 1, up);
    }
}

// ptr[r] = first position whose sorted key is >= r, for r in [0, rows]
__global__ void k_ptr_from_keys(const int *__restrict__ keys, long long cnt, int rows, int *ptr) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p <= cnt;
         p += (long long)gridDim.x * blockDim.x) {
        const int prev = p == 0 ? -1 : keys[p - 1];
        const int cur = p == cnt ? rows : keys[p];
        for (int r = prev + 1; r <= cur; ++r) ptr[r] = (int)p;
    }
}

__global__ void k_strict_flags(const int *__restrict__ rowof, const int *__restrict__ colidx, long long cnt,
                               int forward, int *flag) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p <= cnt;
         p += (long long)gridDim.x * blockDim.x)
        flag[p] = p == cnt ? 0 : (forward ? colidx[p] < rowof[p] : colidx[p] > rowof[p]);
}

// the triangle of main.cu:157-198 in CSR: row i holds its strict entries in
// A's order, then (forward) or before them (backward) the unit diagonal;
// strict entry of rank r gets strict_val[r] when given, else A's value
__global__ void k_tri_scatter(const int *__restrict__ rowof, const int *__restrict__ colidx,
                              const double *__restrict__ val, const int *__restrict__ flag,
                              const int *__restrict__ srank, long long cnt, int forward,
                              const double *__restrict__ strict_val, int *tidx, double *tval, int *trow) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < cnt;
         p += (long long)gridDim.x * blockDim.x) {
        if (!flag[p]) continue;
        const int i = rowof[p], r = srank[p];
        const long long pos = (long long)r + i + (forward ? 0 : 1);
        tidx[pos] = colidx[p];
        tval[pos] = strict_val ? strict_val[r] : val[p];
        if (trow) trow[pos] = i;
    }
}

__global__ void k_tri_rows(const int *__restrict__ rowptr, const int *__restrict__ srank, int m, int forward,
                           int *tptr, int *tidx, double *tval, int *trow) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += gridDim.x * blockDim.x) {
        const int start = srank[rowptr[i]] + i;
        tptr[i] = start;
        if (i == m) continue;
        // diagonal: last of row i (forward) or first (backward)
        const int pos = forward ? srank[rowptr[i + 1]] + i : start;
        tidx[pos] = i;
        tval[pos] = 1.0;
        if (trow) trow[pos] = i;
    }
}

__global__ void k_iota(int *v, long long cnt) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < cnt;
         p += (long long)gridDim.x * blockDim.x)
        v[p] = (int)p;
}

__global__ void k_gather_csc(const int *__restrict__ perm, const int *__restrict__ trow,
                             const double *__restrict__ tval, long long cnt, int *idx, double *val) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < cnt;
         p += (long long)gridDim.x * blockDim.x) {
        const int q = perm[p];
        idx[p] = trow[q];
        val[p] = tval[q];
    }
}

// ------------------------------------------------------------------- host

struct Header {
    int m = 0, n = 0;
    long long nz = 0;
    int field = RBS_MTX_REAL, symmetric = 0;
    long long data_off = 0;
};

// Banner and size line from the first avail bytes (whole: avail is the
// whole file).  Returns RBS_OK, an error code, or -1 when more bytes are
// needed.  Same acceptance as mm_read_banner (mmio.h:254-331): five
// tokens, the banner prefix, "matrix", and a known field and symmetry.
int parse_header(const char *b, long long avail, bool whole, Header &h, std::string &err) {
    long long pos = 0;
    int line_no = 0;
    while (true) {
        if (pos >= avail) {
            if (whole) {
                err = line_no == 0 ? "Matrix Market reader: empty file" : "Matrix Market reader: no size line";
                return RBS_ERR_ARG;
            }
            return -1;
        }
        const char *nl = static_cast<const char *>(memchr(b + pos, '\n', (size_t)(avail - pos)));
        if (!nl && !whole) return -1;
        const long long end = nl ? nl - b : avail;
        const std::string line(b + pos, (size_t)(end - pos));
        const long long next = nl ? end + 1 : avail;
        ++line_no;
        if (line_no == 1) {
            char t[5][64] = {{0}};
            if (sscanf(line.c_str(), "%63s %63s %63s %63s %63s", t[0], t[1], t[2], t[3], t[4]) != 5 ||
                strncmp(t[0], "%%MatrixMarket", 14) != 0) {
                err = "Matrix Market reader: could not process the banner";
                return RBS_ERR_ARG;
            }
            for (int k = 1; k < 5; ++k)
                for (char *q = t[k]; *q; ++q) *q = (char)tolower((unsigned char)*q);
            if (strcmp(t[1], "matrix") != 0) {
                err = "Matrix Market reader: banner object is not 'matrix'";
                return RBS_ERR_ARG;
            }
            if (strcmp(t[2], "coordinate") != 0) {
                err = std::string("Matrix Market reader: '") + t[2] + "' storage is not read (coordinate only)";
                return RBS_ERR_UNSUPPORTED;
            }
            if (!strcmp(t[3], "real")) h.field = RBS_MTX_REAL;
            else if (!strcmp(t[3], "integer")) h.field = RBS_MTX_INTEGER;
            else if (!strcmp(t[3], "pattern")) h.field = RBS_MTX_PATTERN;
            else if (!strcmp(t[3], "complex")) h.field = RBS_MTX_COMPLEX;
            else {
                err = std::string("Matrix Market reader: unknown field '") + t[3] + "'";
                return RBS_ERR_UNSUPPORTED;
            }
            if (!strcmp(t[4], "symmetric") || !strcmp(t[4], "hermitian")) h.symmetric = 1;
            else if (!strcmp(t[4], "general") || !strcmp(t[4], "skew-symmetric")) h.symmetric = 0;
            else {
                err = std::string("Matrix Market reader: unknown symmetry '") + t[4] + "'";
                return RBS_ERR_UNSUPPORTED;
            }
        } else if (!line.empty() && line[0] == '%') {
            // comment
        } else {
            int m = 0, n = 0;
            long long nz = 0;
            if (sscanf(line.c_str(), "%d %d %lld", &m, &n, &nz) == 3) {
                if (m < 0 || n < 0 || nz < 0 || nz > 0x7fffffffLL) {
                    err = "Matrix Market reader: size line out of range";
                    return RBS_ERR_ARG;
                }
                h.m = m;
                h.n = n;
                h.nz = nz;
                h.data_off = next;
                return RBS_OK;
            }
            bool blank = true;
            for (char c : line) blank = blank && isspace((unsigned char)c);
            if (!blank) {
                err = "Matrix Market reader: malformed size line";
                return RBS_ERR_ARG;
            }
        }
        pos = next;
    }
}

// Source of the entry bytes: a file descriptor or a host buffer.
struct Source {
    int fd = -1;
    const unsigned char *buf = nullptr;
    long long size = 0;
    bool read(long long off, long long n, void *dst) const {
        if (buf) {
            memcpy(dst, buf + off, (size_t)n);
            return true;
        }
        char *d = static_cast<char *>(dst);
        while (n > 0) {
            const ssize_t r = pread(fd, d, (size_t)n, (off_t)off);
            if (r <= 0) return false;
            d += r;
            off += r;
            n -= r;
        }
        return true;
    }
};

// one chunk read by several host threads (page-cache copies scale with
// threads; the device copy of the previous chunk runs meanwhile)
bool read_parallel(const Source &src, long long off, long long n, unsigned char *dst) {
    const int P = n >= (4LL << 20) ? (int)std::min(8u, host_threads()) : 1;
    if (P == 1) return src.read(off, n, dst);
    std::vector<char> ok((size_t)P, 1);
    std::vector<std::thread> th;
    for (int t = 0; t < P; ++t) {
        const long long lo = n * t / P, hi = n * (t + 1) / P;
        th.emplace_back([&, t, lo, hi] { ok[(size_t)t] = src.read(off + lo, hi - lo, dst + lo); });
    }
    for (auto &x : th) x.join();
    for (char c : ok)
        if (!c) return false;
    return true;
}

// process-wide pinned staging ring (one reader at a time)
std::mutex g_ring_mu;
unsigned char *g_ring[NRING] = {nullptr, nullptr, nullptr};
cudaEvent_t g_ring_ev[NRING];
int g_ring_dev = -1;

int ring_get(int dev, std::string &err) {
    if (g_ring[0] && g_ring_dev == dev) return RBS_OK;
    if (g_ring[0]) {
        for (int k = 0; k < NRING; ++k) {
            cudaFreeHost(g_ring[k]);
            cudaEventDestroy(g_ring_ev[k]);
            g_ring[k] = nullptr;
        }
    }
    for (int k = 0; k < NRING; ++k) {
        MCK(cudaHostAlloc(reinterpret_cast<void **>(&g_ring[k]), (size_t)CHUNK, cudaHostAllocDefault));
        MCK(cudaEventCreateWithFlags(&g_ring_ev[k], cudaEventDisableTiming));
    }
    g_ring_dev = dev;
    return RBS_OK;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int read_impl(const Source &src, const rbs_options &opt, DeviceMtx &M, std::string &err) {
    const auto t0 = std::chrono::steady_clock::now();
    // header: grow the prefix until the size line is in it
    Header h;
    {
        long long want = std::min<long long>(src.size, 1 << 16);
        std::vector<char> pre;
        while (true) {
            pre.resize((size_t)want);
            if (want && !src.read(0, want, pre.data())) {
                err = "Matrix Market reader: read error";
                return RBS_ERR_ARG;
            }
            const int rc = parse_header(pre.data(), want, want == src.size, h, err);
            if (rc == RBS_OK) break;
            if (rc > 0) return rc;
            want = std::min<long long>(src.size, want * 4);
        }
    }
    M.m = h.m;
    M.n = h.n;
    M.nnz_file = h.nz;
    M.field = h.field;
    M.symmetric = h.symmetric;
    M.host_values = 0;
    const int tpe = h.field == RBS_MTX_PATTERN ? 2 : h.field == RBS_MTX_COMPLEX ? 4 : 3;

    if (opt.device >= 0) MCK(cudaSetDevice(opt.device));
    int dev = 0, sms = 148;
    MCK(cudaGetDevice(&dev));
    MCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    M.device = dev;
    cudaStream_t st = nullptr;
    MCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } sg{st};
    Buf buf;
    buf.st = st;
    MCK(pool_for(dev, buf.pool));

    // entry bytes to HBM, padded with spaces to whole tiles
    const long long len = src.size - h.data_off;
    const long long ntiles = (len + TOK_TILE - 1) / TOK_TILE;
    unsigned char *ds = nullptr;
    MCK(buf.get(ds, (size_t)std::max<long long>(ntiles, 1) * TOK_TILE));
    {
        std::lock_guard<std::mutex> lk(g_ring_mu);
        const int rc = ring_get(dev, err);
        if (rc) return rc;
        bool used[NRING] = {false, false, false};
        int k = 0;
        for (long long off = 0; off < len; off += CHUNK, k = (k + 1) % NRING) {
            const long long nb = std::min(CHUNK, len - off);
            if (used[k]) MCK(cudaEventSynchronize(g_ring_ev[k]));
            if (!read_parallel(src, h.data_off + off, nb, g_ring[k])) {
                err = "Matrix Market reader: read error";
                cudaStreamSynchronize(st);
                return RBS_ERR_ARG;
            }
            MCK(cudaMemcpyAsync(ds + off, g_ring[k], (size_t)nb, cudaMemcpyHostToDevice, st));
            MCK(cudaEventRecord(g_ring_ev[k], st));
            used[k] = true;
        }
        if (ntiles * TOK_TILE > len) MCK(cudaMemsetAsync(ds + len, ' ', (size_t)(ntiles * TOK_TILE - len), st));
        MCK(cudaStreamSynchronize(st));
    }
    M.read_ms = ms_since(t0);
    const auto t1 = std::chrono::steady_clock::now();
    const long long nz = h.nz;

    // token starts -> first-token offset of every entry
    long long *tile_cnt = nullptr, *tile_off = nullptr, *entry_pos = nullptr;
    MCK(buf.get(tile_cnt, (size_t)ntiles + 1));
    MCK(buf.get(tile_off, (size_t)ntiles + 1));
    MCK(buf.get(entry_pos, (size_t)nz));
    MCK(cudaMemsetAsync(tile_cnt, 0, sizeof(long long) * ((size_t)ntiles + 1), st));
    if (ntiles) {
        k_tok_count<<<(unsigned)ntiles, TOK_T, 0, st>>>(ds, len, tile_cnt);
        MCK(cudaGetLastError());
    }
    {
        size_t tmp = 0;
        MCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, tile_cnt, tile_off, (long long)ntiles + 1, st));
        void *t = nullptr;
        MCK(buf.get(reinterpret_cast<char *&>(t), tmp));
        MCK(cub::DeviceScan::ExclusiveSum(t, tmp, tile_cnt, tile_off, (long long)ntiles + 1, st));
    }
    long long ntok = 0;
    MCK(cudaMemcpyAsync(&ntok, tile_off + ntiles, sizeof(long long), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    if (ntok < nz * tpe) {
        err = "Matrix Market reader: truncated file: " + std::to_string(nz) + " entries announced, " +
              std::to_string(ntok / tpe) + " present";
        return RBS_ERR_ARG;
    }
    if (ntiles) {
        k_tok_mark<<<(unsigned)ntiles, TOK_T, 0, st>>>(ds, len, tile_off, tpe, nz, entry_pos);
        MCK(cudaGetLastError());
    }

    // entries
    int *row = nullptr, *col = nullptr, *mir = nullptr, *moff = nullptr, *status = nullptr;
    double *v = nullptr;
    unsigned char *hflag = nullptr;
    long long *vpos = nullptr;
    unsigned long long *bad = nullptr;
    MCK(buf.get(row, (size_t)nz));
    MCK(buf.get(col, (size_t)nz));
    MCK(buf.get(v, (size_t)nz));
    MCK(buf.get(mir, (size_t)nz + 1));
    MCK(buf.get(moff, (size_t)nz + 1));
    MCK(buf.get(hflag, (size_t)nz));
    MCK(buf.get(vpos, (size_t)nz));
    MCK(buf.get(status, 4));
    bad = reinterpret_cast<unsigned long long *>(status + 2);
    MCK(cudaMemsetAsync(status, 0, sizeof(int) * 2, st));
    MCK(cudaMemsetAsync(bad, 0xff, sizeof(unsigned long long), st));
    MCK(cudaMemsetAsync(mir + nz, 0, sizeof(int), st));
    if (nz) {
        k_entries<<<(unsigned)((nz + ENT_T - 1) / ENT_T), ENT_T, 0, st>>>(ds, len, entry_pos, nz, h.field,
                                                                         h.symmetric, h.m, h.n,
                                                          row, col, v, mir, hflag, vpos, status, bad);
        MCK(cudaGetLastError());
    }
    int hstat[2] = {0, 0};
    unsigned long long hbad = 0;
    MCK(cudaMemcpyAsync(hstat, status, sizeof(hstat), cudaMemcpyDeviceToHost, st));
    MCK(cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    if (hstat[0]) {
        err = "Matrix Market reader: entry " + std::to_string(hbad + 1) +
              ((hstat[0] & MTX_BAD_TOKEN) ? " is malformed" : " has an index out of range") + " (first such entry)";
        if (!(hstat[0] & MTX_BAD_TOKEN)) return RBS_ERR_STRUCTURE;
        return RBS_ERR_ARG;
    }

    // values outside the exact window: strtod on the host
    if (nz && (h.field == RBS_MTX_REAL || h.field == RBS_MTX_COMPLEX)) {
        int *fidx = nullptr, *nsel = nullptr;
        MCK(buf.get(fidx, (size_t)nz));
        MCK(buf.get(nsel, 1));
        size_t tmp = 0;
        thrust::counting_iterator<int> it(0);
        MCK(cub::DeviceSelect::Flagged(nullptr, tmp, it, hflag, fidx, nsel, nz, st));
        void *t = nullptr;
        MCK(buf.get(reinterpret_cast<char *&>(t), tmp));
        MCK(cub::DeviceSelect::Flagged(t, tmp, it, hflag, fidx, nsel, nz, st));
        int H = 0;
        MCK(cudaMemcpyAsync(&H, nsel, sizeof(int), cudaMemcpyDeviceToHost, st));
        MCK(cudaStreamSynchronize(st));
        if (H > 0) {
            unsigned char *dslots = nullptr;
            double *dhv = nullptr;
            MCK(buf.get(dslots, (size_t)H * SLOT));
            MCK(buf.get(dhv, (size_t)H));
            k_gather_tokens<<<grid_for(H, 256, sms), 256, 0, st>>>(ds, len, fidx, H, vpos, dslots);
            MCK(cudaGetLastError());
            std::vector<unsigned char> slots((size_t)H * SLOT);
            std::vector<int> hidx((size_t)H);
            std::vector<double> hv((size_t)H);
            MCK(cudaMemcpyAsync(slots.data(), dslots, slots.size(), cudaMemcpyDeviceToHost, st));
            MCK(cudaMemcpyAsync(hidx.data(), fidx, sizeof(int) * (size_t)H, cudaMemcpyDeviceToHost, st));
            MCK(cudaStreamSynchronize(st));
            // tokens longer than a slot: the whole token from the device copy
            for (int i = 0; i < H; ++i) {
                if (!slots[(size_t)i * SLOT + SLOT - 1]) continue;
                long long p = 0;
                MCK(cudaMemcpy(&p, vpos + hidx[(size_t)i], sizeof(p), cudaMemcpyDeviceToHost));
                std::string tok;
                for (long long q = p; q < len; q += 256) {
                    char tmpb[256];
                    const long long nb = std::min<long long>(256, len - q);
                    MCK(cudaMemcpy(tmpb, ds + q, (size_t)nb, cudaMemcpyDeviceToHost));
                    long long k = 0;
                    while (k < nb && !isspace((unsigned char)tmpb[k])) ++k;
                    tok.append(tmpb, (size_t)k);
                    if (k < nb) break;
                }
                char *e = nullptr;
                hv[(size_t)i] = strtod(tok.c_str(), &e);
                if (tok.empty() || *e) {
                    err = "Matrix Market reader: entry " + std::to_string(hidx[(size_t)i] + 1) + " has a malformed value";
                    return RBS_ERR_ARG;
                }
            }
            // the rest in parallel
            std::vector<int> bad_at;
            std::mutex bad_mu;
            auto work = [&](int lo, int hi) {
                for (int i = lo; i < hi; ++i) {
                    const char *tok = reinterpret_cast<const char *>(&slots[(size_t)i * SLOT]);
                    if (slots[(size_t)i * SLOT + SLOT - 1]) continue;
                    char *e = nullptr;
                    hv[(size_t)i] = strtod(tok, &e);
                    if (!*tok || *e) {
                        std::lock_guard<std::mutex> g(bad_mu);
                        bad_at.push_back(hidx[(size_t)i]);
                    }
                }
            };
            const int nth = H < 65536 ? 1 : (int)host_threads();
            std::vector<std::thread> th;
            for (int t = 1; t < nth; ++t) th.emplace_back(work, (int)((long long)H * t / nth), (int)((long long)H * (t + 1) / nth));
            work(0, (int)((long long)H / nth));
            for (auto &x : th) x.join();
            if (!bad_at.empty()) {
                err = "Matrix Market reader: entry " + std::to_string(*std::min_element(bad_at.begin(), bad_at.end()) + 1) +
                      " has a malformed value";
                return RBS_ERR_ARG;
            }
            MCK(cudaMemcpyAsync(dhv, hv.data(), sizeof(double) * (size_t)H, cudaMemcpyHostToDevice, st));
            k_scatter_values<<<grid_for(H, 256, sms), 256, 0, st>>>(fidx, H, dhv, v);
            MCK(cudaGetLastError());
            M.host_values = H;
        }
    }

    // symmetric expansion and the stable sort by row
    long long cnt = nz;
    int *keys = nullptr;
    unsigned *codes = nullptr;
    if (h.symmetric && nz) {
        size_t tmp = 0;
        MCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, mir, moff, nz + 1, st));
        void *t = nullptr;
        MCK(buf.get(reinterpret_cast<char *&>(t), tmp));
        MCK(cub::DeviceScan::ExclusiveSum(t, tmp, mir, moff, nz + 1, st));
        int extra = 0;
        MCK(cudaMemcpyAsync(&extra, moff + nz, sizeof(int), cudaMemcpyDeviceToHost, st));
        MCK(cudaStreamSynchronize(st));
        cnt = nz + extra;
    } else if (nz) {
        MCK(cudaMemsetAsync(moff, 0, sizeof(int) * ((size_t)nz + 1), st));
    }
    if (cnt > 0x7fffffffLL) {
        err = "Matrix Market reader: the expanded matrix exceeds 2^31-1 entries";
        return RBS_ERR_UNSUPPORTED;
    }
    M.nnz = cnt;
    MCK(buf.get(keys, (size_t)cnt));
    MCK(buf.get(codes, (size_t)cnt));
    unsigned *scodes = nullptr;
    MCK(buf.get(scodes, (size_t)cnt));
    // the handle's arrays come from the same pool (freed by mtx_free)
    MCK(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&M.rowptr), sizeof(int) * ((size_t)h.m + 1), buf.pool, st));
    MCK(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&M.colidx), sizeof(int) * std::max<size_t>((size_t)cnt, 1),
                                buf.pool, st));
    MCK(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&M.rowof), sizeof(int) * std::max<size_t>((size_t)cnt, 1),
                                buf.pool, st));
    MCK(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&M.val), sizeof(double) * std::max<size_t>((size_t)cnt, 1),
                                buf.pool, st));
    unsigned long long *lu = nullptr;
    MCK(buf.get(lu, 2));
    MCK(cudaMemsetAsync(lu, 0, sizeof(unsigned long long) * 2, st));
    if (cnt) {
        k_expand<<<grid_for(nz, 256, sms), 256, 0, st>>>(row, col, moff, nz, keys, codes);
        MCK(cudaGetLastError());
        size_t tmp = 0;
        const int nbits = bits_for(std::max(h.m, 1));
        MCK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, M.rowof, codes, scodes, (int)cnt, 0, nbits, st));
        void *t = nullptr;
        MCK(buf.get(reinterpret_cast<char *&>(t), tmp));
        MCK(cub::DeviceRadixSort::SortPairs(t, tmp, keys, M.rowof, codes, scodes, (int)cnt, 0, nbits, st));
        k_fill<<<grid_for(cnt, 256, sms), 256, 0, st>>>(scodes, M.rowof, row, col, v, cnt, M.colidx, M.val, lu);
        MCK(cudaGetLastError());
    }
    k_ptr_from_keys<<<grid_for(cnt + 1, 256, sms), 256, 0, st>>>(M.rowof, cnt, h.m, M.rowptr);
    MCK(cudaGetLastError());
    unsigned long long hlu[2] = {0, 0};
    MCK(cudaMemcpyAsync(hlu, lu, sizeof(hlu), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    M.nnz_lower = (long long)hlu[0];
    M.nnz_upper = (long long)hlu[1];
    M.parse_ms = ms_since(t1);
    return RBS_OK;
}

}  // namespace

// Per-device stream-ordered pool for the temporaries of the Matrix Market
// reader and the device analysis: after the first call, allocations and
// frees cost microseconds instead of cudaMalloc/cudaFree's milliseconds and
// device-wide synchronisation.  Up to 4 GB stays reserved between calls;
// the rest returns to the device at the next synchronisation.
namespace {
constexpr int MAX_DEV = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[MAX_DEV] = {};
}  // namespace

cudaError_t device_mem_pool(int dev, cudaMemPool_t &pool) {
    if (dev < 0 || dev >= MAX_DEV) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaError_t e = cudaMemPoolCreate(&g_pool[dev], &props);
        if (e != cudaSuccess) {
            g_pool[dev] = nullptr;
            return e;
        }
        unsigned long long keep = 4ULL << 30;
        e = cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
    }
    pool = g_pool[dev];
    return cudaSuccess;
}

void mtx_free(DeviceMtx &M) {
    if (!M.rowptr && !M.colidx && !M.rowof && !M.val) return;
    int old = 0;
    cudaGetDevice(&old);
    cudaSetDevice(M.device);
    for (void *p : {(void *)M.rowptr, (void *)M.colidx, (void *)M.rowof, (void *)M.val})
        if (p) cudaFreeAsync(p, nullptr);
    cudaStreamSynchronize(nullptr);
    cudaSetDevice(old);
    M.rowptr = M.colidx = M.rowof = nullptr;
    M.val = nullptr;
}

int mtx_read(const char *path, const void *bytes, long long len, const rbs_options &opt, DeviceMtx &M,
             std::string &err) {
    Source src;
    if (path) {
        src.fd = open(path, O_RDONLY);
        if (src.fd < 0) {
            err = std::string("Matrix Market reader: cannot open ") + path;
            return RBS_ERR_ARG;
        }
        struct stat sb;
        if (fstat(src.fd, &sb) != 0) {
            close(src.fd);
            err = std::string("Matrix Market reader: cannot stat ") + path;
            return RBS_ERR_ARG;
        }
        src.size = (long long)sb.st_size;
    } else {
        src.buf = static_cast<const unsigned char *>(bytes);
        src.size = len;
    }
    const int rc = read_impl(src, opt, M, err);
    if (src.fd >= 0) close(src.fd);
    if (rc) mtx_free(M);
    return rc;
}

int mtx_write(const char *path, int m, int n, const int *rp, const int *ci, const double *val, int symmetric,
              std::string &err) {
    // rows in parallel into per-thread text, then written in row order
    const int nth = (int)host_threads();
    std::vector<std::string> part((size_t)nth);
    long long total = 0;
    for (int i = 0; i < m; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k) total += !symmetric || ci[k] <= i;
    auto work = [&](int t) {
        const int lo = (int)((long long)m * t / nth), hi = (int)((long long)m * (t + 1) / nth);
        std::string &o = part[(size_t)t];
        o.reserve((size_t)(rp[hi] - rp[lo]) * 36);
        char line[96];
        for (int i = lo; i < hi; ++i)
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                if (symmetric && ci[k] > i) continue;
                const int len = val ? snprintf(line, sizeof line, "%d %d %.17g\n", i + 1, ci[k] + 1, val[k])
                                    : snprintf(line, sizeof line, "%d %d\n", i + 1, ci[k] + 1);
                o.append(line, (size_t)len);
            }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nth; ++t) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
    FILE *f = fopen(path, "wb");
    if (!f) {
        err = std::string("Matrix Market writer: cannot create ") + path;
        return RBS_ERR_ARG;
    }
    fprintf(f, "%%%%MatrixMarket matrix coordinate %s %s\n%d %d %lld\n", val ? "real" : "pattern",
            symmetric ? "symmetric" : "general", m, n, total);
    bool ok = true;
    for (const auto &o : part) ok = ok && fwrite(o.data(), 1, o.size(), f) == o.size();
    ok = (fclose(f) == 0) && ok;
    if (!ok) {
        err = std::string("Matrix Market writer: write error on ") + path;
        return RBS_ERR_ARG;
    }
    return RBS_OK;
}

int mtx_csr(const DeviceMtx &M, int *d_rowptr, int *d_colidx, double *d_val, std::string &err) {
    MCK(cudaSetDevice(M.device));
    MCK(cudaMemcpy(d_rowptr, M.rowptr, sizeof(int) * ((size_t)M.m + 1), cudaMemcpyDeviceToDevice));
    if (M.nnz) {
        MCK(cudaMemcpy(d_colidx, M.colidx, sizeof(int) * (size_t)M.nnz, cudaMemcpyDeviceToDevice));
        MCK(cudaMemcpy(d_val, M.val, sizeof(double) * (size_t)M.nnz, cudaMemcpyDeviceToDevice));
    }
    return RBS_OK;
}

int mtx_triangle(const DeviceMtx &M, int substitution, int fmt, const double *d_strict, int *d_ptr, int *d_idx,
                 double *d_val, std::string &err) {
    if (M.m != M.n) {
        err = "Matrix Market reader: the triangle needs a square matrix";
        return RBS_ERR_STRUCTURE;
    }
    const int forward = substitution == RBS_FORWARD;
    const long long cnt = M.nnz, m = M.m;
    const long long ntri = m + (forward ? M.nnz_lower : M.nnz_upper);
    if (ntri > 0x7fffffffLL) {
        err = "Matrix Market reader: the triangle exceeds 2^31-1 entries";
        return RBS_ERR_UNSUPPORTED;
    }
    MCK(cudaSetDevice(M.device));
    int sms = 148;
    MCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, M.device));
    cudaStream_t st = nullptr;
    MCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } sg{st};
    Buf buf;
    buf.st = st;
    MCK(pool_for(M.device, buf.pool));
    int *flag = nullptr, *srank = nullptr;
    MCK(buf.get(flag, (size_t)cnt + 1));
    MCK(buf.get(srank, (size_t)cnt + 1));
    k_strict_flags<<<grid_for(cnt + 1, 256, sms), 256, 0, st>>>(M.rowof, M.colidx, cnt, forward, flag);
    MCK(cudaGetLastError());
    {
        size_t tmp = 0;
        MCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag, srank, cnt + 1, st));
        void *t = nullptr;
        MCK(buf.get(reinterpret_cast<char *&>(t), tmp));
        MCK(cub::DeviceScan::ExclusiveSum(t, tmp, flag, srank, cnt + 1, st));
    }
    const bool csc = fmt == RBS_FMT_CSC;
    int *tptr = d_ptr, *tidx = d_idx, *trow = nullptr;
    double *tval = d_val;
    if (csc) {
        MCK(buf.get(tptr, (size_t)m + 1));
        MCK(buf.get(tidx, (size_t)ntri));
        MCK(buf.get(tval, (size_t)ntri));
        MCK(buf.get(trow, (size_t)ntri));
    }
    if (cnt) {
        k_tri_scatter<<<grid_for(cnt, 256, sms), 256, 0, st>>>(M.rowof, M.colidx, M.val, flag, srank, cnt, forward,
                                                               d_strict, tidx, tval, trow);
        MCK(cudaGetLastError());
    }
    k_tri_rows<<<grid_for(m + 1, 256, sms), 256, 0, st>>>(M.rowptr, srank, (int)m, forward, tptr, tidx, tval, trow);
    MCK(cudaGetLastError());
    if (csc) {
        // tranpose.h:7-54: stable by column, rows ascending inside a column
        int *perm = nullptr, *sperm = nullptr, *skeys = nullptr;
        MCK(buf.get(perm, (size_t)ntri));
        MCK(buf.get(sperm, (size_t)ntri));
        MCK(buf.get(skeys, (size_t)ntri));
        if (ntri) {
            k_iota<<<grid_for(ntri, 256, sms), 256, 0, st>>>(perm, ntri);
            MCK(cudaGetLastError());
            size_t tmp = 0;
            const int nbits = bits_for(std::max<long long>(m, 1));
            MCK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, tidx, skeys, perm, sperm, (int)ntri, 0, nbits, st));
            void *t = nullptr;
            MCK(buf.get(reinterpret_cast<char *&>(t), tmp));
            MCK(cub::DeviceRadixSort::SortPairs(t, tmp, tidx, skeys, perm, sperm, (int)ntri, 0, nbits, st));
            k_gather_csc<<<grid_for(ntri, 256, sms), 256, 0, st>>>(sperm, trow, tval, ntri, d_idx, d_val);
            MCK(cudaGetLastError());
        }
        k_ptr_from_keys<<<grid_for(ntri + 1, 256, sms), 256, 0, st>>>(skeys, ntri, (int)m, d_ptr);
        MCK(cudaGetLastError());
    }
    MCK(cudaStreamSynchronize(st));
    return RBS_OK;
}

}  // namespace rbs
