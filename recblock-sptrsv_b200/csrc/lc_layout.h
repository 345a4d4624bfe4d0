// lc_layout.h -- constants and record sizes of the level-chunk layout
// shared by the host analysis (which builds the records) and the kernel
// (level_lc.cuh, which reads them).
#pragma once

#ifdef __CUDACC__
#define LC_HD __host__ __device__
#else
#define LC_HD
#endif

namespace rbs {

constexpr int LC_XW = 8192;  // window rows
constexpr int LC_NB = 32;    // mbarrier slots (chunks in flight at most)
constexpr int LC_D = 2;      // gather distance in chunks
constexpr int LC_RMAX = 1024;
// threads of the CTA: the random band factor's chunks hold about 170 rows,
// and 512 threads left two thirds of the warps idle at every chunk barrier
// (c2r forward 28.0 -> 27.3 ms, the 512-system batch 10.0 -> 9.75 ms at 256)
constexpr int LC_T = 256;
constexpr int LC_SMEM = 232448 - 1024;  // dynamic shared memory (227 KB less room for the static part)
constexpr int LC_RING = ((LC_SMEM - LC_XW * 8 - LC_NB * 8) / 16) * 16;
constexpr int LC_FMAX = ((LC_RING / 6) / 16) * 16;  // about six chunks in flight
constexpr int LC_HDR_INTS = 8;
static_assert(LC_XW >= (LC_D + 1) * LC_RMAX, "old dependencies must be final when gathered");

struct LcChunk {  // 16-byte units unless noted
    int src64, bytes64;  // static record, FP64 layout
    int src32, bytes32;  // static record, FP32 layout
    int ring;            // ring offset
    int issue;           // chunk iteration at whose start the copy is issued
    int blo, bn;         // rows: the chunk's block rows are [blo, blo + bn) (blo = -1: scattered)
    int bs64, bs32;      // offset of the right-hand-side area from the record start
};
constexpr int LC_TAB_INTS = 10;
static_assert(sizeof(LcChunk) == LC_TAB_INTS * sizeof(int), "table rows are LC_TAB_INTS ints");

LC_HD constexpr int lc_pad4(int n) { return (n + 3) & ~3; }  // ints up to a 16-byte multiple
LC_HD constexpr long long lc_padv(int n, int es) { return (long long)((n * (long long)es + 15) / 16) * 16; }  // bytes

// Record of a chunk of nr rows with no old and nrec recent entries whose
// recent entries form ncols jagged columns.  Ints: header, dest[nr],
// rlen[nr], rpo[nr+1], cs[ncols+1]; then inv[nr] (VT), colr[nrec] (int),
// valr[nrec] (VT), colo[no] (int), valo[no] (VT); the ring also reserves
// gx[no] and the right-hand-side area bs (VT) behind the copied part: nr
// values, or a 16-byte-aligned bulk copy of b[blo, blo+nr) with up to
// 16 bytes of slack at either end.
LC_HD constexpr long long lc_static_bytes(int nr, int no, int nrec, int ncols, int es) {
    return 4LL * (LC_HDR_INTS + 2 * lc_pad4(nr) + lc_pad4(nr + 1) + lc_pad4(ncols + 1)) + lc_padv(nr, es) +
           4LL * lc_pad4(nrec) + lc_padv(nrec, es) + 4LL * lc_pad4(no) + lc_padv(no, es);
}
LC_HD constexpr long long lc_foot_bytes(int nr, int no, int nrec, int ncols, int es) {
    return lc_static_bytes(nr, no, nrec, ncols, es) + lc_padv(no, es) + lc_padv(nr + 32 / es, es);
}

}  // namespace rbs
