// analysis.cpp -- host analysis: validation, level sets, level-set
// permutation, recursive-block geometry, per-block statistics, the
// reference's per-block method codes, kernel selection and the
// processing-order execution layout.
//
// Integer outputs that the reference also produces (level order, labels,
// block bounds, nnz per block, method codes, local level counts, packed
// arrays) are bit-identical to recblock-sptrsv's CPU analysis
// (recblocking_preprocess.h get_recblock_size + L_/U_preprocessing); the
// packed reference-format arrays are rebuilt on demand by export_reference.
#include <algorithm>
#include <thread>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>

#include "lc_layout.h"
#include "rbs_internal.h"

namespace rbs {

namespace {

constexpr int kLongRow = SQ_LONGROW;
constexpr int kMedRow = SQ_MEDROW;

int lowbit(int t) { return t & -t; }

// Stable CSR(rows x cols) -> CSC transposition (tranpose.h:7-54 semantics:
// entries of a column appear in ascending row order).  Large matrices are
// transposed on host threads, each owning a range of output columns of about
// equal size and scanning in order the rows of every row group whose column
// span meets its range.
template <typename IV, typename DV>
void transpose(int rows, int cols, const int *ptr, const int *idx, const double *val, std::vector<int> &tptr, IV &tidx,
               DV &tval) {
    int nnz = ptr[rows];
    tptr.assign((size_t)cols + 1, 0);
    for (int k = 0; k < nnz; ++k) tptr[(size_t)idx[k] + 1]++;
    for (int c = 0; c < cols; ++c) tptr[(size_t)c + 1] += tptr[c];
    tidx.resize((size_t)nnz);
    tval.resize(val ? (size_t)nnz : 0);
    const int parts = nnz < (1 << 20) ? 1 : 16;
    std::vector<int> cut((size_t)parts + 1, cols);  // output columns [cut[t], cut[t+1])
    for (int t = 1; t < parts; ++t)
        cut[t] = (int)(std::lower_bound(tptr.begin(), tptr.end(), (int)((long long)nnz * t / parts)) - tptr.begin());
    cut[0] = 0;
    constexpr int kGroup = 256;  // rows per group
    const int ngroup = (rows + kGroup - 1) / kGroup;
    std::vector<int> gmin((size_t)ngroup, INT_MAX), gmax((size_t)ngroup, -1);  // column span of a group
    if (parts > 1)
        parallel_for(((size_t)ngroup + 1023) / 1024, [&](size_t i) {
            for (int g = (int)i * 1024; g < std::min(ngroup, (int)i * 1024 + 1024); ++g)
                for (int k = ptr[g * kGroup]; k < ptr[std::min(rows, g * kGroup + kGroup)]; ++k) {
                    gmin[g] = std::min(gmin[g], idx[k]);
                    gmax[g] = std::max(gmax[g], idx[k]);
                }
        });
    parallel_for((size_t)parts, [&](size_t t) {
        const int lo = cut[t], hi = cut[t + 1];
        if (lo >= hi) return;
        std::vector<int> fill(tptr.begin() + lo, tptr.begin() + hi);
        for (int g = 0; g < ngroup; ++g) {
            if (parts > 1 && (gmax[g] < lo || gmin[g] >= hi)) continue;
            for (int r = g * kGroup; r < std::min(rows, g * kGroup + kGroup); ++r)
                for (int k = ptr[r]; k < ptr[r + 1]; ++k) {
                    const int c = idx[k];
                    if (c < lo || c >= hi) continue;
                    const int d = fill[c - lo]++;
                    tidx[d] = r;
                    if (val) tval[d] = val[k];
                }
        }
    });
}

// Kahn breadth-first level sets in the discovery order of findlevel.h:7-83:
// in-degree = entries per row (diagonal included), a row joins the next
// level the moment its in-degree reaches 1, levels are walked in the order
// their rows were discovered and each column in stored order.
// Returns the level count, or -1 if a level makes no progress.
int bfs_levels(const int *cp, const int *ri, int m, std::vector<int> &levelPtr, std::vector<int> &item) {
    std::vector<int> deg((size_t)m, 0);
    for (int k = 0; k < cp[m]; ++k) deg[ri[k]]++;
    item.resize((size_t)m);
    levelPtr.clear();
    levelPtr.push_back(0);
    int tail = 0;
    for (int i = 0; i < m; ++i)
        if (deg[i] == 1) item[tail++] = i;
    levelPtr.push_back(tail);
    int head = 0;
    while (tail != m) {
        int end = tail;
        if (head == end) return -1;  // no root / cycle: the reference spins forever here
        for (; head < end; ++head) {
            int node = item[head];
            for (int k = cp[node]; k < cp[node + 1]; ++k) {
                int r = ri[k];
                if (--deg[r] == 1) item[tail++] = r;
            }
        }
        if (tail == end) return -1;
        levelPtr.push_back(tail);
    }
    return (int)levelPtr.size() - 1;
}

int pick_group(double avg) {
    if (avg < 3) return 1;
    if (avg < 6) return 2;
    if (avg < 12) return 4;
    if (avg < 24) return 8;
    if (avg < 48) return 16;
    return 32;
}

// Kernel choice.  REFERENCE maps each reference method to this library's
// kernel of the same kind; AUTO uses a latency/bandwidth cost model of the
// B200 (constants measured on a B200 with bench.py).
void select_kernel(ExecBlock &b, const rbs_options &opt, const std::vector<int> &lvl_sizes) {
    if (!b.tri) {
        if (b.nnz == 0) {
            b.kernel = RBS_K_EMPTY;
            b.group = 1;
            return;
        }
        b.kernel = RBS_K_SPMV;
        double avg = (double)b.nnz / std::max(1, b.nonempty);
        if (opt.select == RBS_SELECT_REFERENCE)
            b.group = (b.ref_method == 0 || b.ref_method == 1) ? 1 : 32;
        else
            b.group = pick_group(avg);
        return;
    }
    int off = b.nnz - b.m;  // strictly off-diagonal entries
    double avg = (double)off / std::max(1, b.m);
    b.group = pick_group(avg);
    if (off == 0) {
        b.kernel = RBS_K_DIAG;
        return;
    }
    if (opt.select == RBS_SELECT_REFERENCE) {
        switch (b.ref_method) {
        case 0: b.kernel = RBS_K_DIAG; break;
        case 1: b.kernel = b.bandwidth <= 8 ? RBS_K_BANDSCAN : RBS_K_SEQ; break;
        case 2: b.kernel = RBS_K_LEVEL; break;
        default: b.kernel = RBS_K_SYNCFREE; break;
        }
        return;
    }
    // AUTO cost model (microseconds).
    double bytes = (double)off * 12.0 + (double)b.m * 24.0;
    double passes = 0;
    for (int w : lvl_sizes) passes += std::max(1.0, std::ceil((double)w * b.group / 1024.0));
    double t_level = passes * 0.12 + bytes / 180e3 + 4.0;
    double t_sync = (double)b.nlv * 0.9 + bytes / 4.0e6 + 4.0;
    double t_seq = (double)b.m * 0.012 + bytes / 120e3 + 4.0;
    double t_scan = b.bandwidth <= 8 ? bytes * 3.0 / 3.0e6 + 25.0 : 1e30;
    double best = t_sync;
    b.kernel = RBS_K_SYNCFREE;
    if (t_level < best) { best = t_level; b.kernel = RBS_K_LEVEL; }
    if (t_seq < best) { best = t_seq; b.kernel = RBS_K_SEQ; }
    if (t_scan < best) { best = t_scan; b.kernel = RBS_K_BANDSCAN; }
}

// The processing-order CSR (full_rp/col/val) from a row view of the matrix:
// row r holds entries rp[r]..rp[r+1] (columns rc, values rv), the entries of
// one column in the order the CSC holds them.  Processing row p is row
// perm[p] with its columns renumbered to processing positions and stably
// sorted -- the arrays of the column walk in processing order (a stable sort
// by processing column, then by row), built row by row on host threads.
void full_csr_from_rows(Plan &P, const int *rp, const int *rc, const double *rv, const std::vector<int> &pos_of) {
    const int n = P.n;
    P.full_rp.assign((size_t)n + 1, 0);
    for (int p = 0; p < n; ++p) {
        const int r = P.perm[p];
        P.full_rp[(size_t)p + 1] = P.full_rp[p] + (rp[r + 1] - rp[r]);
    }
    P.full_col.resize((size_t)P.full_rp[n]);
    P.full_val.resize((size_t)P.full_rp[n]);
    constexpr int kRows = 1 << 14;
    parallel_for(((size_t)n + kRows - 1) / kRows, [&](size_t chunk) {
        std::vector<std::pair<int, int>> key;  // (processing column, entry) of a long row
        const int p0 = (int)chunk * kRows, p1 = std::min(n, p0 + kRows);
        for (int p = p0; p < p1; ++p) {
            const int r = P.perm[p], b = rp[r], len = rp[r + 1] - b;
            int *oc = P.full_col.data() + P.full_rp[p];
            double *ov = P.full_val.data() + P.full_rp[p];
            if (len <= 64) {
                for (int j = 0; j < len; ++j) {  // insertion: equal columns keep their order
                    const int q = pos_of[rc[b + j]];
                    const double v = rv[b + j];
                    int i = j;
                    for (; i > 0 && oc[i - 1] > q; --i) {
                        oc[i] = oc[i - 1];
                        ov[i] = ov[i - 1];
                    }
                    oc[i] = q;
                    ov[i] = v;
                }
            } else {
                key.resize((size_t)len);
                for (int j = 0; j < len; ++j) key[j] = {pos_of[rc[b + j]], j};
                std::sort(key.begin(), key.end());  // by column, then entry: stable
                for (int j = 0; j < len; ++j) {
                    oc[j] = key[j].first;
                    ov[j] = rv[b + key[j].second];
                }
            }
        }
    });
}

}  // namespace

// Algorithmic bytes of one FP64 single-RHS pass over a block: every stored
// entry once (8-byte value + 4-byte index), the row pointer, and per row the
// right-hand side read plus the result written; triangles also read the
// inverse diagonal; squares read the x segment they multiply once.
double block_bytes(const Plan &P, const ExecBlock &B) {
    (void)P;
    if (B.tri) return (double)(B.nnz - B.m) * 12.0 + 4.0 * (B.m + 1) + 24.0 * B.m;
    if (B.nnz == 0) return 0.0;
    return (double)B.nnz * 12.0 + 4.0 * (B.nrows + 1) + 16.0 * B.nonempty + 8.0 * B.ncols +
           (B.rows_off >= 0 ? 4.0 * B.nrows : 0.0);
}

// Layouts a triangle needs: the ones of its kernel, or, when the kernels
// are chosen by measurement (RBS_SELECT_TUNE), every one it is eligible for.
static bool wants_level(const ExecBlock &b, const rbs_options &opt) {
    return b.tri && (b.kernel == RBS_K_LEVEL || (opt.select == RBS_SELECT_TUNE && b.nnz > b.m));
}
static bool wants_band(const ExecBlock &b, const rbs_options &opt) {
    return b.tri && b.bandwidth <= 8 &&
           (b.kernel == RBS_K_BANDSCAN || (opt.select == RBS_SELECT_TUNE && b.nnz > b.m));
}

// Level-chunk layout of every level triangle (level_lc.cuh).  Rows of each
// independent segment (the whole triangle, or the rows of one system of a
// batch) are taken level by level; a chunk takes consecutive rows of one
// level while it stays within LC_RMAX rows and LC_FMAX bytes of ring
// footprint.  Within a chunk rows are ordered by their count of recent
// entries (largest first, ties in level order), which fixes their virtual
// row numbers.  An entry is "recent" when its dependency is still in the
// window of the last LC_XW virtual rows after the chunk is solved, "old"
// otherwise (gathered ahead).  Records are placed in the kernel's
// shared-memory ring in order, wrapping to 0 when the next one does not
// fit; a record's copy is issued once every chunk whose ring bytes it reuses
// has been solved and its mbarrier slot is free.
// One triangle's level-chunk layout into `out`, record and table offsets
// relative to `out` (build_lc merges the blocks in order and rebases them).
struct LcOut {
    bulk_vector<uint32_t> rec64, rec32;
    std::vector<int> tab, segs;
};
// Appends parts to dst in order: record starts in the tables (16-byte
// units) and the first chunk of every segment triple rebased; the copies run
// on host threads and the parts are emptied.  first_seg[i] receives the
// index of part i's first segment triple in dst.
static void lc_append(LcOut &dst, const std::vector<LcOut *> &parts, std::vector<long long> *first_seg = nullptr) {
    const size_t np = parts.size();
    if (np == 1 && dst.rec64.empty() && dst.rec32.empty() && dst.tab.empty() && dst.segs.empty()) {
        std::swap(dst, *parts[0]);  // nothing to rebase
        if (first_seg) first_seg->assign(1, 0);
        return;
    }
    std::vector<size_t> o64(np), o32(np), otab(np), oseg(np);
    size_t n64 = dst.rec64.size(), n32 = dst.rec32.size(), ntab = dst.tab.size(), nseg = dst.segs.size();
    for (size_t i = 0; i < np; ++i) {
        o64[i] = n64;
        o32[i] = n32;
        otab[i] = ntab;
        oseg[i] = nseg;
        n64 += parts[i]->rec64.size();
        n32 += parts[i]->rec32.size();
        ntab += parts[i]->tab.size();
        nseg += parts[i]->segs.size();
    }
    dst.rec64.resize(n64);
    dst.rec32.resize(n32);
    dst.tab.resize(ntab);
    dst.segs.resize(nseg);
    if (first_seg) {
        first_seg->resize(np);
        for (size_t i = 0; i < np; ++i) (*first_seg)[i] = (long long)(oseg[i] / 3);
    }
    parallel_for(np, [&](size_t i) {
        LcOut &p = *parts[i];
        if (!p.rec64.empty()) std::memcpy(dst.rec64.data() + o64[i], p.rec64.data(), p.rec64.size() * 4);
        if (!p.rec32.empty()) std::memcpy(dst.rec32.data() + o32[i], p.rec32.data(), p.rec32.size() * 4);
        const int r64_base = (int)(o64[i] / 4), r32_base = (int)(o32[i] / 4), tab_base = (int)(otab[i] / LC_TAB_INTS);
        for (size_t j = 0; j < p.tab.size(); ++j) {
            const size_t f = j % LC_TAB_INTS;
            dst.tab[otab[i] + j] = p.tab[j] + (f == 0 ? r64_base : f == 2 ? r32_base : 0);
        }
        for (size_t j = 0; j < p.segs.size(); ++j) dst.segs[oseg[i] + j] = p.segs[j] + (j % 3 == 0 ? tab_base : 0);
        LcOut().rec64.swap(p.rec64);
        LcOut().rec32.swap(p.rec32);
    });
}
static void build_lc_block(const Plan &P, ExecBlock &B, const rbs_options &opt, const std::vector<int> &level,
                           LcOut &out, bool seg_threads) {
    B.lc_ok = 0;
    B.lc_nseg = 0;
    B.lc_seg_off = -1;
    if (!wants_level(B, opt) || B.nnz == B.m) return;
    const int m = B.m;
    const int *rp = P.rp_pool.data() + B.rp_off;
    const int *cl = P.col_pool.data();
    const double *vl = P.val_pool.data();
    // segment of every row (ids in order of first appearance)
    int nseg = 1;
    std::vector<int> seg((size_t)m, 0);
    if (!P.seg_rows.empty()) {
        std::vector<int> id(P.seg_rows.size(), -1);
        nseg = 0;
        constexpr int kRows = 1 << 14;
        parallel_for(((size_t)m + kRows - 1) / kRows, [&](size_t ch) {
            for (int r = (int)ch * kRows; r < std::min(m, (int)ch * kRows + kRows); ++r) {
                const int o = P.perm[(size_t)B.r0 + r];
                seg[(size_t)r] = (int)(std::upper_bound(P.seg_rows.begin(), P.seg_rows.end(), o) - P.seg_rows.begin()) - 1;
            }
        });
        for (int r = 0; r < m; ++r) {
            int &sg = seg[(size_t)r];
            if (id[(size_t)sg] < 0) id[(size_t)sg] = nseg++;
            sg = id[(size_t)sg];
        }
    }
    // rows level by level (stable), then split by segment
    std::vector<int> lstart((size_t)B.nlv + 1, 0);
    for (int r = 0; r < m; ++r) lstart[(size_t)level[(size_t)B.r0 + r] + 1]++;
    for (int l = 0; l < B.nlv; ++l) lstart[(size_t)l + 1] += lstart[(size_t)l];
    std::vector<int> bylev((size_t)m);
    {
        std::vector<int> fill(lstart.begin(), lstart.end() - 1);
        for (int r = 0; r < m; ++r) bylev[(size_t)fill[(size_t)level[(size_t)B.r0 + r]]++] = r;
    }
    std::vector<int> scount((size_t)nseg + 1, 0);
    for (int r = 0; r < m; ++r) scount[(size_t)seg[(size_t)r] + 1]++;
    for (int q = 0; q < nseg; ++q) scount[(size_t)q + 1] += scount[(size_t)q];
    std::vector<int> seq((size_t)m);
    {
        std::vector<int> fill(scount.begin(), scount.end() - 1);
        for (int t = 0; t < m; ++t) {
            const int r = bylev[(size_t)t];
            seq[(size_t)fill[(size_t)seg[(size_t)r]]++] = r;
        }
    }
    // Segments are independent systems (no entry of one refers to a row of
    // another): chunks, ring placement and records are built per segment,
    // on host threads when seg_threads is set, and the records merged in
    // the segment order below.
    struct Ch { int v0, nr, no, nrec, ncols, maxlen; };
    std::vector<std::vector<Ch>> chunks((size_t)nseg);
    std::vector<std::vector<int>> roff((size_t)nseg), iss((size_t)nseg);
    std::vector<char> seg_ok((size_t)nseg, 1);
    std::vector<int> vpos((size_t)m, -1);
    // chunks of segment q (its rows in seq reordered inside every chunk and
    // their vpos assigned), then their ring offsets and issue iterations
    auto layout = [&](size_t qz) {
        const int q = (int)qz;
        std::vector<int> rl((size_t)LC_RMAX);
        auto counts = [&](const int *rows, int nr, int thr, int &no, int &nrec, int &ncols) {
            no = nrec = ncols = 0;
            for (int t = 0; t < nr; ++t) {
                const int r = rows[t];
                int rr = 0;
                for (int k = rp[r]; k < rp[r + 1]; ++k) rr += vpos[(size_t)cl[k]] >= thr;
                rl[(size_t)t] = rr;
                nrec += rr;
                no += rp[r + 1] - rp[r] - rr;
                ncols = std::max(ncols, rr);
            }
        };
        int *sq = seq.data() + scount[(size_t)q];
        const int len = scount[(size_t)q + 1] - scount[(size_t)q];
        auto &ch = chunks[(size_t)q];
        int i = 0;
        while (i < len) {
            const int L = level[(size_t)B.r0 + sq[i]];
            const int thr_c = i + LC_RMAX - LC_XW;  // no later threshold is larger
            int nr = 0, no = 0, nrec = 0, ncols = 0;
            while (i + nr < len && nr < LC_RMAX && level[(size_t)B.r0 + sq[i + nr]] == L) {
                const int r = sq[i + nr];
                int ro = 0, rr = 0;
                for (int k = rp[r]; k < rp[r + 1]; ++k) (vpos[(size_t)cl[k]] < thr_c ? ro : rr)++;
                if (lc_foot_bytes(nr + 1, no + ro, nrec + rr, std::max(ncols, rr), 8) > LC_FMAX) break;
                ++nr;
                no += ro;
                nrec += rr;
                ncols = std::max(ncols, rr);
            }
            if (nr == 0) {  // one row alone does not fit the ring
                seg_ok[(size_t)q] = 0;
                return;
            }
            // exact split with this chunk's own threshold
            for (;;) {
                counts(sq + i, nr, i + nr - LC_XW, no, nrec, ncols);
                if (lc_foot_bytes(nr, no, nrec, ncols, 8) <= LC_FMAX || nr == 1) break;
                --nr;
            }
            if (lc_foot_bytes(nr, no, nrec, ncols, 8) > LC_FMAX) {
                seg_ok[(size_t)q] = 0;
                return;
            }
            // rows by recent count, largest first (stable)
            std::vector<int> idx((size_t)nr);
            for (int t = 0; t < nr; ++t) idx[(size_t)t] = t;
            std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return rl[(size_t)a] > rl[(size_t)b]; });
            std::vector<int> rows((size_t)nr);
            for (int t = 0; t < nr; ++t) rows[(size_t)t] = sq[i + idx[(size_t)t]];
            for (int t = 0; t < nr; ++t) {
                sq[i + t] = rows[(size_t)t];
                vpos[(size_t)rows[(size_t)t]] = i + t;
            }
            int maxlen = 0;
            for (int t = 0; t < nr; ++t) maxlen = std::max(maxlen, rp[rows[(size_t)t] + 1] - rp[rows[(size_t)t]]);
            ch.push_back({i, nr, no, nrec, ncols, maxlen});
            i += nr;
        }
        // ring placement and issue iterations
        const int nch = (int)ch.size();
        auto &ro = roff[(size_t)q];
        auto &is = iss[(size_t)q];
        ro.resize((size_t)nch);
        is.resize((size_t)nch);
        long long head = 0;
        std::vector<long long> fb((size_t)nch);
        for (int j = 0; j < nch; ++j) {
            const Ch &c = ch[(size_t)j];
            const long long F = lc_foot_bytes(c.nr, c.no, c.nrec, c.ncols, 8);
            fb[(size_t)j] = F;
            if (head + F > LC_RING) head = 0;
            ro[(size_t)j] = (int)(head / 16);
            head += F;
            // mbarrier slot j % LC_NB: every thread must have seen chunk j - LC_NB
            // land (its gather, at chunk iteration j - LC_NB - LC_D or in the
            // prologue) and passed a CTA barrier since, i.e. the end of that
            // iteration (iteration 0 for chunks gathered in the prologue)
            int at = j > 0 ? is[(size_t)j - 1] : 0;
            if (j >= LC_NB) at = std::max(at, std::max(1, j - LC_NB - LC_D + 1));
            long long scanned = 0;
            for (int k = j - 1; k >= 0 && scanned <= 2LL * LC_RING; --k) {
                const long long a0 = 16LL * ro[(size_t)k], a1 = a0 + fb[(size_t)k];
                const long long b0 = 16LL * ro[(size_t)j], b1 = b0 + F;
                if (a0 < b1 && b0 < a1) {
                    at = std::max(at, k + 1);
                    break;
                }
                scanned += fb[(size_t)k];
            }
            if (at > std::max(0, j - LC_D)) {
                seg_ok[(size_t)q] = 0;
                return;
            }
            is[(size_t)j] = at;
        }
    };
    if (seg_threads) parallel_for((size_t)nseg, layout);
    else
        for (int q = 0; q < nseg; ++q) layout((size_t)q);
    for (int q = 0; q < nseg; ++q)
        if (!seg_ok[(size_t)q]) return;
    // records of segment q into so, offsets relative to so
    auto records = [&](int q, LcOut &so) {
        const int *sq = seq.data() + scount[(size_t)q];
        const auto &ch = chunks[(size_t)q];
        const int nch = (int)ch.size();
        so.segs.insert(so.segs.end(), {(int)(so.tab.size() / LC_TAB_INTS), nch, nch ? roff[(size_t)q][0] : 0});
        std::vector<int> dest, rlen, rpo, cs, colr, colo;
        std::vector<double> inv, valr, valo;
        for (int j = 0; j < nch; ++j) {
            const Ch &c = ch[(size_t)j];
            const int thr = c.v0 + c.nr - LC_XW;
            dest.assign((size_t)c.nr, 0);
            rlen.assign((size_t)c.nr, 0);
            rpo.assign(1, 0);
            inv.assign((size_t)c.nr, 0.0);
            colo.clear();
            valo.clear();
            for (int t = 0; t < c.nr; ++t) {
                const int r = sq[c.v0 + t];
                dest[(size_t)t] = r;
                inv[(size_t)t] = P.inv_diag[(size_t)B.r0 + r];
                for (int k = rp[r]; k < rp[r + 1]; ++k) {
                    if (vpos[(size_t)cl[k]] >= thr) rlen[(size_t)t]++;
                    else {
                        colo.push_back(cl[k]);
                        valo.push_back(vl[k]);
                    }
                }
                rpo.push_back((int)colo.size());
            }
            cs.assign((size_t)c.ncols + 1, 0);
            for (int k = 0; k < c.ncols; ++k) {
                int cnt = 0;
                while (cnt < c.nr && rlen[(size_t)cnt] > k) ++cnt;  // rlen is non-increasing
                cs[(size_t)k + 1] = cs[(size_t)k] + cnt;
            }
            colr.assign((size_t)c.nrec, 0);
            valr.assign((size_t)c.nrec, 0.0);
            for (int t = 0; t < c.nr; ++t) {
                const int r = sq[c.v0 + t];
                int kk = 0;
                for (int k = rp[r]; k < rp[r + 1]; ++k) {
                    const int vd = vpos[(size_t)cl[k]];
                    if (vd < thr) continue;
                    colr[(size_t)(cs[(size_t)kk] + t)] = vd & (LC_XW - 1);
                    valr[(size_t)(cs[(size_t)kk] + t)] = vl[k];
                    ++kk;
                }
            }
            const int rnext = j + 1 < nch ? roff[(size_t)q][(size_t)j + 1] : 0;
            // contiguous block rows: the kernel bulk-copies their right-hand side
            int dmin = dest[0], dmax = dest[0];
            for (int t = 1; t < c.nr; ++t) {
                dmin = std::min(dmin, dest[(size_t)t]);
                dmax = std::max(dmax, dest[(size_t)t]);
            }
            const int blo = dmax - dmin + 1 == c.nr ? dmin : -1;
            auto emit = [&](bulk_vector<uint32_t> &pool, int es) -> std::pair<int, int> {
                const size_t base = pool.size();
                const long long bytes = lc_static_bytes(c.nr, c.no, c.nrec, c.ncols, es);
                pool.resize(base + (size_t)(bytes / 4), 0u);
                uint32_t *w = pool.data() + base;
                const int hdr[LC_HDR_INTS] = {c.nr, c.no, c.nrec, c.v0, rnext, c.ncols, c.maxlen, blo};
                std::memcpy(w, hdr, sizeof(hdr));
                size_t o = LC_HDR_INTS;
                auto put_i = [&](const std::vector<int> &v) {
                    if (!v.empty()) std::memcpy(w + o, v.data(), v.size() * 4);
                    o += (size_t)lc_pad4((int)v.size());
                };
                auto put_v = [&](const std::vector<double> &v) {
                    if (es == 8) {
                        if (!v.empty()) std::memcpy(w + o, v.data(), v.size() * 8);
                    } else {
                        for (size_t t = 0; t < v.size(); ++t) {
                            const float f = (float)v[t];
                            std::memcpy(w + o + t, &f, 4);
                        }
                    }
                    o += (size_t)(lc_padv((int)v.size(), es) / 4);
                };
                put_i(dest);
                put_i(rlen);
                put_i(rpo);
                put_i(cs);
                put_v(inv);
                put_i(colr);
                put_v(valr);
                put_i(colo);
                put_v(valo);
                return {(int)(base / 4), (int)(bytes / 16)};
            };
            const auto r64 = emit(so.rec64, 8);
            const auto r32 = emit(so.rec32, 4);
            const int bs64 = (int)((lc_static_bytes(c.nr, c.no, c.nrec, c.ncols, 8) + lc_padv(c.no, 8)) / 16);
            const int bs32 = (int)((lc_static_bytes(c.nr, c.no, c.nrec, c.ncols, 4) + lc_padv(c.no, 4)) / 16);
            so.tab.insert(so.tab.end(), {r64.first, r64.second, r32.first, r32.second, roff[(size_t)q][(size_t)j],
                                         iss[(size_t)q][(size_t)j], blo, blo >= 0 ? c.nr : 0, bs64, bs32});
        }
    };
    // segments in order of decreasing work (the persistent kernel's queue)
    B.lc_ok = 1;
    B.lc_nseg = nseg;
    B.lc_seg_off = 0;  // set when the blocks are merged
    std::vector<int> order((size_t)nseg);
    for (int q = 0; q < nseg; ++q) order[(size_t)q] = q;
    auto work = [&](int q) {
        long long e = 0;
        for (const Ch &c : chunks[(size_t)q]) e += c.no + c.nrec;
        return (long long)chunks[(size_t)q].size() * 4096 + e;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
    if (!seg_threads) {
        for (int q : order) records(q, out);
        return;
    }
    std::vector<LcOut> so((size_t)nseg);
    parallel_for((size_t)nseg, [&](size_t q) { records((int)q, so[q]); });
    std::vector<LcOut *> parts;
    for (int q : order) parts.push_back(&so[(size_t)q]);
    lc_append(out, parts);
}

static void build_lc(Plan &P, const rbs_options &opt, const std::vector<int> &level) {
    P.lc_rec64.clear();
    P.lc_rec32.clear();
    P.lc_tab.clear();
    P.lc_segs.clear();
    // blocks are independent: built on host threads (or, in a batch, one
    // after another with their systems on host threads), merged in block
    // order
    const size_t nb = P.blocks.size();
    std::vector<LcOut> outs(nb);
    if (P.seg_rows.empty())
        parallel_for(nb, [&](size_t b) { build_lc_block(P, P.blocks[b], opt, level, outs[b], false); });
    else
        for (size_t b = 0; b < nb; ++b) build_lc_block(P, P.blocks[b], opt, level, outs[b], true);
    std::vector<LcOut *> parts;
    std::vector<size_t> which;
    for (size_t b = 0; b < nb; ++b)
        if (P.blocks[b].lc_ok) {
            parts.push_back(&outs[b]);
            which.push_back(b);
        }
    LcOut all;
    std::vector<long long> first;
    lc_append(all, parts, &first);
    for (size_t i = 0; i < which.size(); ++i) P.blocks[which[i]].lc_seg_off = first[i];
    P.lc_rec64.swap(all.rec64);
    P.lc_rec32.swap(all.rec32);
    P.lc_tab.swap(all.tab);
    P.lc_segs.swap(all.segs);
}

int host_bfs_levels(const int *cp, const int *ri, int m, std::vector<int> &levelPtr, std::vector<int> &item) {
    return bfs_levels(cp, ri, m, levelPtr, item);
}

int auto_lv(int m, int device_id) {
    // main.cu:245-254: smallest li >= 1 with m / 2^(li+1) below the wave size
    int li;
    for (li = 1; li <= 100; ++li)
        if (m / std::pow(2.0, li + 1) < (device_id == 0 ? 92160 : 58880)) break;
    return li;
}

int analyse_host(Plan &P, const int *ptr, const int *idx, const double *val, int n, int nnz, int fmt,
                 int substitution, int lv, const rbs_options &opt, std::string &err,
                 const std::vector<int> *seg_rows) {
    auto t0 = std::chrono::steady_clock::now();
    if (n <= 0 || nnz < n || !ptr || !idx || !val) {
        err = "rbs_analyse: need n > 0, nnz >= n and non-null arrays";
        return RBS_ERR_ARG;
    }
    if (substitution != RBS_FORWARD && substitution != RBS_BACKWARD) {
        err = "rbs_analyse: substitution must be RBS_FORWARD or RBS_BACKWARD";
        return RBS_ERR_ARG;
    }
    if (fmt != RBS_FMT_CSC && fmt != RBS_FMT_CSR) {
        err = "rbs_analyse: fmt must be RBS_FMT_CSC or RBS_FMT_CSR";
        return RBS_ERR_ARG;
    }
    if (ptr[0] != 0 || ptr[n] != nnz) {
        err = "rbs_analyse: pointer array must start at 0 and end at nnz";
        return RBS_ERR_STRUCTURE;
    }
    if (long long c = first_bad(n, [&](long long c) { return ptr[c + 1] < ptr[c]; }); c >= 0) {
        err = "rbs_analyse: pointer array decreases at " + std::to_string(c);
        return RBS_ERR_STRUCTURE;
    }
    if (long long k = first_bad(nnz, [&](long long k) { return idx[k] < 0 || idx[k] >= n; }); k >= 0) {
        err = "rbs_analyse: index out of range at entry " + std::to_string(k);
        return RBS_ERR_STRUCTURE;
    }
    P.opt = opt;
    P.n = n;
    P.nnz = nnz;
    P.sub = substitution;
    // 1. the reference's input layout: CSC with the diagonal first (forward)
    //    or last (backward) in every column
    if (fmt == RBS_FMT_CSR) {
        transpose(n, n, ptr, idx, val, P.in_cp, P.in_ri, P.in_va);
    } else {
        P.in_cp.assign(ptr, ptr + n + 1);
        P.in_ri.resize((size_t)nnz);
        P.in_va.resize((size_t)nnz);
        constexpr int kCopy = 1 << 22;  // entries per host-thread copy
        parallel_for(((size_t)nnz + kCopy - 1) / kCopy, [&](size_t i) {
            const size_t k0 = i * kCopy, len = std::min<size_t>(kCopy, (size_t)nnz - k0);
            std::memcpy(P.in_ri.data() + k0, idx + k0, len * sizeof(int));
            std::memcpy(P.in_va.data() + k0, val + k0, len * sizeof(double));
        });
    }
    const int *cp = P.in_cp.data(), *ri = P.in_ri.data();
    const double *va = P.in_va.data();
    // the first column that breaks a rule (found on host threads), then its
    // message from the checks below
    const long long bad_col = first_bad(n, [&](long long c) {
        const int b = cp[c], e = cp[c + 1];
        if (b == e) return true;
        const int dpos = substitution == RBS_FORWARD ? b : e - 1;
        if (ri[dpos] != c || va[dpos] == 0.0) return true;
        for (int k = b; k < e; ++k) {
            const int r = ri[k];
            if (!(substitution == RBS_FORWARD ? r >= c : r <= c) || (k != dpos && r == c)) return true;
        }
        return false;
    });
    for (int c = bad_col < 0 ? n : (int)bad_col; c < n; ++c) {
        int b = cp[c], e = cp[c + 1];
        if (b == e) {
            err = "rbs_analyse: column " + std::to_string(c) + " has no diagonal";
            return RBS_ERR_STRUCTURE;
        }
        int dpos = substitution == RBS_FORWARD ? b : e - 1;
        if (ri[dpos] != c) {
            err = "rbs_analyse: diagonal of column " + std::to_string(c) + " missing or not " +
                  (substitution == RBS_FORWARD ? "first" : "last");
            return RBS_ERR_STRUCTURE;
        }
        if (va[dpos] == 0.0) {
            err = "rbs_analyse: zero diagonal in column " + std::to_string(c);
            return RBS_ERR_STRUCTURE;
        }
        for (int k = b; k < e; ++k) {
            int r = ri[k];
            bool ok = substitution == RBS_FORWARD ? r >= c : r <= c;
            if (!ok) {
                err = "rbs_analyse: entry (" + std::to_string(r) + "," + std::to_string(c) + ") outside the " +
                      (substitution == RBS_FORWARD ? "lower" : "upper") + " triangle";
                return RBS_ERR_STRUCTURE;
            }
            if (k != dpos && r == c) {
                err = "rbs_analyse: duplicate diagonal in column " + std::to_string(c);
                return RBS_ERR_STRUCTURE;
            }
        }
    }
    // 3. level sets in the reference's discovery order
    int nlevel = bfs_levels(cp, ri, n, P.bfs_ptr, P.bfs_item);
    if (nlevel < 0) {
        err = "rbs_analyse: level search stuck (dependency cycle)";
        return RBS_ERR_STRUCTURE;
    }
    P.nlevel = nlevel;
    // labels (utils_reordering.h:130-159) and processing positions
    P.label.resize(n);
    P.perm.resize(n);
    std::vector<int> pos_of((size_t)n);
    constexpr int kLab = 1 << 16;  // positions per host-thread chunk (the level order is a permutation)
    parallel_for(((size_t)n + kLab - 1) / kLab, [&](size_t ch) {
        for (int i = (int)ch * kLab; i < std::min(n, (int)ch * kLab + kLab); ++i) {
            int orig = P.bfs_item[i];
            P.label[orig] = substitution == RBS_FORWARD ? i : n - 1 - i;
            P.perm[i] = orig;  // processing position i is BFS position i in both directions
            pos_of[orig] = i;
        }
    });

    // 4. processing-order CSR with columns ascending (the result of a stable
    //    sort by processing column and then by row), row by row from the
    //    input rows (CSR input) or from the CSC's stable transpose
    if (fmt == RBS_FMT_CSR) {
        full_csr_from_rows(P, ptr, idx, val, pos_of);
    } else {
        std::vector<int> rp;
        bulk_vector<int> rc;
        bulk_vector<double> rv;
        transpose(n, n, cp, ri, va, rp, rc, rv);
        full_csr_from_rows(P, rp.data(), rc.data(), rv.data(), pos_of);
    }
    P.analyse_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return analyse_after_levels(P, n, nnz, substitution, lv, opt, err, seg_rows);
}

// Steps after the level sets: recursion depth, blocks, statistics, kernel
// choice and pools, from the processing-order CSR (full_rp/col/val), the
// BFS order and the labels -- computed by analyse_host above or on the
// device (dev_analysis.cu).
int analyse_after_levels(Plan &P, int n, int nnz, int substitution, int lv, const rbs_options &opt, std::string &err,
                         const std::vector<int> *seg_rows, DevRows *dev_rows) {
    auto t0 = std::chrono::steady_clock::now();
    (void)nnz;
    P.opt = opt;
    P.n = n;
    P.nnz = nnz;
    P.sub = substitution;
    P.seg_rows.clear();
    if (seg_rows) P.seg_rows = *seg_rows;
    // 2. recursion depth (main.cu:245-254 for lv == -1)
    if (lv == -1) {
        lv = auto_lv(n, opt.lv_device_id);
        while (lv > 0 && (1 << lv) > n) --lv;
    }
    if (lv < 0 || lv > 24 || (1 << lv) > n) {
        err = "rbs_analyse: lv must satisfy 0 <= lv and 2^lv <= n";
        return RBS_ERR_ARG;
    }
    P.lv = lv;
    const int T = 1 << lv;
    P.sum_block = 2 * T - 1;
    P.step = n / T;
    const int s = P.step;

    const int *frp = P.full_rp.data(), *fcol = P.full_col.data();
    const double *fval = P.full_val.data();

    // 5. blocks in processing coordinates
    auto tri_of = [&](int p) { return std::min(p / s, T - 1); };
    P.blocks.assign((size_t)P.sum_block, ExecBlock{});
    for (int b = 0; b < P.sum_block; ++b) {
        ExecBlock &B = P.blocks[b];
        B.index = b;
        B.tri = (b & 1) == 0;
        B.rows_off = B.long_off = B.med_off = B.map_off = B.lvl_off = -1;
        B.medrows = 0;
        B.band_w = B.band_c = B.band_nch = 0;
        B.band_off = -1;
        B.ell_ok = B.ell_nchunks = 0;
        B.ell_chunk_off = B.ell_lo = B.ell_hi = -1;
        B.ca_ok = B.ca_w = B.ca_win = 0;
        B.ca_tab_off = B.ca_lo = B.ca_hi = -1;
        B.lc_ok = B.lc_nseg = 0;
        B.lc_seg_off = -1;
        B.lvl_var = LVL_PLAIN;
        if (B.tri) {
            int i = b / 2;
            B.r0 = i * s;
            B.m = (i == T - 1 ? n : (i + 1) * s) - B.r0;
            B.c0 = B.r0;
            B.ncols = B.m;
        } else {
            int t = (b + 1) / 2, lb = lowbit(t);
            B.r0 = t * s;
            B.m = (t + lb == T ? n : (t + lb) * s) - B.r0;
            B.c0 = (t - lb) * s;
            B.ncols = t * s - B.c0;
        }
    }
    // per-row entry counts of every block, local levels, bandwidth
    std::vector<std::vector<int>> rowcnt((size_t)P.sum_block);
    for (int b = 0; b < P.sum_block; ++b) rowcnt[b].assign((size_t)P.blocks[b].m, 0);
    std::vector<int> level((size_t)n, 0), reach((size_t)n);
    P.inv_diag.resize((size_t)n);
    // (block, row) slots in block order, for the device path
    std::vector<long long> slot_base((size_t)P.sum_block + 1, 0);
    for (int b = 0; b < P.sum_block; ++b) slot_base[(size_t)b + 1] = slot_base[(size_t)b] + P.blocks[b].m;
    constexpr int kRows = 1 << 14;
    if (dev_rows) {
        // counts, inverse diagonals, reach and local levels on the device (dev_pools.cu)
        std::vector<int> flat;
        int rc = dev_block_counts(*dev_rows, T, s, slot_base, flat, P.inv_diag, reach, err);
        if (rc) return rc;
        for (int b = 0; b < P.sum_block; ++b)
            std::copy(flat.begin() + slot_base[(size_t)b], flat.begin() + slot_base[(size_t)b + 1], rowcnt[b].begin());
        // chain-like graphs (the level search itself ran on the host): the
        // recurrence below on the host, a dependency at a time on the device
        // would cost an L2 round trip per row
        if (T > 1 && P.device_bfs && (rc = dev_local_levels(*dev_rows, T, s, opt.spin_limit, level, err))) return rc;
    } else
    // counts, inverse diagonals and the reach p - (first column) of every row
    // on host threads (row p owns row p of every block it meets) ...
    parallel_for(((size_t)n + kRows - 1) / kRows, [&](size_t chunk) {
        for (int p = (int)chunk * kRows; p < std::min(n, (int)chunk * kRows + kRows); ++p) {
            int i = tri_of(p);
            int tb = 2 * i;
            const ExecBlock &TB = P.blocks[tb];
            int minq = p;
            for (int k = frp[p]; k < frp[p + 1]; ++k) {
                int q = fcol[k];
                if (q == p) {
                    P.inv_diag[p] = 1.0 / fval[k];
                    continue;
                }
                if (q >= TB.r0) {
                    rowcnt[tb][p - TB.r0]++;
                    minq = std::min(minq, q);
                } else {
                    int j = tri_of(q);
                    int h = 31 - __builtin_clz((unsigned)(i ^ j));
                    int t = i & ~((1 << h) - 1);
                    int sb = 2 * t - 1;
                    rowcnt[sb][p - P.blocks[sb].r0]++;
                }
            }
            reach[p] = p - minq;
        }
    });
    // ... then the local levels: a recurrence in row order within each
    // triangle (triangles on host threads).  The local levels of a single
    // triangle are the level sets themselves (a row's level is one more than
    // the highest level among its dependencies in both).
    if (T == 1) {
        for (size_t L = 0; L + 1 < P.bfs_ptr.size(); ++L)
            std::fill(level.begin() + P.bfs_ptr[L], level.begin() + P.bfs_ptr[L + 1], (int)L);
    } else if (!dev_rows || !P.device_bfs) {
        parallel_for((size_t)T, [&](size_t i) {
            const ExecBlock &TB = P.blocks[2 * i];
            for (int p = TB.r0; p < TB.r0 + TB.m; ++p) {
                int lvmax = -1;
                for (int k = frp[p]; k < frp[p + 1]; ++k) {
                    const int q = fcol[k];
                    if (q != p && q >= TB.r0) lvmax = std::max(lvmax, level[q]);
                }
                level[p] = lvmax + 1;
            }
        });
    }
    for (int p = 0; p < n; ++p) {
        ExecBlock &TB = P.blocks[2 * tri_of(p)];
        TB.bandwidth = std::max(TB.bandwidth, reach[p]);
    }
    // block statistics, the reference's method codes and the kernel choice:
    // blocks are independent, done on host threads
    std::vector<std::vector<int>> lvl_sizes((size_t)P.sum_block);
    parallel_for((size_t)P.sum_block, [&](size_t bi) {
        const int b = (int)bi;
        ExecBlock &B = P.blocks[b];
        long long tot = 0;
        int nonempty = 0, longrows = 0, lenmax = B.m > 0 ? rowcnt[b][0] : 0;
        long long longlen = 0;
        for (int r = 0; r < B.m; ++r) {
            int c = rowcnt[b][r];
            tot += c;
            lenmax = std::max(lenmax, c);
            if (c) {
                ++nonempty;
                if (c > kLongRow) {
                    ++longrows;
                    longlen += c;
                }
            }
        }
        if (B.tri) {
            B.nnz = (int)(tot + B.m);
            int nl = 0;
            for (int r = 0; r < B.m; ++r) nl = std::max(nl, level[B.r0 + r] + 1);
            B.nlv = B.nnz == B.m ? 1 : nl;  // recblocking_preprocess.h:478-479
            lvl_sizes[b].assign((size_t)B.nlv, 0);
            int contiguous = 1;
            for (int r = 0; r < B.m; ++r) {
                int L = B.nnz == B.m ? 0 : level[B.r0 + r];
                lvl_sizes[b][L]++;
                if (r > 0 && L < (B.nnz == B.m ? 0 : level[B.r0 + r - 1])) contiguous = 0;
            }
            B.contiguous = contiguous;
            B.maxwidth = *std::max_element(lvl_sizes[b].begin(), lvl_sizes[b].end());
            // recblocking_preprocess.h:472-709
            if (B.nnz == B.m) B.ref_method = 0;
            else {
                int nnzr = B.nnz / B.m;
                if (B.nlv > 20000) B.ref_method = 1;
                else if ((nnzr <= 15 && B.nlv <= 20) || (nnzr == 1 && B.nlv <= 100)) B.ref_method = 2;
                else B.ref_method = 3;
            }
        } else {
            B.nnz = (int)tot;
            B.nonempty = nonempty;
            B.longrows = longrows;
            B.lenmax = lenmax;
            // recblocking_preprocess.h:824-922 (an empty square divides by zero there)
            if (B.nnz == 0) B.ref_method = -1;
            else {
                int nnzr = (int)((B.nnz - longlen) / nonempty);
                double empty_ratio = 100 * (double)(B.m - nonempty) / (double)B.m;
                if (nnzr <= 12 && empty_ratio <= 50) B.ref_method = 0;
                else if (nnzr <= 12 && empty_ratio > 50) B.ref_method = 1;
                else if (nnzr > 12 && empty_ratio <= 15) B.ref_method = 2;
                else B.ref_method = 3;
            }
        }
        select_kernel(B, opt, lvl_sizes[b]);
        // The sync-free kernel's lane group.  A deep triangle (32 levels or
        // more) is bound by its level chain, where each level waits for its
        // longest rows: there the group is sized for the rows' tail, the
        // 99th percentile at about 2 entries per lane (the power-law
        // factor's deepest backward triangle, 74 levels with a 99th
        // percentile of 18, runs at 16 lanes in 0.21 ms against 0.35 ms at
        // the mean's 2).  A shallow triangle is bound by its rows'
        // throughput, and extra lanes only add warps that idle on its short
        // rows (21 levels with a 99th percentile of 10: 57 us at 1 lane,
        // 70 us at 4), so it keeps the group for the mean.
        B.sf_group = B.group;
        if (B.tri && B.nnz > B.m && B.m > 0 && B.nlv >= 32) {
            std::vector<int> t(rowcnt[b].begin(), rowcnt[b].end());
            const size_t k = (size_t)((double)(t.size() - 1) * 0.99);
            std::nth_element(t.begin(), t.begin() + (long long)k, t.end());
            int g = 1;
            while (g < 32 && g * 2 < t[k]) g <<= 1;
            B.sf_group = std::max(B.group, g);
        }
    });

    // 6. pools.  Squares use a row list (DCSR) when more than half of their
    //    rows are empty; rows longer than 2048 go to the split kernel.
    P.rp_pool.clear();
    P.col_pool.clear();
    P.val_pool.clear();
    P.lvl_pool.clear();
    P.map_pool.clear();
    P.rows_pool.clear();
    long long total_entries = 0;
    for (int b = 0; b < P.sum_block; ++b) total_entries += P.blocks[b].tri ? P.blocks[b].nnz - P.blocks[b].m : P.blocks[b].nnz;
    P.col_pool.reserve((size_t)total_entries);
    P.val_pool.reserve((size_t)total_entries);
    // entry offset of every (block, local row) so the fill is one pass over
    // rows.  Blocks are independent: their sizes on host threads, then the
    // pools' offsets in block order, then every block fills its own parts
    // (row pointer, row lists, level pointer and map) on host threads.
    std::vector<std::vector<int>> rowstart((size_t)P.sum_block);
    struct PoolSizes {
        long long ent = 0;
        int nrows = 0, nlong = 0, nmed = 0;
        bool dcsr = false, med = false, lvl = false, map = false;
    };
    std::vector<PoolSizes> ps((size_t)P.sum_block);
    parallel_for((size_t)P.sum_block, [&](size_t bi) {
        const ExecBlock &B = P.blocks[bi];
        PoolSizes &z = ps[bi];
        const std::vector<int> &rc = rowcnt[bi];
        z.dcsr = !B.tri && B.kernel == RBS_K_SPMV &&
                 (opt.select == RBS_SELECT_REFERENCE ? (B.ref_method == 1 || B.ref_method == 3) : 2 * B.nonempty < B.m);
        z.med = !B.tri && B.kernel == RBS_K_SPMV && B.group < 32 && B.lenmax > kMedRow;
        int nonempty = 0;
        for (int r = 0; r < B.m; ++r) {
            const int c = rc[r];
            z.ent += c;
            nonempty += c != 0;
            z.nlong += c > kLongRow;
            z.nmed += c > kMedRow && c <= kLongRow;
        }
        z.nrows = z.dcsr ? nonempty : B.m;
        z.lvl = wants_level(B, opt);
        z.map = z.lvl && !B.contiguous;
    });
    long long ent = 0, rp_n = 0, rows_n = 0, lvl_n = 0, map_n = 0;
    std::vector<long long> ent0((size_t)P.sum_block), rows_dcsr0((size_t)P.sum_block);
    for (int b = 0; b < P.sum_block; ++b) {
        ExecBlock &B = P.blocks[b];
        const PoolSizes &z = ps[(size_t)b];
        ent0[(size_t)b] = ent;
        ent += z.ent;
        B.rp_off = rp_n;
        rp_n += (long long)z.nrows + 1;
        B.nrows = z.nrows;
        rows_dcsr0[(size_t)b] = rows_n;
        if (z.dcsr) {
            B.rows_off = rows_n;
            rows_n += z.nrows;
        }
        if (!B.tri && B.longrows) {
            // positions in the row pointer: the row for CSR, the list index for DCSR
            B.long_off = rows_n;
            rows_n += z.nlong;
        }
        if (z.med) {
            // single RHS: rows of kMedRow+1..kLongRow entries take a warp each
            B.med_off = z.nmed ? rows_n : -1;
            B.medrows = z.nmed;
            rows_n += z.nmed;
        }
        if (z.lvl) {
            B.lvl_off = lvl_n;
            lvl_n += (long long)B.nlv + 1;
            if (z.map) {
                B.map_off = map_n;
                map_n += B.m;
            }
        }
    }
    P.rp_pool.resize((size_t)rp_n);
    P.rows_pool.resize((size_t)rows_n);
    P.lvl_pool.resize((size_t)lvl_n);
    P.map_pool.resize((size_t)map_n);
    parallel_for((size_t)P.sum_block, [&](size_t bi) {
        const int b = (int)bi;
        const ExecBlock &B = P.blocks[bi];
        const PoolSizes &z = ps[bi];
        const std::vector<int> &rc = rowcnt[bi];
        std::vector<int> &rs = rowstart[bi];
        rs.resize((size_t)B.m + 1);
        rs[0] = (int)ent0[bi];
        for (int r = 0; r < B.m; ++r) rs[(size_t)r + 1] = rs[(size_t)r] + rc[r];
        int *rp = P.rp_pool.data() + B.rp_off;
        if (z.dcsr) {
            int *rows = P.rows_pool.data() + rows_dcsr0[bi];
            int cnt = 0;
            for (int r = 0; r < B.m; ++r)
                if (rc[r]) {
                    rows[cnt] = r;
                    rp[cnt++] = rs[(size_t)r];
                }
            rp[cnt] = rs[(size_t)B.m];
        } else {
            for (int r = 0; r <= B.m; ++r) rp[r] = rs[(size_t)r];
        }
        if (!B.tri && B.longrows) {
            int *out = P.rows_pool.data() + B.long_off, pos = 0, k = 0;
            for (int r = 0; r < B.m; ++r) {
                if (z.dcsr && rc[r] == 0) continue;
                if (rc[r] > kLongRow) out[k++] = pos;
                ++pos;
            }
        }
        if (z.med && z.nmed) {
            int *out = P.rows_pool.data() + B.med_off, pos = 0, k = 0;
            for (int r = 0; r < B.m; ++r) {
                if (z.dcsr && rc[r] == 0) continue;
                if (rc[r] > kMedRow && rc[r] <= kLongRow) out[k++] = pos;
                ++pos;
            }
        }
        if (z.lvl) {
            int *lp = P.lvl_pool.data() + B.lvl_off;
            lp[0] = 0;
            for (int L = 0; L < B.nlv; ++L) lp[L + 1] = lp[L] + lvl_sizes[bi][L];
            if (z.map) {
                std::vector<int> fillL(lp, lp + B.nlv);
                int *mp = P.map_pool.data() + B.map_off;
                for (int r = 0; r < B.m; ++r) {
                    const int L = B.nnz == B.m ? 0 : level[B.r0 + r];
                    mp[fillL[L]++] = r;
                }
            }
        }
        (void)b;
    });
    if (dev_rows) {  // the entry pools filled on the device
        int rc = dev_pool_fill(*dev_rows, T, s, slot_base[(size_t)P.sum_block], ent, P.col_pool, P.val_pool, err);
        if (rc) return rc;
    } else {
    P.col_pool.resize((size_t)ent);
    P.val_pool.resize((size_t)ent);
        std::vector<std::vector<int>> cur((size_t)P.sum_block);
        for (int b = 0; b < P.sum_block; ++b) cur[b].assign(rowstart[b].begin(), rowstart[b].end() - 1);
        // row p owns row p of every block it meets: rows filled on host threads
        constexpr int kRows = 1 << 14;
        parallel_for(((size_t)n + kRows - 1) / kRows, [&](size_t chunk) {
            for (int p = (int)chunk * kRows; p < std::min(n, (int)chunk * kRows + kRows); ++p) {
                int i = tri_of(p);
                int tb = 2 * i;
                const ExecBlock &TB = P.blocks[tb];
                for (int k = frp[p]; k < frp[p + 1]; ++k) {
                    int q = fcol[k];
                    if (q == p) continue;
                    int b, lc;
                    if (q >= TB.r0) {
                        b = tb;
                        lc = q - TB.r0;
                    } else {
                        int j = tri_of(q);
                        int h = 31 - __builtin_clz((unsigned)(i ^ j));
                        int t = i & ~((1 << h) - 1);
                        b = 2 * t - 1;
                        lc = q - P.blocks[b].c0;
                    }
                    int d = cur[b][p - P.blocks[b].r0]++;
                    P.col_pool[d] = lc;
                    P.val_pool[d] = fval[k];
                }
            }
        });
    }
    // 7. band layout of band-scan triangles: row r of the block is row
    //    i = r % C of chunk j = r / C; its coefficient of x_{r-1-d} sits at
    //    band_coef[band_off + (i*nch + j)*W + d], its inverse diagonal at
    //    band_inv[band_off/W + i*nch + j].
    P.band_coef.clear();
    P.band_inv.clear();
    for (ExecBlock &B : P.blocks) {
        if (!wants_band(B, opt)) continue;
        int W = 1;
        while (W < std::max(1, B.bandwidth)) W <<= 1;
        B.band_w = W;
        // rows per chunk: halved from 16 while the triangle has fewer chunks
        // than two CTAs of 256 per SM of a 148-SM part would take, down to
        // max(4, W) rows (below W the chunks' share of the scans outweighs
        // their row steps); 125,000 rows: 4-row chunks, 123 CTAs
        B.band_c = 16;
        while (B.band_c > std::max(4, W) && ((long long)B.m + B.band_c - 1) / B.band_c < 2LL * 148 * 256)
            B.band_c >>= 1;
        B.band_nch = (B.m + B.band_c - 1) / B.band_c;
        B.band_off = (long long)P.band_coef.size();
        const long long slots = (long long)B.band_nch * B.band_c;
        P.band_coef.resize(P.band_coef.size() + (size_t)(slots * W), 0.0);
        P.band_inv.resize(P.band_inv.size() + (size_t)slots, 0.0);
        const long long inv_off = B.band_off / W;
        for (int r = 0; r < B.m; ++r) {
            const long long o = (long long)(r % B.band_c) * B.band_nch + r / B.band_c;
            P.band_inv[(size_t)(inv_off + o)] = P.inv_diag[(size_t)B.r0 + r];
            const int s0 = P.rp_pool[(size_t)B.rp_off + r], s1 = P.rp_pool[(size_t)B.rp_off + r + 1];
            for (int k = s0; k < s1; ++k) {
                const int d = r - P.col_pool[k] - 1;
                P.band_coef[(size_t)(B.band_off + o * W + d)] += P.val_pool[k];
            }
        }
    }
    // 10. level-ELL layout of level triangles with narrow levels (<= 1024
    //     rows) and short rows (<= 4 entries): the cp.async-staged kernel
    //     (level_ca.cuh).  Per level a table entry {lo, off, w, 0}; the block's
    //     ELL width W in {1, 2, 4}; entry j of row lo+i at off + i*W + j
    //     (row-major, padding column -1), blocks start on a 4-entry boundary.
    P.ca_tab.clear();
    P.ca_col.clear();
    P.ca_val.clear();
    for (ExecBlock &B : P.blocks) {
        if (!wants_level(B, opt) || !B.contiguous) continue;
        const int *rp = P.rp_pool.data() + B.rp_off;
        const int *lvp = P.lvl_pool.data() + B.lvl_off;
        int wmax = 0;
        bool ok = true;
        for (int l = 0; l < B.nlv && ok; ++l) {
            if (lvp[l + 1] - lvp[l] > 1024) ok = false;
            for (int r = lvp[l]; r < lvp[l + 1]; ++r) wmax = std::max(wmax, rp[r + 1] - rp[r]);
        }
        if (!ok || wmax > 4) continue;
        const int W = wmax <= 1 ? 1 : wmax <= 2 ? 2 : 4;
        B.ca_ok = 1;
        B.ca_w = W;
        while (P.ca_col.size() % 4) {
            P.ca_col.push_back(-1);
            P.ca_val.push_back(0.0);
        }
        B.ca_tab_off = (long long)P.ca_tab.size();
        B.ca_lo = (long long)P.ca_col.size();
        for (int l = 0; l < B.nlv; ++l) {
            const int lo = lvp[l], w = lvp[l + 1] - lo;
            P.ca_tab.insert(P.ca_tab.end(), {lo, (int)((long long)lo * W), w, 0});
        }
        P.ca_tab.insert(P.ca_tab.end(), {B.m, (int)((long long)B.m * W), 0, 0});
        P.ca_col.resize(P.ca_col.size() + (size_t)B.m * W, -1);
        P.ca_val.resize(P.ca_val.size() + (size_t)B.m * W, 0.0);
        for (int r = 0; r < B.m; ++r)
            for (int j = 0; j < rp[r + 1] - rp[r]; ++j) {
                const size_t dst = (size_t)(B.ca_lo + (long long)r * W + j);
                P.ca_col[dst] = P.col_pool[rp[r] + j];
                P.ca_val[dst] = P.val_pool[rp[r] + j];
            }
        B.ca_hi = (long long)P.ca_col.size();
        // window-only blocks: every dependency of level l lies in
        // [hi_l - CA_WINDOW_ROWS, lo_l); columns become window slots
        bool win = true;
        for (int l = 0; l < B.nlv && win; ++l)
            for (int r = lvp[l]; r < lvp[l + 1] && win; ++r)
                for (int j = 0; j < rp[r + 1] - rp[r]; ++j)
                    if (P.col_pool[rp[r] + j] < lvp[l + 1] - CA_WINDOW_ROWS) win = false;
        if (win) {
            B.ca_win = 1;
            for (long long e = B.ca_lo; e < B.ca_hi; ++e)
                P.ca_col[(size_t)e] = P.ca_col[(size_t)e] < 0 ? CA_WINDOW_ROWS
                                                             : (P.ca_col[(size_t)e] & (CA_WINDOW_ROWS - 1));
        }
    }
    if (P.ca_col.size() > (size_t)0x7fffffff) {
        err = "rbs_analyse: ELL pool too large";
        return RBS_ERR_NOMEM;
    }
    // 11. level-chunk records (level_lc.cuh) and the level kernel of every
    //     level triangle
    build_lc(P, opt, level);
    // 12. ELL chunks of single-CTA triangles (the CTA sync-free kernel,
    //    cta_syncfree.cuh): chunks of <= 512 rows and <= 2048 ELL slots,
    //    column-major inside a chunk, padding column -1; built after the
    //    staged and chunk layouts, for the triangles that have neither (or,
    //    when tuning, for every candidate)
    P.ell_col.clear();
    P.ell_val.clear();
    P.ell_chunks.clear();
    constexpr int RMAX = 512, EMAX = 2048;
    // chunk bounds and pool offsets first (chunk starts 16-byte aligned),
    // then the pool filled chunk by chunk on host threads
    std::vector<int> ell_blocks;
    long long ell_size = 0;
    for (ExecBlock &B : P.blocks) {
        if (!wants_level(B, opt)) continue;
        // only the kernel choice's fallback outside tuning: a triangle with a
        // staged or chunk layout never runs this kernel then
        if (opt.select != RBS_SELECT_TUNE && (B.ca_ok || B.lc_ok)) continue;
        const int *rp = P.rp_pool.data() + B.rp_off;
        std::vector<int> cuts{0}, widths;
        bool ok = true;
        int w = 0, rows = 0;
        for (int r = 0; r < B.m && ok; ++r) {
            const int len = rp[r + 1] - rp[r];
            if (len > EMAX) ok = false;
            const int w2 = std::max(w, len);
            if (rows == RMAX || (long long)(rows + 1) * w2 > EMAX) {
                cuts.push_back(r);
                widths.push_back(w);
                w = len;
                rows = 1;
            } else {
                w = w2;
                ++rows;
            }
        }
        if (!ok) continue;
        cuts.push_back(B.m);
        widths.push_back(w);
        const int nch = (int)widths.size();
        B.ell_ok = 1;
        B.ell_nchunks = nch;
        B.ell_chunk_off = (long long)P.ell_chunks.size() / 4;
        B.ell_lo = ell_size;
        for (int q = 0; q < nch; ++q) {
            ell_size = (ell_size + 3) & ~3LL;
            const int R0 = cuts[q], R1 = cuts[q + 1], W = widths[q];
            P.ell_chunks.insert(P.ell_chunks.end(), {R0, R1, W, (int)ell_size});
            ell_size += (long long)(R1 - R0) * W;
        }
        B.ell_hi = ell_size;
        ell_blocks.push_back(B.index);
    }
    if (ell_size > 0x7fffffffLL) {
        err = "rbs_analyse: ELL pool too large";
        return RBS_ERR_NOMEM;
    }
    P.ell_col.resize((size_t)ell_size);
    P.ell_val.resize((size_t)ell_size);
    {
        // chunk i of the pool fills its slots and the alignment gap before it
        std::vector<std::pair<int, int>> where;  // (block, chunk) of every pool chunk in order
        for (int b : ell_blocks)
            for (int q = 0; q < P.blocks[(size_t)b].ell_nchunks; ++q) where.push_back({b, q});
        parallel_for(where.size(), [&](size_t i) {
            const ExecBlock &B = P.blocks[(size_t)where[i].first];
            const int *ch = P.ell_chunks.data() + 4 * (B.ell_chunk_off + where[i].second);
            const int R0 = ch[0], R = ch[1] - ch[0], W = ch[2];
            const long long off = ch[3];
            const long long gap0 = i == 0 ? 0 : (where[i].second == 0 ? P.blocks[(size_t)where[i - 1].first].ell_hi
                                                                       : (long long)ch[-1] + (long long)(ch[-3] - ch[-4]) * ch[-2]);
            std::fill(P.ell_col.begin() + gap0, P.ell_col.begin() + off + (long long)R * W, -1);
            std::fill(P.ell_val.begin() + gap0, P.ell_val.begin() + off + (long long)R * W, 0.0);
            const int *rp = P.rp_pool.data() + B.rp_off;
            for (int t = 0; t < R; ++t) {
                const int r = R0 + t;
                for (int j = 0; j < rp[r + 1] - rp[r]; ++j) {
                    P.ell_col[(size_t)(off + (long long)j * R + t)] = P.col_pool[rp[r] + j];
                    P.ell_val[(size_t)(off + (long long)j * R + t)] = P.val_pool[rp[r] + j];
                }
            }
        });
    }
    for (ExecBlock &B : P.blocks) {
        if (!B.tri || B.kernel != RBS_K_LEVEL) continue;
        // staged level-ELL first (short rows, narrow levels: its per-level cost
        // is lowest), then level chunks, then the CTA sync-free and plain kernels
        B.lvl_var = B.ca_ok ? LVL_CA : B.lc_ok ? LVL_LC : B.ell_ok ? LVL_CSF : LVL_PLAIN;
    }
    auto t1 = std::chrono::steady_clock::now();
    P.analyse_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
    return RBS_OK;
}

// The reference-format packing of recblocking_preprocess.h:298-967 (see
// export_reference): the level-permuted CSC, every block cut out with the
// reference's bounds filter and packed into recblock_Ptr/Index/Val and the
// DCSR row lists, local level sets of the triangles.
static int build_ref_pack(const Plan &P, bool fwd, const std::vector<int> &blk_m, const std::vector<int> &blk_n,
                          const std::vector<int> &blk_nnz, const std::vector<int> &stu, const std::vector<int> &std_,
                          const std::vector<int> &sru, const std::vector<int> &srd, const std::vector<int> &srl,
                          const std::vector<int> &srr, const std::vector<int> &method, RefPack &R,
                          std::string &err) {
    const int n = P.n, nnz = P.nnz, sum = P.sum_block;
    std::vector<int> cp_new((size_t)n + 1), ri_new((size_t)nnz);
    std::vector<double> va_new((size_t)nnz);
    cp_new[0] = 0;
    for (int i = 0; i < n; ++i) {
        int src = fwd ? P.bfs_item[i] : P.bfs_item[n - 1 - i];
        int len = P.in_cp[src + 1] - P.in_cp[src];
        cp_new[i + 1] = cp_new[i] + len;
        for (int j = 0; j < len; ++j) {
            ri_new[cp_new[i] + j] = P.label[P.in_ri[P.in_cp[src] + j]];
            va_new[cp_new[i] + j] = P.in_va[P.in_cp[src] + j];
        }
    }
    auto &ptr_offset = R.ptr_offset, &index_offset = R.index_offset, &dcsr_offset = R.dcsr_offset;
    ptr_offset.assign(sum + 1, 0);
    index_offset.assign(sum + 1, 0);
    dcsr_offset.assign(sum + 1, 0);
    int ps = 1, is = 0, ds = 0;
    for (int b = 0; b < sum; ++b) {
        if ((b & 1) == 0) { ps += blk_n[b] + 1; is += blk_nnz[b]; }
        else { ps += blk_m[b]; is += blk_nnz[b]; ds += blk_m[b]; }
    }
    auto &Ptr = R.Ptr, &Index = R.Index, &Dcsr = R.Dcsr;
    auto &Val = R.Val;
    auto &nlv = R.nlv, &longrow = R.longrow, &m_new_dcsr = R.m_new_dcsr;
    auto &lvl_ptr = R.lvl_ptr, &lvl_item = R.lvl_item, &m_lv = R.m_lv, &off_lv = R.off_lv, &nnz_lv = R.nnz_lv;
    Ptr.assign((size_t)ps, 0);
    Index.assign((size_t)std::max(is, 1), 0);
    Dcsr.assign((size_t)std::max(ds, 1), 0);
    Val.assign((size_t)std::max(is, 1), 0.0);
    nlv.assign(sum, 0);
    longrow.assign(sum, 0);
    m_new_dcsr.assign(sum, -1);
    ptr_offset[0] = 1;
    index_offset[0] = 0;
    dcsr_offset[0] = 0;
    int nz = 0;
    for (int b = 0; b < sum; ++b) {
        const int bm = blk_m[b], bn = blk_n[b];
        int po = ptr_offset[b];
        std::vector<int> scp((size_t)bn + 1, 0), sri;
        std::vector<double> sva;
        if ((b & 1) == 0) {
            int up = stu[b], down = std_[b];
            for (int c = up; c < down; ++c) {
                for (int k = cp_new[c]; k < cp_new[c + 1]; ++k) {
                    int r = ri_new[k];
                    if (fwd ? r < down : r >= up) {
                        sri.push_back(r - up);
                        sva.push_back(va_new[k]);
                    }
                }
                scp[(size_t)(c - up) + 1] = (int)sri.size();
            }
            std::vector<int> rrp, rci;
            std::vector<double> rva;
            transpose(bn, bm, scp.data(), sri.data(), sva.data(), rrp, rci, rva);
            std::vector<int> lp, li;
            int nl = 1;
            if (bm == (int)sri.size()) {
                lp = {0, bm};
                li.resize((size_t)bm);
                for (int i = 0; i < bm; ++i) li[i] = i;
            } else {
                nl = bfs_levels(scp.data(), sri.data(), bm, lp, li);
                if (nl < 0) { err = "export: local level search stuck"; return RBS_ERR_STRUCTURE; }
            }
            nlv[b] = nl;
            lvl_ptr.insert(lvl_ptr.end(), lp.begin(), lp.end());
            lvl_item.insert(lvl_item.end(), li.begin(), li.end());
            int meth = method[b];
            if (meth == 0 || meth == 3) {
                for (int i = 0; i < bn; ++i) {
                    for (int k = scp[i]; k < scp[i + 1]; ++k) { Index[nz] = sri[k]; Val[nz] = sva[k]; ++nz; }
                    Ptr[po + i] = Ptr[po + i - 1] + scp[i + 1] - scp[i];
                }
            } else if (meth == 2) {
                for (int l = 0; l < nl; ++l) {
                    m_lv.push_back(lp[l + 1] - lp[l]);
                    off_lv.push_back(lp[l]);
                    int sacc = 0;
                    for (int q = lp[l]; q < lp[l + 1]; ++q) sacc += rrp[q + 1] - rrp[q];
                    nnz_lv.push_back(sacc);
                }
                for (int i = 0; i < bm; ++i) {
                    for (int k = rrp[i]; k < rrp[i + 1]; ++k) { Index[nz] = rci[k]; Val[nz] = rva[k]; ++nz; }
                    Ptr[po + i] = Ptr[po + i - 1] + rrp[i + 1] - rrp[i];
                }
            } else {
                Ptr[po] = 0;
                int c = 0;
                for (int i = 0; i < bm; ++i) {
                    for (int k = rrp[i]; k < rrp[i + 1]; ++k) { Index[nz] = rci[k]; Val[nz] = rva[k]; ++nz; ++c; }
                    Ptr[po + i + 1] = c;
                }
            }
            ptr_offset[b + 1] = po + bm + (meth == 1 ? 1 : 0);
            index_offset[b + 1] = nz;
            dcsr_offset[b + 1] = dcsr_offset[b];
        } else {
            int up = sru[b], down = srd[b], left = srl[b], right = srr[b];
            for (int c = left; c < right; ++c) {
                for (int k = cp_new[c]; k < cp_new[c + 1]; ++k) {
                    int r = ri_new[k];
                    if (r >= up && r < down) {
                        sri.push_back(r - up);
                        sva.push_back(va_new[k]);
                    }
                }
                scp[(size_t)(c - left) + 1] = (int)sri.size();
            }
            std::vector<int> rrp, rci;
            std::vector<double> rva;
            transpose(bn, bm, scp.data(), sri.data(), sva.data(), rrp, rci, rva);
            for (int i = 0; i < bm; ++i)
                for (int k = rrp[i]; k < rrp[i + 1]; ++k) { Index[nz] = rci[k]; Val[nz] = rva[k]; ++nz; }
            int real_i = 0, dcsr_i = 0, meth = method[b];
            int lr = 0;
            for (int i = 0; i < bm; ++i)
                if (rrp[i + 1] - rrp[i] > kLongRow) ++lr;
            longrow[b] = meth >= 0 ? lr : 0;
            if (meth == 0 || meth == 2) {
                for (int i = 0; i < bm; ++i) Ptr[po + i] = Ptr[po + i - 1] + rrp[i + 1] - rrp[i];
                real_i = bm;
            } else if (meth == 1 || meth == 3) {
                for (int i = 0; i < bm; ++i)
                    if (rrp[i + 1] != rrp[i]) {
                        Ptr[po + dcsr_i] = Ptr[po + dcsr_i - 1] + rrp[i + 1] - rrp[i];
                        Dcsr[dcsr_offset[b] + dcsr_i] = i;
                        ++dcsr_i;
                    }
                real_i = dcsr_i;
                m_new_dcsr[b] = dcsr_i;
            }
            ptr_offset[b + 1] = po + real_i;
            index_offset[b + 1] = nz;
            dcsr_offset[b + 1] = dcsr_offset[b] + dcsr_i;
        }
    }
    return RBS_OK;
}

// ---------------------------------------------------------------------------
// Reference-format outputs, rebuilt from the plan on request.  This follows
// recblocking_preprocess.h:298-967 (get_recblock_size, L_preprocessing) and
// its U twin (:969-1474): the level-permuted CSC keeps each column's entry
// order, each block is cut out with the reference's bounds filter, triangles
// get their local level sets from the BFS and are packed as CSC (methods 0,3)
// or CSR (method 2, method 1 with a private zero-based pointer), squares as
// CSR or DCSR, and recblock_Ptr blocks share their first entry with the
// previous block's last entry.
// ---------------------------------------------------------------------------
int export_reference(const Plan &P, const std::string &name, std::vector<int> &iv, std::vector<double> &dv,
                     bool &is_double, std::string &err) {
    const int n = P.n, nnz = P.nnz, sum = P.sum_block;
    const bool fwd = P.sub == RBS_FORWARD;
    is_double = false;
    iv.clear();
    dv.clear();
    auto mirror = [&](int lo, int hi, int &a, int &b) {  // processing range -> reference range
        if (fwd) { a = lo; b = hi; } else { a = n - hi; b = n - lo; }
    };
    // geometry
    std::vector<int> loc_off(sum, 0), tmp_off(sum, 0), blk_m(sum), blk_n(sum), blk_nnz(sum);
    std::vector<int> stu(sum, -1), std_(sum, -1), sru(sum, -1), srd(sum, -1), srr(sum, -1), srl(sum, -1);
    std::vector<int> method(sum), kernel(sum), medrow(sum);
    for (int b = 0; b < sum; ++b) {
        const ExecBlock &B = P.blocks[b];
        blk_m[b] = B.m;
        blk_n[b] = B.ncols;
        blk_nnz[b] = B.nnz;
        method[b] = B.ref_method;
        kernel[b] = B.kernel;
        medrow[b] = B.medrows;
        if (B.tri) {
            mirror(B.r0, B.r0 + B.m, stu[b], std_[b]);
            loc_off[b] = stu[b];
        } else {
            mirror(B.r0, B.r0 + B.m, sru[b], srd[b]);
            mirror(B.c0, B.c0 + B.ncols, srl[b], srr[b]);
            tmp_off[b] = sru[b];
            loc_off[b] = srl[b];
        }
    }
    auto put = [&](const std::vector<int> &v) { iv = v; return RBS_OK; };
    if (name == "loc_off") return put(loc_off);
    if (name == "tmp_off") return put(tmp_off);
    if (name == "blk_m") return put(blk_m);
    if (name == "blk_n") return put(blk_n);
    if (name == "blk_nnz") return put(blk_nnz);
    if (name == "subtri_up") return put(stu);
    if (name == "subtri_down") return put(std_);
    if (name == "subrec_up") return put(sru);
    if (name == "subrec_down") return put(srd);
    if (name == "subrec_right") return put(srr);
    if (name == "subrec_left") return put(srl);
    if (name == "method") return put(method);
    if (name == "kernel") return put(kernel);
    if (name == "medrow") return put(medrow);  // per block: rows of the single-RHS warp-per-row pass
    if (name == "perm") return put(P.perm);
    if (name == "levelItem") {
        // utils_reordering.h:189-197: reversed for backward
        iv = P.bfs_item;
        if (!fwd) std::reverse(iv.begin(), iv.end());
        return RBS_OK;
    }
    if (name == "levelPtr") return put(P.bfs_ptr);
    if (name == "group") {
        iv.resize(sum);
        for (int b = 0; b < sum; ++b) iv[b] = P.blocks[b].group;
        return RBS_OK;
    }
    if (name == "local_nlv") {
        iv.resize(sum);
        for (int b = 0; b < sum; ++b) iv[b] = P.blocks[b].tri ? P.blocks[b].nlv : 0;
        return RBS_OK;
    }
    if (name == "ell_col") {
        iv.assign(P.ell_col.begin(), P.ell_col.end());
        return RBS_OK;
    }
    if (name == "ell_chunks") return put(P.ell_chunks);
    if (name == "ell_val") {
        is_double = true;
        dv.assign(P.ell_val.begin(), P.ell_val.end());
        return RBS_OK;
    }
    if (name == "ell_block") {  // per block: first chunk, chunk count (-1 if not ELL)
        iv.assign(2 * sum, -1);
        for (int b = 0; b < sum; ++b)
            if (P.blocks[b].ell_ok) {
                iv[2 * b] = (int)P.blocks[b].ell_chunk_off;
                iv[2 * b + 1] = P.blocks[b].ell_nchunks;
            }
        return RBS_OK;
    }
    if (name == "reordered_colptr" || name == "reordered_rowidx") {
        // the reference's level-permuted CSC (utils_reordering.h:102-187):
        // the device analysis's own arrays when it ran, else rebuilt here
        if (!P.dev_reorder_cp.empty()) return put(name == "reordered_colptr" ? P.dev_reorder_cp : P.dev_reorder_ri);
        std::vector<int> ncp((size_t)n + 1, 0), nri;
        nri.reserve((size_t)nnz);
        for (int i = 0; i < n; ++i) {
            const int src = P.bfs_item[(size_t)(fwd ? i : n - 1 - i)];
            for (int k = P.in_cp[(size_t)src]; k < P.in_cp[(size_t)src + 1]; ++k) nri.push_back(P.label[(size_t)P.in_ri[(size_t)k]]);
            ncp[(size_t)i + 1] = (int)nri.size();
        }
        return put(name == "reordered_colptr" ? ncp : nri);
    }
    if (name == "analyse_ms") {  // total analysis, of which on the device, level search on the device (1/0)
        is_double = true;
        dv = {P.analyse_ms, P.device_analyse_ms, (double)P.device_bfs};
        return RBS_OK;
    }
    if (name == "lc_consts") {  // the layout constants the records were built for
        iv = {LC_XW, LC_NB, LC_D, LC_RMAX, LC_T, LC_RING, LC_FMAX, LC_HDR_INTS};
        return RBS_OK;
    }
    // the execution pools' index arrays (row pointers, row lists, level
    // pointers and level maps of all blocks), for inspection
    if (name == "rp_pool") return put(P.rp_pool);
    if (name == "rows_pool") return put(P.rows_pool);
    if (name == "lvl_pool") return put(P.lvl_pool);
    if (name == "map_pool") return put(P.map_pool);
    if (name == "ca_tab") return put(P.ca_tab);
    if (name == "ca_col") return put(P.ca_col);
    if (name == "ca_val") {
        is_double = true;
        dv = P.ca_val;
        return RBS_OK;
    }
    if (name == "ca_block") {  // per block: table offset, first entry, ELL width, columns are window
                               // slots (1/0) (all -1: no level-ELL layout)
        iv.assign(4 * sum, -1);
        for (int b = 0; b < sum; ++b)
            if (P.blocks[b].ca_ok) {
                iv[4 * b] = (int)P.blocks[b].ca_tab_off;
                iv[4 * b + 1] = (int)P.blocks[b].ca_lo;
                iv[4 * b + 2] = P.blocks[b].ca_w;
                iv[4 * b + 3] = P.blocks[b].ca_win;
            }
        return RBS_OK;
    }
    if (name == "lc_tab") return put(P.lc_tab);
    if (name == "lc_segs") return put(P.lc_segs);
    if (name == "lc_rec64" || name == "lc_rec32") {  // 16-byte-aligned words, returned as int32
        const auto &w = name == "lc_rec64" ? P.lc_rec64 : P.lc_rec32;
        iv.resize(w.size());
        if (!w.empty()) std::memcpy(iv.data(), w.data(), w.size() * 4);
        return RBS_OK;
    }
    if (name == "lc_block") {  // per block: first segment, segments (-1 if none), level kernel variant
        iv.assign(3 * sum, -1);
        for (int b = 0; b < sum; ++b) {
            if (P.blocks[b].lc_ok) {
                iv[3 * b] = (int)P.blocks[b].lc_seg_off;
                iv[3 * b + 1] = P.blocks[b].lc_nseg;
            }
            iv[3 * b + 2] = P.blocks[b].lvl_var;
        }
        return RBS_OK;
    }
    if (name == "block_rows") {  // per block: processing-order first row, rows
        iv.resize(2 * sum);
        for (int b = 0; b < sum; ++b) {
            iv[2 * b] = P.blocks[b].r0;
            iv[2 * b + 1] = P.blocks[b].m;
        }
        return RBS_OK;
    }
    if (name == "inv_diag") {
        is_double = true;
        dv = P.inv_diag;
        return RBS_OK;
    }
    if (name == "block_bytes") {
        is_double = true;
        dv.resize(sum);
        for (int b = 0; b < sum; ++b) dv[b] = block_bytes(P, P.blocks[b]);
        return RBS_OK;
    }
    if (name == "sizes") {
        int ps = 1, is = 0, ds = 0;  // recblocking_preprocess.h:370-384
        for (int b = 0; b < sum; ++b) {
            if ((b & 1) == 0) { ps += blk_n[b] + 1; is += blk_nnz[b]; }
            else { ps += blk_m[b]; is += blk_nnz[b]; ds += blk_m[b]; }
        }
        iv = {ps, is, ds};
        return RBS_OK;
    }
    // Everything below needs the reference-order permuted CSC and the
    // per-block extraction: built once per plan, on the first request.
    if (!P.ref_pack) {
        auto pk = std::make_shared<RefPack>();
        int rc = build_ref_pack(P, fwd, blk_m, blk_n, blk_nnz, stu, std_, sru, srd, srl, srr, method, *pk, err);
        if (rc) return rc;
        P.ref_pack = pk;
    }
    const RefPack &R = *P.ref_pack;
    const auto &ptr_offset = R.ptr_offset, &index_offset = R.index_offset, &dcsr_offset = R.dcsr_offset;
    const auto &Ptr = R.Ptr, &Index = R.Index, &Dcsr = R.Dcsr;
    const auto &Val = R.Val;
    const auto &nlv = R.nlv, &longrow = R.longrow, &m_new_dcsr = R.m_new_dcsr;
    const auto &lvl_ptr = R.lvl_ptr, &lvl_item = R.lvl_item, &m_lv = R.m_lv, &off_lv = R.off_lv, &nnz_lv = R.nnz_lv;
    if (name == "ptr_offset") return put(ptr_offset);
    if (name == "index_offset") return put(index_offset);
    if (name == "dcsrindex_offset") return put(dcsr_offset);
    if (name == "recblock_Ptr") { iv.assign(Ptr.begin(), Ptr.begin() + ptr_offset[sum]); return RBS_OK; }
    if (name == "recblock_Index") { iv.assign(Index.begin(), Index.begin() + index_offset[sum]); return RBS_OK; }
    if (name == "recblock_dcsr_rowidx") { iv.assign(Dcsr.begin(), Dcsr.begin() + dcsr_offset[sum]); return RBS_OK; }
    if (name == "recblock_Val") {
        is_double = true;
        dv.assign(Val.begin(), Val.begin() + index_offset[sum]);
        return RBS_OK;
    }
    if (name == "nlv") return put(nlv);
    if (name == "longrow") return put(longrow);
    if (name == "m_new_dcsr") return put(m_new_dcsr);
    if (name == "lvl_ptr") return put(lvl_ptr);
    if (name == "lvl_item") return put(lvl_item);
    if (name == "m_lv") return put(m_lv);
    if (name == "offset_lv") return put(off_lv);
    if (name == "nnz_lv") return put(nnz_lv);
    err = "rbs_plan_export: unknown name '" + name + "'";
    return RBS_ERR_ARG;
}

}  // namespace rbs
