/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * CPU restatement of recblock-sptrsv's analysis (level sets, level-set
 * reordering, recursive-block geometry, per-block extraction, method choice
 * and packing) and of serial substitution.  Each function names the
 * reference lines it follows.  Paths are relative to the reference project
 * directory recblock-sptrsv/.
 */
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <sched.h>
#include <stdatomic.h>
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* utils.h:98-113 exclusive_scan, in place over `len` entries */
static void excl_scan(int *a, int len) {
    if (len <= 1) return;
    int carry = a[0];
    a[0] = 0;
    for (int i = 1; i < len; ++i) {
        int cur = a[i];
        a[i] = a[i - 1] + carry;
        carry = cur;
    }
}

void orc_transpose(int m, int n, int nnz, const int *ptr, const int *idx, const double *val,
                   int *tptr, int *tidx, double *tval) {
    /* tranpose.h:17-25: column histogram + exclusive scan */
    memset(tptr, 0, sizeof(int) * (size_t)(n + 1));
    for (int k = 0; k < nnz; ++k) tptr[idx[k]]++;
    excl_scan(tptr, n + 1);
    if (!tidx) return; /* tranpose.h:92-108 (_litelite) */
    /* tranpose.h:31-51: scatter rows in ascending order -> stable */
    int *fill = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    memcpy(fill, tptr, sizeof(int) * (size_t)(n + 1));
    for (int r = 0; r < m; ++r) {
        for (int k = ptr[r]; k < ptr[r + 1]; ++k) {
            int c = idx[k];
            int dst = fill[c]++;
            tidx[dst] = r;
            if (val && tval) tval[dst] = val[k];
        }
    }
    free(fill);
}

int orc_findlevel(const int *cscColPtr, const int *cscRowIdx, const int *csrRowPtr, int m,
                  int *nlevel, int *levelPtr, int *levelItem) {
    /* findlevel.h:16-22: in-degree = row length, diagonal included */
    int *deg = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
    for (int i = 0; i < m; ++i) deg[i] = csrRowPtr[i + 1] - csrRowPtr[i];
    /* findlevel.h:31-50: roots are rows whose only entry is the diagonal */
    int tail = 0;
    levelPtr[0] = 0;
    for (int i = 0; i < m; ++i)
        if (deg[i] == 1) levelItem[tail++] = i;
    levelPtr[1] = tail;
    /* findlevel.h:53-72: walk each level in discovery order; a row joins the
     * next level when its in-degree drops to exactly 1 */
    int lvl = 1;
    while (levelPtr[lvl] != m) {
        for (int p = levelPtr[lvl - 1]; p < levelPtr[lvl]; ++p) {
            int node = levelItem[p];
            for (int k = cscColPtr[node]; k < cscColPtr[node + 1]; ++k) {
                int r = cscRowIdx[k];
                if (--deg[r] == 1) levelItem[tail++] = r;
            }
        }
        ++lvl;
        levelPtr[lvl] = tail;
        if (levelPtr[lvl] == levelPtr[lvl - 1]) { /* the reference spins here forever */
            free(deg);
            return -1;
        }
    }
    *nlevel = lvl;
    free(deg);
    return 0;
}

int orc_reorder_colrow(const int *colptr, const int *rowidx, const double *val, int m, int nnz,
                       int substitution, int *colptr_new, int *rowidx_new, double *val_new,
                       int *levelItem) {
    /* utils_reordering.h:114-128: row counts, then level sets */
    int *rowptr = (int *)malloc(sizeof(int) * (size_t)(m + 1));
    int *levelPtr = (int *)malloc(sizeof(int) * (size_t)(m + 1));
    orc_transpose(m, m, nnz, colptr, rowidx, NULL, rowptr, NULL, NULL);
    int nlv = 0;
    if (orc_findlevel(colptr, rowidx, rowptr, m, &nlv, levelPtr, levelItem) != 0) {
        free(rowptr);
        free(levelPtr);
        return -1;
    }
    /* utils_reordering.h:130-159: new label of every row.  Forward: the
     * inverse of levelItem (the key/value quicksort on unique keys).
     * Backward: levelItem[i] gets label m-1-i. */
    int *perm = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
    for (int i = 0; i < m; ++i)
        perm[levelItem[i]] = substitution == ORC_FORWARD ? i : m - 1 - i;
    /* utils_reordering.h:166-181: columns in level order (reversed for
     * backward), entries of a column keep their order */
    colptr_new[0] = 0;
    for (int i = 0; i < m; ++i) {
        int src = substitution == ORC_FORWARD ? levelItem[i] : levelItem[m - 1 - i];
        int len = colptr[src + 1] - colptr[src];
        colptr_new[i + 1] = colptr_new[i] + len;
        for (int j = 0; j < len; ++j) {
            rowidx_new[colptr_new[i] + j] = rowidx[colptr[src] + j];
            val_new[colptr_new[i] + j] = val ? val[colptr[src] + j] : 0.0;
        }
    }
    /* utils_reordering.h:184-187: relabel rows */
    for (int k = 0; k < nnz; ++k) rowidx_new[k] = perm[rowidx_new[k]];
    /* utils_reordering.h:189-197: backward keeps levelItem in new-label order */
    if (substitution == ORC_BACKWARD) {
        for (int i = 0; i < m / 2; ++i) {
            int t = levelItem[i];
            levelItem[i] = levelItem[m - 1 - i];
            levelItem[m - 1 - i] = t;
        }
    }
    free(perm);
    free(rowptr);
    free(levelPtr);
    return 0;
}

/* lowest set bit: the reference reaches it with the figure[] loop
 * (recblocking_preprocess.h:109-134 / 223-248) */
static int lowbit(int t) { return t & (-t); }

/* recblocking_preprocess.h:45-55: judge[j] = sum_{i=lv-1-j}^{lv-1} 2^i; a
 * square whose preceding triangle count equals one of them reaches the
 * matrix edge */
static int reaches_edge(int t, int lv) {
    for (int j = 0; j < lv; ++j) {
        int s = 0;
        for (int i = lv - 1 - j; i <= lv - 1; ++i) s += 1 << i;
        if (s == t) return 1;
    }
    return 0;
}

void orc_geometry(const int *colptr, const int *rowidx, int m, int lv, int substitution,
                  int *loc_off, int *tmp_off, int *blk_m, int *blk_n, int *blk_nnz,
                  int *subtri_up, int *subtri_down, int *subrec_up, int *subrec_down,
                  int *subrec_right, int *subrec_left) {
    int tri = 1 << lv, sum = 2 * tri - 1;
    int step = m / tri; /* recblocking_preprocess.h:37 */
    for (int i = 0; i < sum; ++i) {
        loc_off[i] = tmp_off[i] = 0; /* zeroed by the solver entry (recblocking_solver.h:42-45) */
        subtri_up[i] = subtri_down[i] = subrec_up[i] = subrec_down[i] = -1;
        subrec_right[i] = subrec_left[i] = -1;
    }
    int t = 0;
    if (substitution == ORC_FORWARD) { /* recblocking_preprocess.h:57-178 */
        int tu = 0, td = step;
        for (int i = 0; i < sum; ++i) {
            if ((i & 1) == 0) {
                blk_m[i] = blk_n[i] = td - tu;
                subtri_up[i] = tu;
                subtri_down[i] = td;
                int c = 0;
                for (int j = tu; j < td; ++j)
                    for (int k = colptr[j]; k < colptr[j + 1]; ++k)
                        if (rowidx[k] < td) ++c;
                blk_nnz[i] = c;
                loc_off[i] = tu;
                tu += step;
                td += step;
                ++t;
            } else {
                int up = td - step;
                int down = up + lowbit(t) * step;
                int right = up;
                int left = right - (down - up);
                if (reaches_edge(t, lv)) down = m;
                blk_m[i] = down - up;
                blk_n[i] = right - left;
                int c = 0;
                for (int j = left; j < right; ++j)
                    for (int k = colptr[j]; k < colptr[j + 1]; ++k)
                        if (rowidx[k] >= up && rowidx[k] < down) ++c;
                blk_nnz[i] = c;
                tmp_off[i] = up;
                loc_off[i] = left;
                if (i == sum - 2) td = m;
                subrec_up[i] = up;
                subrec_down[i] = down;
                subrec_right[i] = right;
                subrec_left[i] = left;
            }
        }
    } else { /* recblocking_preprocess.h:179-292 */
        int tu = m - step, td = m;
        for (int i = 0; i < sum; ++i) {
            if ((i & 1) == 0) {
                blk_m[i] = blk_n[i] = td - tu;
                subtri_up[i] = tu;
                subtri_down[i] = td;
                int c = 0;
                for (int j = tu; j < td; ++j)
                    for (int k = colptr[j]; k < colptr[j + 1]; ++k)
                        if (rowidx[k] >= tu) ++c;
                blk_nnz[i] = c;
                loc_off[i] = tu;
                tu -= step;
                td -= step;
                ++t;
            } else {
                int down = tu + step;
                int up = down - lowbit(t) * step;
                int left = down;
                int right = left + (down - up);
                if (reaches_edge(t, lv)) up = 0;
                blk_m[i] = down - up;
                blk_n[i] = right - left;
                int c = 0;
                for (int j = left; j < right; ++j)
                    for (int k = colptr[j]; k < colptr[j + 1]; ++k)
                        if (rowidx[k] >= up && rowidx[k] < down) ++c;
                blk_nnz[i] = c;
                tmp_off[i] = up;
                loc_off[i] = left;
                if (i == sum - 2) tu = 0;
                subrec_up[i] = up;
                subrec_down[i] = down;
                subrec_right[i] = right;
                subrec_left[i] = left;
            }
        }
    }
}

#define ALLOC_I(n) ((int *)calloc((size_t)((n) > 0 ? (n) : 1), sizeof(int)))
#define ALLOC_D(n) ((double *)calloc((size_t)((n) > 0 ? (n) : 1), sizeof(double)))

int orc_analyse(const int *colptr, const int *rowidx, const double *val, int m, int nnz,
                int substitution, int lv, orc_blocks *o) {
    memset(o, 0, sizeof(*o));
    int tri = 1 << lv, sum = 2 * tri - 1;
    o->lv = lv;
    o->sum_block = sum;
    o->m = m;
    o->nnz = nnz;
    int *cp = ALLOC_I(m + 1), *ri = ALLOC_I(nnz);
    double *va = ALLOC_D(nnz);
    o->levelItem = ALLOC_I(m);
    /* recblocking_preprocess.h:335-337 */
    if (orc_reorder_colrow(colptr, rowidx, val, m, nnz, substitution, cp, ri, va, o->levelItem) != 0) {
        free(cp); free(ri); free(va);
        return -1;
    }
#define A(f) o->f = ALLOC_I(sum)
    A(method); A(nlv); A(m_new); A(longrow); A(lenmax);
    A(loc_off); A(tmp_off); A(blk_m); A(blk_n); A(blk_nnz);
    A(subtri_up); A(subtri_down); A(subrec_up); A(subrec_down); A(subrec_right); A(subrec_left);
#undef A
    /* recblocking_preprocess.h:346-348 */
    orc_geometry(cp, ri, m, lv, substitution, o->loc_off, o->tmp_off, o->blk_m, o->blk_n, o->blk_nnz,
                 o->subtri_up, o->subtri_down, o->subrec_up, o->subrec_down, o->subrec_right,
                 o->subrec_left);
    /* recblocking_preprocess.h:370-384 and recblocking_solver.h:65-67 */
    o->ptr_size = 1;
    o->idx_size = 0;
    o->dcsr_size = 0;
    for (int i = 0; i < sum; ++i) {
        if ((i & 1) == 0) {
            o->ptr_size += o->blk_n[i] + 1;
            o->idx_size += o->blk_nnz[i];
        } else {
            o->ptr_size += o->blk_m[i];
            o->idx_size += o->blk_nnz[i];
            o->dcsr_size += o->blk_m[i];
        }
    }
    o->recblock_Ptr = ALLOC_I(o->ptr_size);
    o->recblock_Index = ALLOC_I(o->idx_size);
    o->recblock_Val = ALLOC_D(o->idx_size);
    o->recblock_dcsr_rowidx = ALLOC_I(o->dcsr_size);
    o->ptr_offset = ALLOC_I(sum + 1);
    o->index_offset = ALLOC_I(sum + 1);
    o->dcsrindex_offset = ALLOC_I(sum + 1);
    o->loc_item_off = ALLOC_I(sum);
    o->loc_ptr_off = ALLOC_I(sum);
    o->lvl_item = ALLOC_I(m);
    o->lvl_ptr = ALLOC_I(m + tri);
    o->m_lv = ALLOC_I(m + tri);
    o->offset_lv = ALLOC_I(m + tri);
    o->nnz_lv = ALLOC_I(m + tri);
    o->recblock_Ptr[0] = 0;     /* recblocking_solver.h:85 */
    o->ptr_offset[0] = 1;       /* recblocking_solver.h:92-94 */
    o->index_offset[0] = 0;
    o->dcsrindex_offset[0] = 0;

    int *P = o->recblock_Ptr;
    int nz = 0;          /* recblock_nnz_ptr */
    int item_off = 0, lptr_off = 0;
    for (int b = 0; b < sum; ++b) {
        int bm = o->blk_m[b], bn = o->blk_n[b], bnnz = o->blk_nnz[b];
        if ((b & 1) == 0) {
            /* recblocking_preprocess.h:432-451: extract the triangle as CSC */
            int up = o->subtri_up[b], down = o->subtri_down[b];
            int *scp = ALLOC_I(bn + 1), *sri = ALLOC_I(bnnz);
            double *sva = ALLOC_D(bnnz);
            int q = 0;
            for (int c = up; c < down; ++c) {
                for (int k = cp[c]; k < cp[c + 1]; ++k) {
                    int r = ri[k];
                    int keep = substitution == ORC_FORWARD ? r < down : r >= up;
                    if (keep) {
                        sri[q] = r - up;
                        sva[q] = va[k];
                        ++q;
                    }
                }
                scp[c - up + 1] = q;
            }
            /* :457-463 CSR copy of the triangle */
            int *rrp = ALLOC_I(bm + 1), *rci = ALLOC_I(bnnz);
            double *rva = ALLOC_D(bnnz);
            orc_transpose(bn, bm, bnnz, scp, sri, sva, rrp, rci, rva);
            /* :469-484 local level sets unless diagonal-only */
            int fast = bm == bnnz;
            int nlv = 1;
            int *lp = o->lvl_ptr + lptr_off, *li = o->lvl_item + item_off;
            if (fast) {
                lp[0] = 0;
                lp[1] = bm;
                for (int i = 0; i < bm; ++i) li[i] = i;
            } else if (orc_findlevel(scp, sri, rrp, bm, &nlv, lp, li) != 0) {
                free(scp); free(sri); free(sva); free(rrp); free(rci); free(rva);
                free(cp); free(ri); free(va);
                return -1;
            }
            o->nlv[b] = nlv;
            o->loc_item_off[b] = item_off;
            o->loc_ptr_off[b] = lptr_off;
            int method;
            if (fast) {
                method = 0; /* :487-513 */
            } else {
                int nnzr = bnnz / bm; /* :516 */
                if (nlv > 20000) method = 1;                                            /* :518 */
                else if ((nnzr <= 15 && nlv <= 20) || (nnzr == 1 && nlv <= 100)) method = 2; /* :624 */
                else method = 3;                                                       /* :664 */
            }
            o->method[b] = method;
            int po = o->ptr_offset[b];
            if (method == 0 || method == 3) { /* CSC packing :498-508, :698-708 */
                for (int i = 0; i < bn; ++i) {
                    for (int k = scp[i]; k < scp[i + 1]; ++k) {
                        o->recblock_Index[nz] = sri[k];
                        o->recblock_Val[nz] = sva[k];
                        ++nz;
                    }
                    P[po + i] = P[po + i - 1] + scp[i + 1] - scp[i];
                }
            } else if (method == 2) { /* CSR packing :652-662, level arrays :632-645 */
                for (int l = 0; l < nlv; ++l) {
                    o->m_lv[lptr_off + l] = lp[l + 1] - lp[l];
                    o->offset_lv[lptr_off + l] = lp[l];
                    int s = 0;
                    for (int p = lp[l]; p < lp[l + 1]; ++p) s += rrp[p + 1] - rrp[p];
                    o->nnz_lv[lptr_off + l] = s;
                }
                for (int i = 0; i < bm; ++i) {
                    for (int k = rrp[i]; k < rrp[i + 1]; ++k) {
                        o->recblock_Index[nz] = rci[k];
                        o->recblock_Val[nz] = rva[k];
                        ++nz;
                    }
                    P[po + i] = P[po + i - 1] + rrp[i + 1] - rrp[i];
                }
            } else { /* method 1: private zero-based CSR pointer :603-616 */
                P[po] = 0;
                int c = 0;
                for (int i = 0; i < bm; ++i) {
                    for (int k = rrp[i]; k < rrp[i + 1]; ++k) {
                        o->recblock_Index[nz] = rci[k];
                        o->recblock_Val[nz] = rva[k];
                        ++nz;
                        ++c;
                    }
                    P[po + i + 1] = c;
                }
            }
            /* :726-731 */
            o->ptr_offset[b + 1] = po + bm + (method == 1 ? 1 : 0);
            o->index_offset[b + 1] = nz;
            o->dcsrindex_offset[b + 1] = o->dcsrindex_offset[b];
            item_off += bm;
            lptr_off += nlv + 1;
            free(scp); free(sri); free(sva); free(rrp); free(rci); free(rva);
        } else {
            /* :749-776 extract the square as CSC, transpose to CSR */
            int up = o->subrec_up[b], down = o->subrec_down[b];
            int left = o->subrec_left[b], right = o->subrec_right[b];
            int *scp = ALLOC_I(bn + 1), *sri = ALLOC_I(bnnz);
            double *sva = ALLOC_D(bnnz);
            int q = 0;
            for (int c = left; c < right; ++c) {
                for (int k = cp[c]; k < cp[c + 1]; ++k) {
                    int r = ri[k];
                    if (r >= up && r < down) {
                        sri[q] = r - up;
                        sva[q] = va[k];
                        ++q;
                    }
                }
                scp[c - left + 1] = q;
            }
            int *rrp = ALLOC_I(bm + 1), *rci = ALLOC_I(bnnz);
            double *rva = ALLOC_D(bnnz);
            orc_transpose(bn, bm, bnnz, scp, sri, sva, rrp, rci, rva);
            /* :783-793 entries in CSR order */
            for (int i = 0; i < bm; ++i)
                for (int k = rrp[i]; k < rrp[i + 1]; ++k) {
                    o->recblock_Index[nz] = rci[k];
                    o->recblock_Val[nz] = rva[k];
                    ++nz;
                }
            /* :800-826 row statistics */
            int nonempty = 0, lenmax = bm > 0 ? rrp[1] - rrp[0] : 0, longrow = 0, longlen = 0;
            for (int i = 1; i <= bm; ++i) {
                int len = rrp[i] - rrp[i - 1];
                if (len > lenmax) lenmax = len;
                if (len != 0) {
                    if (len > ORC_LONGROW_THRESHOLD) {
                        ++longrow;
                        longlen += len;
                    }
                    ++nonempty;
                }
            }
            o->m_new[b] = nonempty;
            o->longrow[b] = longrow;
            o->lenmax[b] = lenmax;
            int po = o->ptr_offset[b];
            int real_i = 0, dcsr_i = 0, method = -1;
            if (bnnz != 0) { /* an empty square divides by zero at :825 in the reference */
                int nnzr = (bnnz - longlen) / nonempty;
                double empty_ratio = 100 * (double)(bm - nonempty) / (double)bm;
                if (nnzr <= 12 && empty_ratio <= 50) method = 0;       /* :835 */
                else if (nnzr <= 12 && empty_ratio > 50) method = 1;   /* :856 */
                else if (nnzr > 12 && empty_ratio <= 15) method = 2;   /* :880 */
                else method = 3;                                       /* :898 */
                if (method == 0 || method == 2) {
                    for (int i = 0; i < bm; ++i) P[po + i] = P[po + i - 1] + rrp[i + 1] - rrp[i];
                    real_i = bm;
                } else {
                    int dbase = o->dcsrindex_offset[b];
                    for (int i = 0; i < bm; ++i) {
                        if (rrp[i + 1] != rrp[i]) {
                            P[po + dcsr_i] = P[po + dcsr_i - 1] + rrp[i + 1] - rrp[i];
                            o->recblock_dcsr_rowidx[dbase + dcsr_i] = i;
                            ++dcsr_i;
                        }
                    }
                    real_i = dcsr_i;
                }
            }
            o->method[b] = method;
            o->nlv[b] = 0;
            /* :952-954 */
            o->ptr_offset[b + 1] = po + real_i;
            o->index_offset[b + 1] = nz;
            o->dcsrindex_offset[b + 1] = o->dcsrindex_offset[b] + dcsr_i;
            free(scp); free(sri); free(sva); free(rrp); free(rci); free(rva);
        }
    }
    free(cp); free(ri); free(va);
    return 0;
}

void orc_blocks_free(orc_blocks *o) {
    void *ps[] = {o->method, o->nlv, o->m_new, o->longrow, o->lenmax, o->loc_off, o->tmp_off,
                  o->blk_m, o->blk_n, o->blk_nnz, o->subtri_up, o->subtri_down, o->subrec_up,
                  o->subrec_down, o->subrec_right, o->subrec_left, o->ptr_offset, o->index_offset,
                  o->dcsrindex_offset, o->recblock_Ptr, o->recblock_Index, o->recblock_Val,
                  o->recblock_dcsr_rowidx, o->levelItem, o->loc_item_off, o->loc_ptr_off,
                  o->lvl_item, o->lvl_ptr, o->m_lv, o->offset_lv, o->nnz_lv};
    for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); ++i) free(ps[i]);
    memset(o, 0, sizeof(*o));
}

int orc_auto_lv(int m, int device_id) {
    /* main.cu:245-254 */
    int li;
    for (li = 1; li <= 100; ++li)
        if (m / pow(2, li + 1) < (device_id == 0 ? 92160 : 58880)) break;
    return li;
}

static int find_diag(const int *rowptr, const int *colidx, int i) {
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
        if (colidx[k] == i) return k;
    return -1;
}

int orc_sptrsv_csr(int n, const int *rowptr, const int *colidx, const double *val,
                   int substitution, const double *b, double *x) {
    for (int s = 0; s < n; ++s) {
        int i = substitution == ORC_FORWARD ? s : n - 1 - s;
        int d = find_diag(rowptr, colidx, i);
        if (d < 0 || val[d] == 0.0) return -1;
        double acc = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (k != d) acc += val[k] * x[colidx[k]];
        x[i] = (b[i] - acc) / val[d];
    }
    return 0;
}

int orc_sptrsv_csr_compensated(int n, const int *rowptr, const int *colidx, const double *val,
                               int substitution, const double *b, double *x) {
    /* Neumaier's improved Kahan summation of b_i - sum_j a_ij x_j */
    for (int s = 0; s < n; ++s) {
        int i = substitution == ORC_FORWARD ? s : n - 1 - s;
        int d = find_diag(rowptr, colidx, i);
        if (d < 0 || val[d] == 0.0) return -1;
        double sum = b[i], comp = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            if (k == d) continue;
            double term = -(val[k] * x[colidx[k]]);
            double t = sum + term;
            if (fabs(sum) >= fabs(term)) comp += (sum - t) + term;
            else comp += (term - t) + sum;
            sum = t;
        }
        x[i] = (sum + comp) / val[d];
    }
    return 0;
}

/* Level-scheduled substitution (the CPU baseline of the benchmark; not used
 * as a checker).  prepare: level of row i = 1 + the highest level among its
 * dependencies (columns j < i forward, j > i backward), rows bucketed by
 * level in row order, and a copy of the matrix in that order (the order the
 * reference's level-set reordering gives, utils_reordering.h:102-210):
 * row q of the copy is row item[q], its off-diagonal entries in stored order
 * with columns renumbered to positions, its diagonal apart; plus a copy in
 * the rows' own order with the diagonal apart.  solve, nthreads >= 1: each
 * level's rows split over the threads (rows of one level are independent;
 * a spin barrier between levels, runs of small levels solved by one
 * thread), each row reading its b entry and writing its x entry in the
 * caller's order as it is solved; nthreads == 0: serial substitution over
 * the second copy.  Every row sums its entries in stored order and divides
 * by the diagonal last, as orc_sptrsv_csr does, so results are identical to
 * it bit for bit. */
int orc_levels_prepare(int n, const int *rowptr, const int *colidx, const double *val, int substitution,
                       orc_levels *L) {
    memset(L, 0, sizeof(*L));
    int *lev = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int nl = 0;
    for (int s = 0; s < n; ++s) {
        int i = substitution == ORC_FORWARD ? s : n - 1 - s;
        int d = find_diag(rowptr, colidx, i), m = -1;
        if (d < 0 || val[d] == 0.0) {
            free(lev);
            return -1;
        }
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int j = colidx[k];
            if (k == d) continue;
            if (j < 0 || j >= n || ((substitution == ORC_FORWARD) ? j >= i : j <= i)) {
                free(lev);
                return -1; /* outside the triangle */
            }
            if (lev[j] > m) m = lev[j];
        }
        lev[i] = m + 1;
        if (m + 2 > nl) nl = m + 2;
    }
    L->n = n;
    L->nlevel = nl;
    L->substitution = substitution;
    L->lp = (int *)calloc((size_t)nl + 1, sizeof(int));
    L->item = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *pos = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) L->lp[lev[i] + 1]++;
    for (int l = 0; l < nl; ++l) L->lp[l + 1] += L->lp[l];
    int *fill = (int *)malloc(sizeof(int) * (size_t)(nl > 0 ? nl : 1));
    memcpy(fill, L->lp, sizeof(int) * (size_t)nl);
    for (int i = 0; i < n; ++i) L->item[fill[lev[i]]++] = i;
    for (int q = 0; q < n; ++q) pos[L->item[q]] = q;
    const int off = rowptr[n] - n;
    L->prp = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    L->pci = (int *)malloc(sizeof(int) * (size_t)(off > 0 ? off : 1));
    L->pva = (double *)malloc(sizeof(double) * (size_t)(off > 0 ? off : 1));
    L->pdiag = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    L->px = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    int o = 0;
    L->prp[0] = 0;
    for (int q = 0; q < n; ++q) {
        int i = L->item[q], d = find_diag(rowptr, colidx, i);
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            if (k == d) continue;
            L->pci[o] = pos[colidx[k]];
            L->pva[o++] = val[k];
        }
        L->prp[q + 1] = o;
        L->pdiag[q] = val[d];
    }
    L->nrp = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    L->nci = (int *)malloc(sizeof(int) * (size_t)(off > 0 ? off : 1));
    L->nva = (double *)malloc(sizeof(double) * (size_t)(off > 0 ? off : 1));
    L->ndiag = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    o = 0;
    L->nrp[0] = 0;
    for (int i = 0; i < n; ++i) {
        int d = find_diag(rowptr, colidx, i);
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            if (k == d) continue;
            L->nci[o] = colidx[k];
            L->nva[o++] = val[k];
        }
        L->nrp[i + 1] = o;
        L->ndiag[i] = val[d];
    }
    free(fill);
    free(pos);
    free(lev);
    return 0;
}

/* levels of fewer rows than this are solved by one thread of the team, a
 * run of them between two barriers (a barrier costs more than the rows) */
#define LV_SMALL 192

/* sense-reversing spin barrier of the solve's thread team */
typedef struct {
    atomic_int count, sense;
    int n;
} lv_barrier;

static void lv_wait(lv_barrier *br, int *local) {
    *local = !*local;
    if (atomic_fetch_add(&br->count, 1) == br->n - 1) {
        atomic_store(&br->count, 0);
        atomic_store(&br->sense, *local);
    } else {
        int spins = 0;
        while (atomic_load(&br->sense) != *local)
            if (++spins > 4096) {
                sched_yield();
                spins = 0;
            }
    }
}

typedef struct {
    const orc_levels *L;
    const double *b;
    double *x;
    lv_barrier *br;
    atomic_int *go; /* set once the team's size is final */
    int t, nt;
} lv_task;

static void *lv_run(void *arg) {
    const lv_task *w = (const lv_task *)arg;
    while (!atomic_load(w->go)) sched_yield();
    const orc_levels *L = w->L;
    const int n = L->n, t = w->t, nt = w->nt;
    const int *lp = L->lp, *item = L->item, *prp = L->prp, *pci = L->pci;
    const double *pva = L->pva, *pdiag = L->pdiag;
    double *px = L->px;
    int local = 0;
    (void)n;
    for (int l = 0; l < L->nlevel;) {
        int lo = lp[l], hi = lp[l + 1], next = l + 1;
        if (nt > 1 && hi - lo < LV_SMALL) {
            /* a run of small levels: thread 0 solves them in order, one barrier */
            while (next < L->nlevel && lp[next + 1] - lp[next] < LV_SMALL) ++next;
            hi = lp[next];
            if (t != 0) hi = lo;
        } else {
            const int cnt = hi - lo;
            hi = lo + (int)((long long)cnt * (t + 1) / nt);
            lo = lo + (int)((long long)cnt * t / nt);
        }
        for (int q = lo; q < hi; ++q) {
            double acc = 0.0;
            for (int k = prp[q]; k < prp[q + 1]; ++k) acc += pva[k] * px[pci[k]];
            const double v = (w->b[item[q]] - acc) / pdiag[q];
            px[q] = v;
            w->x[item[q]] = v;
        }
        if (nt > 1) lv_wait(w->br, &local);
        l = next;
    }
    return NULL;
}

void orc_levels_solve(const orc_levels *L, const double *b, double *x, int nthreads) {
    if (nthreads <= 0) { /* serial, the rows' own order */
        const int n = L->n;
        for (int s = 0; s < n; ++s) {
            const int i = L->substitution == ORC_FORWARD ? s : n - 1 - s;
            double acc = 0.0;
            for (int k = L->nrp[i]; k < L->nrp[i + 1]; ++k) acc += L->nva[k] * x[L->nci[k]];
            x[i] = (b[i] - acc) / L->ndiag[i];
        }
        return;
    }
    if (nthreads > 256) nthreads = 256;
    lv_barrier br;
    atomic_int go;
    atomic_init(&br.count, 0);
    atomic_init(&br.sense, 0);
    atomic_init(&go, 0);
    lv_task w[256];
    pthread_t th[256];
    int started = 1;
    for (int t = 0; t < nthreads; ++t) w[t] = (lv_task){L, b, x, &br, &go, t, nthreads};
    for (int t = 1; t < nthreads; ++t) {
        if (pthread_create(&th[t], NULL, lv_run, &w[t]) != 0) break;
        ++started;
    }
    /* the team is the threads that started (the caller included) */
    br.n = started;
    for (int t = 0; t < started; ++t) w[t].nt = started;
    atomic_store(&go, 1);
    lv_run(&w[0]);
    for (int t = 1; t < started; ++t) pthread_join(th[t], NULL);
}

void orc_levels_free(orc_levels *L) {
    free(L->lp);
    free(L->item);
    free(L->prp);
    free(L->pci);
    free(L->pva);
    free(L->pdiag);
    free(L->px);
    free(L->nrp);
    free(L->nci);
    free(L->nva);
    free(L->ndiag);
    memset(L, 0, sizeof(*L));
}

int orc_sptrsv_csr_multi(int n, const int *rowptr, const int *colidx, const double *val,
                         int substitution, int k, const double *b, int ldb, double *x, int ldx) {
    for (int c = 0; c < k; ++c)
        if (orc_sptrsv_csr(n, rowptr, colidx, val, substitution, b + (size_t)c * ldb,
                           x + (size_t)c * ldx) != 0)
            return -1;
    return 0;
}

void orc_spmv_csr(int n, const int *rowptr, const int *colidx, const double *val,
                  const double *x, double *y) {
    for (int i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) acc += val[k] * x[colidx[k]];
        y[i] = acc;
    }
}

int orc_ilu0_csr(int n, const int *rowptr, const int *colidx, const double *val, double *lu) {
    int *diag = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int k = 0; k < rowptr[n]; ++k) lu[k] = val[k];
    for (int i = 0; i < n; ++i) {
        diag[i] = -1;
        for (int p = rowptr[i]; p < rowptr[i + 1]; ++p)
            if (colidx[p] == i) diag[i] = p;
        if (diag[i] < 0) {
            free(diag);
            return -1;
        }
    }
    for (int i = 0; i < n; ++i) {
        for (int p = rowptr[i]; p < diag[i]; ++p) {
            const int k = colidx[p];
            const double piv = lu[diag[k]];
            if (piv == 0.0) {
                free(diag);
                return -2;
            }
            const double a = lu[p] / piv;
            lu[p] = a;
            /* a_ij -= a_ik * a_kj for j > k present in both rows (both sorted) */
            int t = diag[k] + 1;
            for (int q = p + 1; q < rowptr[i + 1]; ++q) {
                const int j = colidx[q];
                while (t < rowptr[k + 1] && colidx[t] < j) ++t;
                if (t < rowptr[k + 1] && colidx[t] == j) {
                    volatile double prod = a * lu[t];
                    lu[q] = lu[q] - prod;
                }
            }
        }
        if (lu[diag[i]] == 0.0) {
            free(diag);
            return -2;
        }
    }
    free(diag);
    return 0;
}

int orc_ic0_csr(int n, const int *rowptr, const int *colidx, const double *val, double *l) {
    /* lower triangle, columns ascending, diagonal last in every row */
    for (int i = 0; i < n; ++i) {
        const int b = rowptr[i], e = rowptr[i + 1];
        if (e <= b || colidx[e - 1] != i) return -1;
        for (int p = b; p + 1 < e; ++p)
            if (colidx[p] >= colidx[p + 1] || colidx[p] < 0) return -1;
    }
    for (int k = 0; k < rowptr[n]; ++k) l[k] = val[k];
    int bad = 0;
    for (int i = 0; i < n; ++i) {
        const int b = rowptr[i], d = rowptr[i + 1] - 1;
        for (int p = b; p < d; ++p) {
            /* l_ik = (a_ik - sum_{j<k} l_ij l_kj) / l_kk, j ascending over both rows */
            const int k = colidx[p], kd = rowptr[k + 1] - 1;
            double s = l[p];
            int qi = b, qk = rowptr[k];
            while (qi < p && qk < kd) {
                if (colidx[qi] == colidx[qk]) {
                    volatile double prod = l[qi] * l[qk];
                    s = s - prod;
                    ++qi;
                    ++qk;
                } else if (colidx[qi] < colidx[qk]) {
                    ++qi;
                } else {
                    ++qk;
                }
            }
            l[p] = s / l[kd];
        }
        /* l_ii = sqrt(a_ii - sum_j l_ij^2), j ascending */
        double s = l[d];
        for (int p = b; p < d; ++p) {
            volatile double prod = l[p] * l[p];
            s = s - prod;
        }
        if (!(s > 0.0) && !bad) bad = 1;
        l[d] = s > 0.0 ? sqrt(s) : s;
    }
    return bad ? -2 : 0;
}

/* ---- Matrix Market input (mmio_highlevel.h:137-296) -------------------- */

void orc_free(void *p) { free(p); }

int orc_mtx_read(const char *path, int *m, int *n, int *nnz, int *field, int *symmetric, int **rowptr,
                 int **colidx, double **val) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char line[1025], w[5][64];
    /* mm_read_banner (mmio.h:254-331): five tokens, banner prefix, lower-cased words */
    if (!fgets(line, sizeof line, f) ||
        sscanf(line, "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) != 5 ||
        strncmp(w[0], "%%MatrixMarket", 14) != 0) {
        fclose(f);
        return -2;
    }
    for (int k = 1; k < 5; ++k)
        for (char *q = w[k]; *q; ++q) *q = (char)tolower((unsigned char)*q);
    if (strcmp(w[1], "matrix") || strcmp(w[2], "coordinate")) {
        fclose(f);
        return strcmp(w[1], "matrix") ? -2 : -3;
    }
    int fld = !strcmp(w[3], "real") ? 0 : !strcmp(w[3], "integer") ? 1 : !strcmp(w[3], "pattern") ? 2
            : !strcmp(w[3], "complex") ? 3 : -1;
    if (fld < 0) {
        fclose(f);
        return -3;
    }
    int sym = !strcmp(w[4], "symmetric") || !strcmp(w[4], "hermitian");
    /* mm_read_mtx_crd_size (mmio.h:339-367): skip '%' lines, then M N nz */
    int M = 0, N = 0, NZ = 0;
    do {
        if (!fgets(line, sizeof line, f)) {
            fclose(f);
            return -4;
        }
    } while (line[0] == '%');
    if (sscanf(line, "%d %d %d", &M, &N, &NZ) != 3) {
        int got;
        do {
            got = fscanf(f, "%d %d %d", &M, &N, &NZ);
            if (got == EOF) {
                fclose(f);
                return -4;
            }
        } while (got != 3);
    }
    /* entries in file order (mmio_highlevel.h:182-216), 0-based */
    int *I = (int *)malloc(sizeof(int) * (size_t)(NZ > 0 ? NZ : 1));
    int *J = (int *)malloc(sizeof(int) * (size_t)(NZ > 0 ? NZ : 1));
    double *V = (double *)malloc(sizeof(double) * (size_t)(NZ > 0 ? NZ : 1));
    int rc = 0;
    for (int k = 0; k < NZ && !rc; ++k) {
        int i = 0, j = 0, iv = 0;
        double re = 1.0, im = 0.0;
        int want = fld == 2 ? 2 : fld == 3 ? 4 : 3, got;
        if (fld == 0) got = fscanf(f, "%d %d %lg", &i, &j, &re);
        else if (fld == 1) {
            got = fscanf(f, "%d %d %d", &i, &j, &iv);
            re = iv;
        } else if (fld == 2) got = fscanf(f, "%d %d", &i, &j);
        else got = fscanf(f, "%d %d %lg %lg", &i, &j, &re, &im);
        if (got != want) rc = -5;
        else if (i < 1 || i > M || j < 1 || j > N) rc = -6;
        I[k] = i - 1;
        J[k] = j - 1;
        V[k] = re;
    }
    fclose(f);
    if (rc) {
        free(I);
        free(J);
        free(V);
        return rc;
    }
    /* mmio_highlevel.h:218-290: row counts (mirrors included), scan, and
     * placement in file order, the mirrored entry right after its entry */
    int *ptr = (int *)calloc((size_t)M + 1, sizeof(int));
    for (int k = 0; k < NZ; ++k) {
        ptr[I[k] + 1]++;
        if (sym && I[k] != J[k]) ptr[J[k] + 1]++;
    }
    for (int r = 0; r < M; ++r) ptr[r + 1] += ptr[r];
    int total = ptr[M];
    int *ci = (int *)malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));
    double *cv = (double *)malloc(sizeof(double) * (size_t)(total > 0 ? total : 1));
    int *fill = (int *)malloc(sizeof(int) * (size_t)(M > 0 ? M : 1));
    for (int r = 0; r < M; ++r) fill[r] = ptr[r];
    for (int k = 0; k < NZ; ++k) {
        int d = fill[I[k]]++;
        ci[d] = J[k];
        cv[d] = V[k];
        if (sym && I[k] != J[k]) {
            d = fill[J[k]]++;
            ci[d] = I[k];
            cv[d] = V[k];
        }
    }
    free(fill);
    free(I);
    free(J);
    free(V);
    *m = M;
    *n = N;
    *nnz = total;
    *field = fld;
    *symmetric = sym;
    *rowptr = ptr;
    *colidx = ci;
    *val = cv;
    return 0;
}

int orc_tri_extract(int m, const int *rowptr, const int *colidx, const double *val, int substitution,
                    const double *strict_val, int *trowptr, int *tcolidx, double *tval) {
    /* main.cu:157-198 */
    int p = 0, r = 0;
    trowptr[0] = 0;
    for (int i = 0; i < m; ++i) {
        if (substitution == ORC_BACKWARD) {
            tcolidx[p] = i;
            tval[p++] = 1.0;
        }
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            const int c = colidx[k];
            if (substitution == ORC_FORWARD ? c < i : c > i) {
                tcolidx[p] = c;
                tval[p++] = strict_val ? strict_val[r] : val[k];
                ++r;
            }
        }
        if (substitution == ORC_FORWARD) {
            tcolidx[p] = i;
            tval[p++] = 1.0;
        }
        trowptr[i + 1] = p;
    }
    return p;
}
