/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of recblock-sptrsv's CPU analysis and a serial FP64
 * substitution, used as the checker for the B200 library.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
 * product never links or calls it.
 *
 * Parity pin: the integer outputs of this restatement are checked against
 * golden vectors produced by the reference's own analysis code
 * (recblocking_preprocess.h get_recblock_size + L_/U_preprocessing), compiled
 * from the reference sources by oracle/Makefile into oracle/_ref/.
 *
 * The value oracle (orc_sptrsv_csr) is a restatement of textbook serial
 * substitution: the reference has no CPU triangular solve; its only value
 * check is main.cu:296-317 against x_ref.
 */
#ifndef RBS_ORACLE_H
#define RBS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_FORWARD 0  /* common.h:25 SUBSTITUTION_FORWARD */
#define ORC_BACKWARD 1 /* common.h:26 SUBSTITUTION_BACKWARD */
#define ORC_LONGROW_THRESHOLD 2048 /* utils_spmv_cuda.h:9 */

/* tranpose.h:7-54 -- CSR(m x n) -> CSC, stable by rows.  val/tval may be NULL. */
void orc_transpose(int m, int n, int nnz, const int *ptr, const int *idx, const double *val,
                   int *tptr, int *tidx, double *tval);

/* findlevel.h:7-83 -- Kahn BFS level sets in discovery order.
 * Returns 0, or -1 when a level makes no progress (the reference loops forever there). */
int orc_findlevel(const int *cscColPtr, const int *cscRowIdx, const int *csrRowPtr, int m,
                  int *nlevel, int *levelPtr, int *levelItem);

/* utils_reordering.h:102-210 -- symmetric level-set permutation of a CSC. */
int orc_reorder_colrow(const int *colptr, const int *rowidx, const double *val, int m, int nnz,
                       int substitution, int *colptr_new, int *rowidx_new, double *val_new,
                       int *levelItem);

/* recblocking_preprocess.h:15-296 -- recursive-block geometry.  All arrays
 * have 2^(lv+1)-1 entries; entries that the reference leaves unset are
 * written as -1 here. */
void orc_geometry(const int *colptr, const int *rowidx, int m, int lv, int substitution,
                  int *loc_off, int *tmp_off, int *blk_m, int *blk_n, int *blk_nnz,
                  int *subtri_up, int *subtri_down, int *subrec_up, int *subrec_down,
                  int *subrec_right, int *subrec_left);

/* Outputs of L_preprocessing / U_preprocessing (recblocking_preprocess.h:387-967, 969-1474). */
typedef struct orc_blocks {
    int lv, sum_block, m, nnz;
    int ptr_size, idx_size, dcsr_size;   /* get_recblock_size :370-384 */
    int *method;        /* [sum_block] tri: 0..3, square: 0..3, -1 empty square */
    int *nlv;           /* [sum_block] local levels of tri blocks (1 for fasttrack), 0 for squares */
    int *m_new;         /* [sum_block] nonempty rows of square blocks */
    int *longrow;       /* [sum_block] rows longer than 2048 in square blocks */
    int *lenmax;        /* [sum_block] longest row of square blocks */
    int *loc_off, *tmp_off, *blk_m, *blk_n, *blk_nnz;
    int *subtri_up, *subtri_down, *subrec_up, *subrec_down, *subrec_right, *subrec_left;
    int *ptr_offset, *index_offset, *dcsrindex_offset;  /* [sum_block+1] */
    int *recblock_Ptr;     /* [ptr_size] (unwritten tail entries are 0) */
    int *recblock_Index;   /* [idx_size] */
    double *recblock_Val;  /* [idx_size] */
    int *recblock_dcsr_rowidx; /* [dcsr_size] (unwritten tail entries are 0) */
    int *levelItem;        /* [m] global level order (reversed for backward) */
    /* local level sets of tri blocks, concatenated: block b occupies
     * lvl_item[loc_item_off[b] .. +blk_m[b]) and lvl_ptr[loc_ptr_off[b] .. +nlv[b]+1) */
    int *loc_item_off, *loc_ptr_off, *lvl_item, *lvl_ptr;
    /* method-2 per-level arrays, concatenated like lvl_ptr (nlv entries each) */
    int *m_lv, *offset_lv, *nnz_lv;
} orc_blocks;

/* Full CPU analysis: reorder + geometry + per-block extraction, method choice
 * and packing, on a CSC triangular input.  Returns 0, or -1 on a structure the
 * reference cannot handle (level search stuck). */
int orc_analyse(const int *colptr, const int *rowidx, const double *val, int m, int nnz,
                int substitution, int lv, orc_blocks *out);
void orc_blocks_free(orc_blocks *b);

/* main.cu:245-254 -- automatic recursion depth for lv == -1. */
int orc_auto_lv(int m, int device_id);

/* Serial FP64 substitution on CSR.  lower: x_i = (b_i - sum_{j<i} L_ij x_j)/L_ii
 * for i ascending; upper: descending.  Returns -1 on a zero/missing diagonal. */
/* ILU(0) of a square CSR matrix (columns ascending, diagonal present in
 * every row), row-wise IKJ order restricted to the pattern: lu holds the
 * strict lower part of L (unit diagonal implied) and U.  Not part of the
 * reference (the factor producer its solver is meant for); every update is
 * a separate multiply and subtract, rounded to nearest (no contraction).
 * Returns -1 on a missing diagonal, -2 on a zero pivot. */
int orc_ilu0_csr(int n, const int *rowptr, const int *colidx, const double *val, double *lu);

int orc_sptrsv_csr(int n, const int *rowptr, const int *colidx, const double *val,
                   int substitution, const double *b, double *x);
/* Same with Neumaier-compensated row sums (bounds the oracle's own rounding). */
int orc_sptrsv_csr_compensated(int n, const int *rowptr, const int *colidx, const double *val,
                               int substitution, const double *b, double *x);
/* Level-scheduled substitution over a level-ordered copy of the matrix, on
 * host threads (nthreads >= 1), or serial substitution over a copy in the
 * rows' own order with the diagonal apart (nthreads == 0); results identical
 * to orc_sptrsv_csr (the benchmark's CPU baseline). */
typedef struct orc_levels {
    int n, nlevel, substitution;
    int *lp, *item, *prp, *pci;
    double *pva, *pdiag, *px;
    int *nrp, *nci; /* the rows in their own order, diagonal apart (nthreads == 0) */
    double *nva, *ndiag;
} orc_levels;
int orc_levels_prepare(int n, const int *rowptr, const int *colidx, const double *val, int substitution,
                       orc_levels *L);
void orc_levels_solve(const orc_levels *L, const double *b, double *x, int nthreads);
void orc_levels_free(orc_levels *L);
/* k right-hand sides, column-major with leading dimension ld. */
int orc_sptrsv_csr_multi(int n, const int *rowptr, const int *colidx, const double *val,
                         int substitution, int k, const double *b, int ldb, double *x, int ldx);
/* y = A x  (CSR) */
void orc_spmv_csr(int n, const int *rowptr, const int *colidx, const double *val,
                  const double *x, double *y);

/* IC(0): incomplete Cholesky with zero fill of an SPD matrix given as its
 * lower triangle (CSR, columns ascending, diagonal last in every row);
 * l receives L in that pattern with L L^T matching A on it.  Row by row,
 * l_ik = (a_ik - sum_{j<k} l_ij l_kj) / l_kk over the columns shared by rows
 * i and k in ascending order, then l_ii = sqrt(a_ii - sum_j l_ij^2); every
 * product rounded on its own.  Returns 0, -1 bad structure, -2 a pivot
 * <= 0 (not positive definite on the pattern; l_ii is left as the
 * non-positive value). */
int orc_ic0_csr(int n, const int *rowptr, const int *colidx, const double *val, double *l);

/* mmio_highlevel.h:137-296 (mmio_data, with mm_read_banner and
 * mm_read_mtx_crd_size, mmio.h:254-367): a Matrix Market coordinate file
 * into CSR.  fscanf reads the entries ("%d %d %lg" and the other fields'
 * forms); symmetric and Hermitian files add the mirrored entry (diagonal
 * once); rows ascending, file order inside a row.  The arrays are malloc'd
 * (free with orc_free).  Returns 0, or -1 cannot open, -2 bad banner,
 * -3 not coordinate / unknown field, -4 bad size line, -5 truncated or
 * malformed entry, -6 index out of range (the reference does not check
 * these two). */
int orc_mtx_read(const char *path, int *m, int *n, int *nnz, int *field, int *symmetric, int **rowptr,
                 int **colidx, double **val);
void orc_free(void *p);

/* main.cu:157-198: the unit-diagonal triangle of a square CSR: strictly
 * lower (forward; diagonal last in the row) or upper (backward; diagonal
 * first) entries in A's order; strict entry r takes strict_val[r] when
 * strict_val is not NULL, else A's value.  Output arrays sized m+1 and
 * m + (strict entries); returns the entry count. */
int orc_tri_extract(int m, const int *rowptr, const int *colidx, const double *val, int substitution,
                    const double *strict_val, int *trowptr, int *tcolidx, double *tval);

/* gen.c: the seeded systems of include/rbs_gen.h (kind: 0 band Poisson,
 * 1 2D Laplacian, 2 Zipf, 3 chain, 4 diagonal), restated so that CPU-side
 * inputs need no GPU library; arrays from malloc (free with orc_free). */
int orc_gen_lower_csr(int kind, int n, int grid, double lambda, int band, double zipf_alpha, int zipf_max,
                      int chain_bw, unsigned long long seed, int *n_out, long long *nnz_out, int **rowptr,
                      int **colidx, double **val);
int orc_gen_uniform(unsigned long long seed, long long n, double lo, double hi, double *out);

#ifdef __cplusplus
}
#endif
#endif
