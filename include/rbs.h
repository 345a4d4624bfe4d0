/*
 * rbs.h -- C ABI of the B200 recursive-block sparse triangular solver.
 *
 * Drop-in boundary for recblock-sptrsv's analysis ("preprocess") and solve
 * entry points.  Every function is extern "C", takes plain pointers and
 * sizes, and returns an int status (RBS_OK == 0) where the reference returns
 * void.  Paths in citations are relative to the reference project directory
 * recblock-sptrsv/.
 *
 *   reference                                          replacement
 *   -------------------------------------------------  -----------------------------
 *   recblocking_solver_cuda(...)  recblocking_solver_cuda.h:21-32   recblocking_solver_cuda (same
 *                                                      signature, below) or
 *                                                      rbs_analyse_device + rbs_solve
 *   recblocking_solver(...)       recblocking_solver.h:16-28        recblocking_solver (same
 *                                                      signature) or rbs_analyse + rbs_solve_host
 *   levelset_reordering_colrow_csc[_cuda] + mat_preprocessing[_cuda]
 *   + per-block loop  (recblocking_solver_cuda.h:73-584,
 *     recblocking_preprocess.h:298-967)                 rbs_analyse / rbs_analyse_device
 *   L_calculate / U_calculate (recblocking_calculate.h:15,170)      rbs_solve
 *   device_memfree (recblocking_calculate.h:327)        rbs_plan_free
 *
 * Conventions: the caller owns inputs and outputs; a plan owns its device
 * state; each plan runs on one CUDA stream (rbs_plan_set_stream); distinct
 * plans may be used from distinct host threads.  Errors never hang: every
 * device wait is bounded and reports RBS_ERR_TIMEOUT.
 */
#ifndef RBS_H
#define RBS_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define RBS_OK 0
#define RBS_ERR_ARG 1          /* null pointer, bad size or flag, plan without device state */
#define RBS_ERR_STRUCTURE 2    /* not triangular, diagonal missing/misplaced, index out of range */
#define RBS_ERR_CUDA 3         /* CUDA runtime error (message in rbs_last_error) */
#define RBS_ERR_NOMEM 4        /* host or device allocation failed */
#define RBS_ERR_TIMEOUT 5      /* a bounded device wait expired (dependency never produced) */
#define RBS_ERR_NOCONV 6       /* mixed-precision refinement missed its tolerance */
#define RBS_ERR_BUDGET 7       /* serving: request does not fit the HBM budget */
#define RBS_ERR_UNSUPPORTED 8  /* option combination not built */

/* ---- flags ------------------------------------------------------------ */
#define RBS_FORWARD 0          /* common.h:25 SUBSTITUTION_FORWARD  (lower, L x = b) */
#define RBS_BACKWARD 1         /* common.h:26 SUBSTITUTION_BACKWARD (upper, U x = b) */

#define RBS_FMT_CSC 0          /* the reference's input format (diagonal first/last per column) */
#define RBS_FMT_CSR 1

#define RBS_PREC_FP64 0        /* plain FP64 solve */
#define RBS_PREC_MIXED 1       /* FP32 sweeps + FP64 residual/update refinement to ir_tol */
#define RBS_PREC_FP32 2        /* one FP32 sweep, no refinement */

#define RBS_SELECT_REFERENCE 0 /* the reference's thresholds pick the method per block
                                  (recblocking_preprocess.h:472-709, 835-922); each reference
                                  method maps to this library's kernel of the same kind */
#define RBS_SELECT_AUTO 1      /* cost model over this library's kernels */
#define RBS_SELECT_TUNE 2      /* time the candidate kernels per block at analysis, keep the fastest */

typedef struct rbs_options {
    int select;             /* RBS_SELECT_* (default AUTO) */
    int device;             /* CUDA device ordinal, -1 = current (default -1) */
    int lv_device_id;       /* device id used by the automatic-lv rule main.cu:245-254 (default 0) */
    int host_only;          /* 1: analysis only, no device state (for host-side inspection) */
    int max_rhs;            /* widest k a solve will use (default 1; grows on demand) */
    int mixed;              /* 1: also build FP32 factor copies for RBS_PREC_MIXED/FP32 (default 1) */
    double ir_tol;          /* refinement stop: ||dx||/||x|| <= ir_tol (default 1e-13) */
    int ir_max_iter;        /* default 8 */
    long long spin_limit;   /* polls before a device wait gives up (default 1<<22 with backoff) */
} rbs_options;

typedef struct rbs_stats {
    double ms;              /* device time of the solve, CUDA events on the plan's stream */
    int iterations;         /* refinement corrections applied (0 for FP64/FP32) */
    double correction;      /* last ||dx||/||x|| (mixed) */
    double useful_bytes;    /* nnz*(8+4) + 4*(n+1) + 16*n*k */
    double moved_bytes;     /* algorithmic bytes of all passes actually run */
} rbs_stats;

typedef struct rbs_plan_info {
    int n, nnz, lv, substitution;
    int nlevel;             /* global level count */
    int sum_block;          /* 2^(lv+1)-1 */
    int kernels[8];         /* blocks per kernel kind (RBS_K_*) */
    long long device_bytes; /* device memory held by the plan */
    double analyse_ms;      /* wall time of the analysis */
} rbs_plan_info;

/* kernel kinds reported in rbs_plan_info.kernels / rbs_plan_export("kernel") */
#define RBS_K_DIAG 0        /* diagonal-only triangle (reference method 0) */
#define RBS_K_SYNCFREE 1    /* multi-CTA sync-free triangle (reference method 3) */
#define RBS_K_LEVEL 2       /* single-CTA level-synchronous triangle (reference method 2) */
#define RBS_K_SEQ 3         /* single-CTA sequential triangle (replaces cuSPARSE, method 1) */
#define RBS_K_BANDSCAN 4    /* parallel affine scan for deep narrow-band triangles (method 1) */
#define RBS_K_SPMV 5        /* square block SpMV, fused b -= S x (methods 0..3) */
#define RBS_K_EMPTY 6       /* empty square block */

typedef struct rbs_plan rbs_plan;

void rbs_options_default(rbs_options *opt);

/* Analysis on HOST arrays.  fmt RBS_FMT_CSC: ptr = column pointer (n+1),
 * idx = row indices, diagonal first in each column for RBS_FORWARD and last
 * for RBS_BACKWARD (the layout main.cu:157-238 produces).  RBS_FMT_CSR:
 * ptr = row pointer, any order inside a row.  lv >= 0, or -1 for the
 * reference's automatic rule.  opt may be NULL. */
int rbs_analyse(const int *ptr, const int *idx, const double *val, int n, int nnz, int fmt,
                int substitution, int lv, const rbs_options *opt, rbs_plan **plan);

/* Analysis on DEVICE arrays (the inputs of recblocking_solver_cuda). */
int rbs_analyse_device(const int *d_ptr, const int *d_idx, const double *d_val, int n, int nnz,
                       int fmt, int substitution, int lv, const rbs_options *opt, rbs_plan **plan);

/* Solve with k right-hand sides, DEVICE arrays, column-major with leading
 * dimension ld (>= n).  b is read only (the reference overwrites d_b;
 * recblocking_calculate.h:39).  Returns when the solve is complete.
 * stats may be NULL. */
int rbs_solve(rbs_plan *plan, const double *d_b, double *d_x, int k, int ld, int prec,
              rbs_stats *stats);

/* Same with HOST arrays: copies in, solves, copies out. */
int rbs_solve_host(rbs_plan *plan, const double *b, double *x, int k, int ld, int prec,
                   rbs_stats *stats);

/* Asynchronous variant: enqueue on the plan's stream and return.  Status of
 * the device-side checks is collected by rbs_plan_sync. */
int rbs_solve_async(rbs_plan *plan, const double *d_b, double *d_x, int k, int ld, int prec);
/* Asynchronous HOST-array solve (no counterpart in the reference): b is
 * uploaded on a copy stream into one of two plan-owned staging slots, solved
 * on the plan's stream, and x downloaded on a second copy stream, so
 * consecutive calls overlap one solve with the neighbouring calls' copies.
 * Returns after enqueueing; b must stay unchanged and x unread until
 * rbs_plan_sync, which waits for every enqueued solve and reports the
 * device-side checks.  Use page-locked (pinned) b and x for the copies to
 * overlap.  RBS_PREC_MIXED runs synchronously (its refinement checks each
 * correction on the host). */
int rbs_solve_host_async(rbs_plan *plan, const double *b, double *x, int k, int ld, int prec);
int rbs_plan_sync(rbs_plan *plan);

/* cudaStream_t passed as void* (NULL = the plan's own stream). */
int rbs_plan_set_stream(rbs_plan *plan, void *stream);
/* Allocate the plan's work vectors for k (1..128) right-hand sides now, so
 * later solves of up to k columns allocate and free no device memory (no
 * counterpart in the reference, which allocates inside its solver). */
int rbs_plan_reserve(rbs_plan *plan, int k);
int rbs_plan_info_get(const rbs_plan *plan, rbs_plan_info *info);

/* Many independent systems as one plan (no counterpart in the reference,
 * which solves one system per run).  The `count` systems (host arrays, each
 * in the format of rbs_analyse, all of one direction) are placed on the
 * diagonal of one block-diagonal matrix and analysed together: their level
 * sets interleave in the level order, so a single solve walks all of them
 * at once and every launch carries rows of many systems.  row_offsets
 * (count+1 entries, output) gives where system i's rows start in the packed
 * right-hand sides and solutions passed to rbs_solve / rbs_solve_host.
 * lv = -1 means 0 here: one triangle, one persistent launch per pass. */
int rbs_batch_analyse(int count, const int *const *ptr, const int *const *idx, const double *const *val,
                      const int *n, const int *nnz, int fmt, int substitution, int lv, const rbs_options *opt,
                      rbs_plan **plan, int *row_offsets);

/* ---- request serving (no counterpart in the reference) ----------------
 * A server keeps analysed factors resident on the device (each with its own
 * CUDA stream and work vectors reserved at admission for the batch width,
 * so serving allocates no device memory per solve).  Submitted requests
 * (column-major n x k b and x, host arrays or device arrays, a precision)
 * queue per factor.  One dispatcher thread issues all device work: a factor
 * that is idle takes every queued request of one precision that fits the
 * batch width and solves them as ONE multi-RHS solve, reading device
 * requests' columns in place; requests arriving meanwhile join its next
 * batch, and the batches of all factors overlap on the device (mixed
 * precision refines each factor's batch on its own schedule).  A factor is
 * admitted only if its plan plus work vectors fit the remaining HBM budget;
 * a factor's first host-array request also charges its host staging
 * (RBS_ERR_BUDGET otherwise).  All factors must live on the device that was
 * current when the server was created. */
typedef struct rbs_server rbs_server;
typedef struct rbs_server_stats {
    long long completed;    /* requests finished since the last reset */
    long long solves;       /* right-hand sides solved */
    long long batches;      /* multi-RHS solves run */
    double mean_batch_rhs;  /* right-hand sides per batch */
    double p50_ms, p99_ms;  /* request latency, submit -> result in x */
    double solves_per_s;    /* right-hand sides / (last completion - first submit) */
    int factors;
    long long hbm_used;     /* bytes charged against the budget */
} rbs_server_stats;

int rbs_server_create(long long hbm_budget_bytes, int max_batch_rhs, rbs_server **server);
/* On success the server owns the plan (freed by rbs_server_destroy). */
int rbs_server_add_factor(rbs_server *server, rbs_plan *plan, int *factor_id);
/* Several small factors served as one unit: batch_plan is the block-diagonal
 * plan of rbs_batch_analyse over them, row_offsets its count + 1 offsets.
 * Factor i of the group gets factor_ids[i] (its own n = row_offsets[i+1] -
 * row_offsets[i]; requests use that n as their leading dimension); one
 * launch serves queued requests of all members at once, column c carrying
 * the c-th queued column of every member.  The server owns the plan. */
int rbs_server_add_group(rbs_server *server, rbs_plan *batch_plan, int count, const int *row_offsets,
                         int *factor_ids);
/* b and x must stay valid until rbs_server_wait returns for the ticket. */
int rbs_server_submit(rbs_server *server, int factor_id, const double *b, double *x, int k, int prec,
                      long long *ticket);
/* The same with DEVICE arrays (leading dimension n), read and written in
 * place by the batch's kernels; they must stay valid until the wait. */
int rbs_server_submit_device(rbs_server *server, int factor_id, const double *d_b, double *d_x, int k, int prec,
                             long long *ticket);
int rbs_server_wait(rbs_server *server, long long ticket, double *latency_ms, int *batch_rhs);
int rbs_server_stats_get(rbs_server *server, rbs_server_stats *stats);
int rbs_server_reset_stats(rbs_server *server);
int rbs_server_destroy(rbs_server *server);

/* Copy a named integer (or, for "recblock_Val", double) output of the
 * analysis into dst.  Names follow the reference's variables: "levelItem",
 * "loc_off", "tmp_off", "blk_m", "blk_n", "blk_nnz", "subtri_up",
 * "subtri_down", "subrec_up", "subrec_down", "subrec_right", "subrec_left",
 * "ptr_offset", "index_offset", "dcsrindex_offset", "recblock_Ptr",
 * "recblock_Index", "recblock_Val", "recblock_dcsr_rowidx", "method", "nlv",
 * "longrow", "m_new_dcsr", "lvl_ptr", "lvl_item", "m_lv", "offset_lv",
 * "nnz_lv", "sizes", plus this library's "kernel" (RBS_K_* per block).
 * With dst == NULL only *count is set.  Returns RBS_ERR_ARG for an unknown
 * name or cap < count. */
int rbs_plan_export(const rbs_plan *plan, const char *name, void *dst, long long cap,
                    long long *count);

int rbs_plan_free(rbs_plan *plan);

/* ILU(0) of a square CSR matrix on the device (no counterpart in the
 * reference, which solves with factors it is given): d_lu receives, in A's
 * pattern, the strict lower part of L (unit diagonal implied) and U (on and
 * above the diagonal).  Columns must ascend in every row and every row must
 * hold its diagonal (RBS_ERR_STRUCTURE otherwise, and on a zero pivot).  The
 * factor is the serial row-wise IKJ result bit for bit.  L and U then go to
 * rbs_analyse as RBS_FMT_CSR triangles (L with its unit diagonal written
 * out, RBS_FORWARD; U, RBS_BACKWARD).  Uses opt->device and
 * opt->spin_limit; allocates O(n) scratch; returns when done. */
int rbs_ilu0_device(const int *d_rowptr, const int *d_colidx, const double *d_val, int n, int nnz, double *d_lu,
                    const rbs_options *opt);

/* IC(0) (incomplete Cholesky, zero fill) of a symmetric positive definite
 * matrix on the device (no counterpart in the reference): input is A's
 * lower triangle as CSR, columns ascending and the diagonal last in every
 * row; d_l receives L in that pattern (L L^T equals A on it).  The factor is
 * the serial row algorithm (l_ik = (a_ik - sum_{j<k} l_ij l_kj) / l_kk, then
 * l_ii = sqrt(a_ii - sum_j l_ij^2), ascending columns, separately rounded
 * products) bit for bit.  RBS_ERR_STRUCTURE for a bad pattern or a pivot
 * <= 0.  The preconditioner apply needs one plan for L (RBS_FMT_CSR,
 * RBS_FORWARD) and one for L^T, which is the same arrays read as CSC
 * (RBS_FMT_CSC, RBS_BACKWARD): no transpose is formed. */
int rbs_ic0_device(const int *d_rowptr, const int *d_colidx, const double *d_val, int n, int nnz, double *d_l,
                   const rbs_options *opt);

/* ---- Matrix Market input on the device --------------------------------
 * Replaces mmio_info + mmio_data (mmio_highlevel.h:7-296) and the driver's
 * triangle extraction and CSR->CSC transposition (main.cu:151-236,
 * tranpose.h:7-54).  The host reads the banner and size line and streams the
 * entry bytes to the device, which tokenizes them, converts the numbers,
 * mirrors symmetric / Hermitian entries (diagonal once; skew-symmetric files
 * are read as general, as mmio_data does) and builds the CSR.
 *   - CSR layout as mmio_data's: rows ascending, file order inside a row,
 *     each mirrored entry placed as if it followed its entry in the file.
 *   - Values carry the bits fscanf("%lg") gives (correctly rounded; tokens
 *     outside the device's exact window go to the host's strtod, counted in
 *     host_values); integer fields convert from C ints; pattern -> 1.0;
 *     complex -> the real part.
 *   - Errors instead of the reference's undefined behaviour: a truncated or
 *     malformed entry (RBS_ERR_ARG), an index outside [1, m] x [1, n]
 *     (RBS_ERR_STRUCTURE), array storage or an unknown field
 *     (RBS_ERR_UNSUPPORTED); the message names the first bad entry.
 * The handle holds the CSR in HBM (opt->device; opt may be NULL). */
#define RBS_MTX_REAL 0
#define RBS_MTX_INTEGER 1
#define RBS_MTX_PATTERN 2
#define RBS_MTX_COMPLEX 3
typedef struct rbs_mtx rbs_mtx;
typedef struct rbs_mtx_info {
    int m, n;
    long long nnz_file;   /* entries in the file (the size line's count) */
    long long nnz;        /* entries after symmetric expansion (mmio_data's nnz) */
    long long nnz_lower;  /* strictly lower entries of the expanded matrix */
    long long nnz_upper;  /* strictly upper entries */
    int field;            /* RBS_MTX_* */
    int symmetric;        /* 1: symmetric or Hermitian file, mirrored */
    long long host_values;  /* values converted by the host's strtod */
    double read_ms;       /* header + file bytes into HBM */
    double parse_ms;      /* tokens, numbers, expansion and CSR on the device */
} rbs_mtx_info;
int rbs_mtx_read(const char *path, const rbs_options *opt, rbs_mtx **mtx);
/* the same from a file image in host memory */
int rbs_mtx_read_buffer(const void *bytes, long long len, const rbs_options *opt, rbs_mtx **mtx);
int rbs_mtx_info_get(const rbs_mtx *mtx, rbs_mtx_info *info);
/* A's CSR into caller device arrays: rowptr[m+1], colidx[nnz], val[nnz] */
int rbs_mtx_csr(const rbs_mtx *mtx, int *d_rowptr, int *d_colidx, double *d_val);
/* main.cu:157-198 (+ tranpose.h for RBS_FMT_CSC): the square matrix's
 * strictly lower (RBS_FORWARD) or upper (RBS_BACKWARD) entries with a unit
 * diagonal, the diagonal last (forward) or first (backward) in each row of
 * the CSR; RBS_FMT_CSC gives that CSR's stable transposition, the layout
 * rbs_analyse / recblocking_solver_cuda take.  Strict entry number r, in the
 * CSR's row-major order, takes d_strict_val[r] when d_strict_val is not
 * NULL (main.cu draws these with rand()), else A's value.  Output sizes:
 * m+1 pointers, m + nnz_lower (forward) or m + nnz_upper entries.  A
 * non-square matrix is RBS_ERR_STRUCTURE. */
int rbs_mtx_triangle(const rbs_mtx *mtx, int substitution, int fmt, const double *d_strict_val, int *d_ptr,
                     int *d_idx, double *d_val);
int rbs_mtx_free(rbs_mtx *mtx);
/* Matrix Market output (the reference's mm_write_banner /
 * mm_write_mtx_crd_size, mmio.h): a host CSR written as a coordinate file,
 * entries in row-major order, values with %.17g (read back bit for bit),
 * "pattern" when val is NULL; symmetric != 0 writes only entries with
 * column <= row under a "symmetric" banner. */
int rbs_mtx_write(const char *path, int m, int n, const int *rowptr, const int *colidx, const double *val,
                  int symmetric);

/* Plan serialisation (no counterpart in the reference, which repeats its
 * analysis in every process): rbs_plan_save writes the analysis -- level
 * order, labels, block bounds, kernel choice and every execution layout --
 * to a file; rbs_plan_load reads it back and, unless opt->host_only, builds
 * the device state, with no level search, partition or kernel timing.
 * opt may be NULL (defaults).  A file from another build is rejected
 * (RBS_ERR_ARG). */
int rbs_plan_save(const rbs_plan *plan, const char *path);
int rbs_plan_load(const char *path, const rbs_options *opt, rbs_plan **plan);

/* Per-block device timing (no counterpart in the reference, which times the
 * whole walk with gettimeofday, recblocking_calculate.h:45,164-165).  When
 * enabled, every FP64/FP32 solve records CUDA events around each block's
 * kernels; rbs_plan_block_times returns, per block in the reference's block
 * order, the accumulated milliseconds and the number of timed solves, and
 * the algorithmic bytes one FP64 single-RHS pass of the block moves
 * (entries x 12 + row pointers + b, x and diagonal traffic).
 * Enabling/disabling resets the accumulators. */
int rbs_plan_profile(rbs_plan *plan, int enable);
int rbs_plan_block_times(const rbs_plan *plan, double *ms, double *bytes, long long *solves, int cap);

/* Message of the last error on the calling thread ("" if none). */
const char *rbs_last_error(void);

/* main.cu:245-254: lv for the -lv -1 option. */
int rbs_auto_lv(int m, int device_id);

/* Solve without allocating device memory.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc/cudaFree where they need a solve:
 * a host framework whose caching allocator already holds the device's free
 * memory (a raw cudaMalloc fails, and cudaFree would synchronise the whole
 * device), or a latency-critical loop that forbids allocation after
 * start-up.  The caller passes a triangular CSR (row pointer, column
 * indices, values with the diagonal stored in each row, any order inside a
 * row), b and x, all device pointers; lower for RBS_FORWARD, upper for
 * RBS_BACKWARD.  No analysis: rows are solved in index order by the
 * sync-free kernel.  stream may be NULL (legacy default stream).  The call
 * is synchronous: it reads the row pointer's last entry back to the host
 * and returns when the solve is complete.  A row without its diagonal (or
 * with a zero one) or an entry on the wrong side of the diagonal or outside
 * [0, n) gives RBS_ERR_STRUCTURE; such an entry is never waited on.
 *
 * Scratch: a static device array of RBS_NOALLOC_MAX_ROWS doubles plus 256
 * bytes (about 8 MB), held by every GPU that loads this library until the
 * process exits.  n > RBS_NOALLOC_MAX_ROWS is rejected with RBS_ERR_ARG.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it for the life of the process; do not
 * use this entry point across a cudaDeviceReset.  Every call on a device shares the
 * one array: calls whose work overlaps on the GPU (different streams or
 * host threads) race and corrupt each other's results; serialise them. */
#define RBS_NOALLOC_MAX_ROWS (1 << 20)
int rbs_sptrsv_csr_noalloc(const int *d_rowptr, const int *d_colidx, const double *d_val, int n,
                           int substitution, const double *d_b, double *d_x, void *stream);

/* ---- reference-signature shims ---------------------------------------- */

/* recblocking_solver_cuda.h:21-32.  Same arguments and meaning: device CSC
 * input, solution in d_x, cal_time = mean solve ms over 200 repetitions is
 * ADDED to *cal_time (the reference accumulates), *preprocess_time = analysis
 * ms (the reference sets it for forward only; this sets it for both).
 * Difference: d_b is left as the caller passed it.  Errors are reported
 * through rbs_last_error(). */
void recblocking_solver_cuda(int *d_cscColPtrTR, int *d_cscRowIdxTR, double *d_cscValTR, int m, int n,
                             int nnzTR, double *d_x, double *d_b, int substitution, int lv,
                             double *cal_time, double *preprocess_time);

/* recblocking_solver.h:16-28.  Host CSC input, host b and x; x_ref unused
 * (as in the reference); rhs columns of b/x stored column-major with
 * leading dimension m (the reference hard-codes rhs = 1 in the GPU path). */
void recblocking_solver(int *cscColPtr, int *cscRowIdx, double *cscVal, int m, int n, int nnz, double *b,
                        double *x, double *x_ref, int rhs, int lv, int substitution, double *cal_time);

#ifdef __cplusplus
}
#endif
#endif
