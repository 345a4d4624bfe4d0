/*
 * rbs_gen.h -- seeded synthetic triangular systems.
 *
 * The reference evaluates on SuiteSparse Matrix Market files (README.md:17),
 * which are not available offline.  These generators produce seeded
 * stand-ins with the structural shapes the benchmark configurations name:
 * a banded random lower factor, the lower factor of the 2D 5-point
 * Laplacian, power-law row lengths and a banded chain.  They are utilities
 * for tests, the benchmark and the CLI; they are not part of the drop-in
 * boundary (rbs.h).
 *
 * Every generator returns a LOWER triangular matrix L in CSR with column
 * indices ascending inside each row, so the diagonal is the LAST entry of
 * each row.  The forward input of the solver is CSC(L) (diagonal first in
 * each column, as main.cu:157-176 + tranpose.h:7 produce it); the backward
 * input for U = L^T is CSC(U), which is exactly the CSR arrays of L
 * (diagonal last in each column, as main.cu:178-198 produce it).
 *
 * Values: off-diagonals U(-1,1); diagonal = 1 + sum |off-diagonals of the
 * row| (strict diagonal dominance by rows of L).
 */
#ifndef RBS_GEN_H
#define RBS_GEN_H

#ifdef __cplusplus
extern "C" {
#endif

enum rbs_gen_kind {
    RBS_GEN_BAND_POISSON = 0, /* k ~ Poisson(lambda) per row, distinct cols uniform in [max(0,i-band), i) */
    RBS_GEN_LAPLACE2D = 1,    /* tril of the 5-point Laplacian on grid x grid, natural order */
    RBS_GEN_ZIPF = 2,         /* k ~ Zipf(alpha) on {1..zipf_max}, capped at i, distinct cols uniform in [0, i) */
    RBS_GEN_CHAIN = 3,        /* cols {i-bw, ..., i-1} (the ones >= 0) */
    RBS_GEN_DIAG = 4          /* diagonal only */
};

typedef struct rbs_gen_spec {
    int kind;                 /* rbs_gen_kind */
    int n;                    /* rows (ignored for LAPLACE2D: n = grid*grid) */
    int grid;                 /* LAPLACE2D side */
    double lambda;            /* BAND_POISSON mean off-diagonals per row */
    int band;                 /* BAND_POISSON band width (0 = unbounded, cols in [0,i)) */
    double zipf_alpha;        /* ZIPF exponent */
    int zipf_max;             /* ZIPF support {1..zipf_max} */
    int chain_bw;             /* CHAIN bandwidth */
    unsigned long long seed;  /* one seed per matrix */
} rbs_gen_spec;

/* Generate L (CSR, see above).  Arrays are allocated with malloc and must be
 * released with rbs_gen_free.  Returns 0 on success, nonzero on bad spec or
 * allocation failure. */
int rbs_gen_lower_csr(const rbs_gen_spec *spec, int *n_out, long long *nnz_out,
                      int **rowptr, int **colidx, double **val);

/* n values U(lo, hi) from a seeded stream. */
int rbs_gen_uniform(unsigned long long seed, long long n, double lo, double hi, double *out);

void rbs_gen_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
