/*
 * gen.c -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The seeded synthetic systems of include/rbs_gen.h restated in plain C, so
 * that the CPU side of the benchmark builds its inputs without loading the
 * library under test.  tests/test_oracle_gen.py checks that these arrays
 * equal rbs_gen_lower_csr / rbs_gen_uniform bit for bit.
 *
 * Random words: MT19937-64 (M. Matsumoto and T. Nishimura, "Mersenne
 * Twister: a 623-dimensionally equidistributed uniform pseudorandom number
 * generator", ACM TOMACS 8(1), 1998; the 64-bit parameter set of T. Nishimura,
 * ACM TOMACS 10(4), 2000), with the seeding recurrence the C++ standard
 * gives std::mt19937_64.  Transforms: 53-bit uniforms, multiply-high
 * integers below a bound, Knuth's product-of-uniforms Poisson sampler,
 * Floyd's subset sampling, an inverse-CDF Zipf draw.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

enum { MT_N = 312, MT_M = 156 };

typedef struct {
    uint64_t mt[MT_N];
    int i;
} mt64;

static void mt64_seed(mt64 *s, uint64_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < MT_N; ++i) s->mt[i] = 6364136223846793005ULL * (s->mt[i - 1] ^ (s->mt[i - 1] >> 62)) + (uint64_t)i;
    s->i = MT_N;
}

static uint64_t mt64_next(mt64 *s) {
    static const uint64_t mag[2] = {0ULL, 0xB5026F5AA96619E9ULL};
    const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
    if (s->i >= MT_N) {
        int k;
        uint64_t x;
        for (k = 0; k < MT_N - MT_M; ++k) {
            x = (s->mt[k] & upper) | (s->mt[k + 1] & lower);
            s->mt[k] = s->mt[k + MT_M] ^ (x >> 1) ^ mag[x & 1];
        }
        for (; k < MT_N - 1; ++k) {
            x = (s->mt[k] & upper) | (s->mt[k + 1] & lower);
            s->mt[k] = s->mt[k + MT_M - MT_N] ^ (x >> 1) ^ mag[x & 1];
        }
        x = (s->mt[MT_N - 1] & upper) | (s->mt[0] & lower);
        s->mt[MT_N - 1] = s->mt[MT_M - 1] ^ (x >> 1) ^ mag[x & 1];
        s->i = 0;
    }
    uint64_t y = s->mt[s->i++];
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= y >> 43;
    return y;
}

static double unit(mt64 *s) { return (double)(mt64_next(s) >> 11) * (1.0 / 9007199254740992.0); }
static double uniform(mt64 *s, double lo, double hi) { return lo + (hi - lo) * unit(s); }
static uint64_t below(mt64 *s, uint64_t r) { return (uint64_t)(((unsigned __int128)mt64_next(s) * r) >> 64); }

static int poisson(mt64 *s, double lambda) {
    const double limit = exp(-lambda);
    int k = 0;
    double p = 1.0;
    do {
        ++k;
        p *= unit(s);
    } while (p > limit);
    return k - 1;
}

static int cmp_ll(const void *a, const void *b) {
    const long long x = *(const long long *)a, y = *(const long long *)b;
    return (x > y) - (x < y);
}

/* Floyd: k distinct values of [lo, lo+range), ascending, into out (k slots).
 * `picked` is a scratch array of k entries kept sorted for the membership
 * test (the set, hence the result, does not depend on how it is kept). */
static int sample_distinct(mt64 *s, long long lo, long long range, int k, int *out, long long *picked) {
    if (k <= 0 || range <= 0) return 0;
    if (k >= range) {
        for (long long v = 0; v < range; ++v) out[v] = (int)(lo + v);
        return (int)range;
    }
    int np = 0;
    for (long long j = range - k; j < range; ++j) {
        const long long t = (long long)below(s, (uint64_t)(j + 1));
        int a = 0, b = np;
        while (a < b) {
            const int mid = (a + b) / 2;
            if (picked[mid] < t) a = mid + 1;
            else b = mid;
        }
        const long long v = (a < np && picked[a] == t) ? j : t;
        a = 0;
        b = np;  /* insert v, keeping the array sorted */
        while (a < b) {
            const int mid = (a + b) / 2;
            if (picked[mid] <= v) a = mid + 1;
            else b = mid;
        }
        memmove(picked + a + 1, picked + a, sizeof(long long) * (size_t)(np - a));
        picked[a] = v;
        ++np;
    }
    qsort(picked, (size_t)np, sizeof(long long), cmp_ll);
    for (int q = 0; q < np; ++q) out[q] = (int)(lo + picked[q]);
    return np;
}

/* inverse CDF over {1..kmax}: the first k with u < cdf[k-1] */
static int zipf_draw(mt64 *s, const double *cdf, int kmax) {
    const double u = unit(s);
    int a = 0, b = kmax;
    while (a < b) {
        const int mid = (a + b) / 2;
        if (cdf[mid] <= u) a = mid + 1;
        else b = mid;
    }
    const int k = a + 1;
    return k > kmax ? kmax : k;
}

int orc_gen_lower_csr(int kind, int n_in, int grid, double lambda, int band, double zipf_alpha, int zipf_max,
                      int chain_bw, unsigned long long seed, int *n_out, long long *nnz_out, int **rowptr_out,
                      int **colidx_out, double **val_out) {
    const int n = kind == 1 ? grid * grid : n_in;
    if (n <= 0 || kind < 0 || kind > 4) return 1;
    mt64 *s = (mt64 *)malloc(sizeof(mt64));
    int *rp = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    size_t cap = (size_t)n * 4 + 16, nnz = 0;
    int *ci = (int *)malloc(sizeof(int) * cap);
    double *va = (double *)malloc(sizeof(double) * cap);
    const int rmax = kind == 2 ? zipf_max : kind == 3 ? chain_bw : kind == 1 ? 2 : 0;
    size_t rowcap = 64;
    int *row = (int *)malloc(sizeof(int) * rowcap);
    long long *picked = (long long *)malloc(sizeof(long long) * rowcap);
    double *cdf = NULL;
    if (!s || !rp || !ci || !va || !row || !picked) goto oom;
    (void)rmax;
    mt64_seed(s, seed);
    if (kind == 2) {
        cdf = (double *)malloc(sizeof(double) * (size_t)(zipf_max > 0 ? zipf_max : 1));
        if (!cdf) goto oom;
        double sum = 0;
        for (int k = 1; k <= zipf_max; ++k) {
            sum += pow((double)k, -zipf_alpha);
            cdf[k - 1] = sum;
        }
        for (int k = 0; k < zipf_max; ++k) cdf[k] /= sum;
    }
    rp[0] = 0;
    for (int i = 0; i < n; ++i) {
        int len = 0;
        long long lo = 0, range = 0;
        int want = 0;
        if (kind == 0) {
            lo = band > 0 ? (i - band > 0 ? i - band : 0) : 0;
            range = i - lo;
            want = poisson(s, lambda);
            if (want > range) want = (int)range;
        } else if (kind == 2) {
            want = i > 0 ? zipf_draw(s, cdf, zipf_max) : 0;
            if (want > i) want = i;
            lo = 0;
            range = i;
        }
        size_t need = (size_t)(want > chain_bw ? want : chain_bw) + 2;
        if (need > rowcap) {
            while (rowcap < need) rowcap *= 2;
            int *r2 = (int *)realloc(row, sizeof(int) * rowcap);
            long long *p2 = (long long *)realloc(picked, sizeof(long long) * rowcap);
            if (!r2 || !p2) {
                if (r2) row = r2;
                if (p2) picked = p2;
                goto oom;
            }
            row = r2;
            picked = p2;
        }
        if (kind == 0 || kind == 2) {
            len = sample_distinct(s, lo, range, want, row, picked);
        } else if (kind == 1) {
            const int r = i / grid, c = i % grid;
            if (r > 0) row[len++] = i - grid;
            if (c > 0) row[len++] = i - 1;
        } else if (kind == 3) {
            for (int d = chain_bw; d >= 1; --d)
                if (i - d >= 0) row[len++] = i - d;
        }
        if (nnz + (size_t)len + 1 > cap) {
            while (nnz + (size_t)len + 1 > cap) cap *= 2;
            int *c2 = (int *)realloc(ci, sizeof(int) * cap);
            double *v2 = (double *)realloc(va, sizeof(double) * cap);
            if (!c2 || !v2) {
                if (c2) ci = c2;
                if (v2) va = v2;
                goto oom;
            }
            ci = c2;
            va = v2;
        }
        double asum = 0;
        for (int q = 0; q < len; ++q) {
            const double v = uniform(s, -1.0, 1.0);
            ci[nnz] = row[q];
            va[nnz] = v;
            ++nnz;
            asum += fabs(v);
        }
        ci[nnz] = i;
        va[nnz] = 1.0 + asum;
        ++nnz;
        if (nnz > (size_t)0x7fffffff) goto oom;
        rp[i + 1] = (int)nnz;
    }
    free(s);
    free(row);
    free(picked);
    free(cdf);
    *n_out = n;
    *nnz_out = (long long)nnz;
    *rowptr_out = rp;
    *colidx_out = ci;
    *val_out = va;
    return 0;
oom:
    free(s);
    free(rp);
    free(ci);
    free(va);
    free(row);
    free(picked);
    free(cdf);
    return 2;
}

int orc_gen_uniform(unsigned long long seed, long long n, double lo, double hi, double *out) {
    if (n < 0 || (n > 0 && !out)) return 1;
    mt64 *s = (mt64 *)malloc(sizeof(mt64));
    if (!s) return 2;
    mt64_seed(s, seed);
    for (long long i = 0; i < n; ++i) out[i] = uniform(s, lo, hi);
    free(s);
    return 0;
}
