// Seeded synthetic lower-triangular systems (see include/rbs_gen.h).
//
// Randomness: std::mt19937_64 for raw 64-bit words (its output sequence is
// fixed by the C++ standard); every transform to a distribution is written
// here so results do not depend on the standard library's distributions.
#include "rbs_gen.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <random>
#include <vector>

namespace {

struct Rng {
    std::mt19937_64 eng;
    explicit Rng(unsigned long long s) : eng(s) {}
    uint64_t bits() { return eng(); }
    // uniform in [0,1) with 53 random bits
    double unit() { return (double)(bits() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double lo, double hi) { return lo + (hi - lo) * unit(); }
    // uniform integer in [0, r) by the multiply-high method
    uint64_t below(uint64_t r) {
        return (uint64_t)(((unsigned __int128)bits() * (unsigned __int128)r) >> 64);
    }
    // Knuth's product-of-uniforms Poisson sampler (fine for lambda <= ~30)
    int poisson(double lambda) {
        const double limit = std::exp(-lambda);
        int k = 0;
        double p = 1.0;
        do {
            ++k;
            p *= unit();
        } while (p > limit);
        return k - 1;
    }
};

// Distinct values drawn uniformly from [lo, lo+range), k <= range, returned
// sorted ascending.  Floyd's subset-sampling algorithm.
void sample_distinct(Rng &rng, long long lo, long long range, int k, std::vector<int> &out) {
    out.clear();
    if (k <= 0 || range <= 0) return;
    if (k >= range) {
        for (long long v = 0; v < range; ++v) out.push_back((int)(lo + v));
        return;
    }
    std::vector<long long> picked;
    picked.reserve(k);
    for (long long j = range - k; j < range; ++j) {
        long long t = (long long)rng.below((uint64_t)(j + 1));
        bool seen = false;
        if (k <= 64) {
            for (long long p : picked)
                if (p == t) { seen = true; break; }
        } else {
            // picked stays sorted for larger k
            seen = std::binary_search(picked.begin(), picked.end(), t);
        }
        long long v = seen ? j : t;
        if (k <= 64) picked.push_back(v);
        else picked.insert(std::upper_bound(picked.begin(), picked.end(), v), v);
    }
    std::sort(picked.begin(), picked.end());
    for (long long p : picked) out.push_back((int)(lo + p));
}

struct ZipfTable {
    std::vector<double> cdf;  // cdf[k-1] = P(K <= k)
    ZipfTable(double alpha, int kmax) {
        cdf.resize(kmax);
        double s = 0;
        for (int k = 1; k <= kmax; ++k) {
            s += std::pow((double)k, -alpha);
            cdf[k - 1] = s;
        }
        for (auto &c : cdf) c /= s;
    }
    int draw(Rng &rng) const {
        double u = rng.unit();
        auto it = std::upper_bound(cdf.begin(), cdf.end(), u);
        int k = (int)(it - cdf.begin()) + 1;
        return k > (int)cdf.size() ? (int)cdf.size() : k;
    }
};

}  // namespace

extern "C" int rbs_gen_lower_csr(const rbs_gen_spec *spec, int *n_out, long long *nnz_out,
                                 int **rowptr_out, int **colidx_out, double **val_out) {
    if (!spec || !n_out || !nnz_out || !rowptr_out || !colidx_out || !val_out) return 1;
    int n = spec->kind == RBS_GEN_LAPLACE2D ? spec->grid * spec->grid : spec->n;
    if (n <= 0) return 1;
    Rng rng(spec->seed);
    std::vector<int> rowptr((size_t)n + 1, 0);
    std::vector<int> cols;
    std::vector<double> vals;
    cols.reserve((size_t)n * 4);
    vals.reserve((size_t)n * 4);
    std::vector<int> row;
    ZipfTable *zipf = nullptr;
    if (spec->kind == RBS_GEN_ZIPF) zipf = new ZipfTable(spec->zipf_alpha, spec->zipf_max);

    for (int i = 0; i < n; ++i) {
        row.clear();
        switch (spec->kind) {
        case RBS_GEN_BAND_POISSON: {
            long long lo = spec->band > 0 ? std::max(0, i - spec->band) : 0;
            long long range = i - lo;
            int k = rng.poisson(spec->lambda);
            if (k > range) k = (int)range;
            sample_distinct(rng, lo, range, k, row);
            break;
        }
        case RBS_GEN_LAPLACE2D: {
            int g = spec->grid;
            int r = i / g, c = i % g;
            if (r > 0) row.push_back(i - g);
            if (c > 0) row.push_back(i - 1);
            break;
        }
        case RBS_GEN_ZIPF: {
            int k = i > 0 ? zipf->draw(rng) : 0;
            if (k > i) k = i;
            sample_distinct(rng, 0, i, k, row);
            break;
        }
        case RBS_GEN_CHAIN: {
            for (int d = spec->chain_bw; d >= 1; --d)
                if (i - d >= 0) row.push_back(i - d);
            break;
        }
        case RBS_GEN_DIAG:
            break;
        default:
            delete zipf;
            return 1;
        }
        double asum = 0;
        for (int c : row) {
            double v = rng.uniform(-1.0, 1.0);
            cols.push_back(c);
            vals.push_back(v);
            asum += std::fabs(v);
        }
        cols.push_back(i);
        vals.push_back(1.0 + asum);
        if (cols.size() > (size_t)0x7fffffff) {
            delete zipf;
            return 2;
        }
        rowptr[i + 1] = (int)cols.size();
    }
    delete zipf;

    size_t nnz = cols.size();
    int *rp = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    int *ci = (int *)malloc(sizeof(int) * (nnz ? nnz : 1));
    double *va = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
    if (!rp || !ci || !va) {
        free(rp); free(ci); free(va);
        return 2;
    }
    std::copy(rowptr.begin(), rowptr.end(), rp);
    std::copy(cols.begin(), cols.end(), ci);
    std::copy(vals.begin(), vals.end(), va);
    *n_out = n;
    *nnz_out = (long long)nnz;
    *rowptr_out = rp;
    *colidx_out = ci;
    *val_out = va;
    return 0;
}

extern "C" int rbs_gen_uniform(unsigned long long seed, long long n, double lo, double hi, double *out) {
    if (n < 0 || (n > 0 && !out)) return 1;
    Rng rng(seed);
    for (long long i = 0; i < n; ++i) out[i] = rng.uniform(lo, hi);
    return 0;
}

extern "C" void rbs_gen_free(void *p) { free(p); }
