// Host analysis under the compiler's sanitizers (built and run by
// tests/test_sanitizers.py with -fsanitize=thread, or address + undefined):
// a banded system large enough for every threaded step (transposition, row
// builds, statistics, pool fill, level-chunk and ELL layouts) as CSR forward
// and as CSC backward, in AUTO and TUNE, and a 40-system batch whose
// level-chunk layouts are built per system on host threads, saved to a plan
// file and loaded back; the FP32 copy of its value pool.
#include <algorithm>
#include <cstdio>
#include <random>

#include "rbs_internal.h"

using namespace rbs;

// The host analysis reaches the device block extraction (dev_pools.cu) only
// from rbs_analyse_device; this host-only build never takes that path, so
// the device steps are stand-ins that report it.
namespace rbs {
DevRows::~DevRows() {}
int dev_block_counts(DevRows &, int, int, const std::vector<long long> &, std::vector<int> &, std::vector<double> &,
                     std::vector<int> &, std::string &err) {
    err = "no device in this build";
    return RBS_ERR_UNSUPPORTED;
}
int dev_local_levels(DevRows &, int, int, long long, std::vector<int> &, std::string &err) {
    err = "no device in this build";
    return RBS_ERR_UNSUPPORTED;
}
int dev_pool_fill(DevRows &, int, int, long long, long long, bulk_vector<int> &, bulk_vector<double> &,
                  std::string &err) {
    err = "no device in this build";
    return RBS_ERR_UNSUPPORTED;
}
}  // namespace rbs

static void band(int n, int bw, double lam, unsigned seed, std::vector<int> &rp, std::vector<int> &ci,
                 std::vector<double> &va) {
    std::mt19937_64 g(seed);
    std::poisson_distribution<int> pois(lam);
    rp.assign(1, 0);
    ci.clear();
    va.clear();
    for (int i = 0; i < n; ++i) {
        const int k = std::min(pois(g), std::min(i, bw));
        std::vector<int> cols;
        std::uniform_int_distribution<int> pick(std::max(0, i - bw), std::max(0, i - 1));
        while ((int)cols.size() < k) {
            const int c = pick(g);
            if (std::find(cols.begin(), cols.end(), c) == cols.end()) cols.push_back(c);
        }
        std::sort(cols.begin(), cols.end());
        for (int c : cols) {
            ci.push_back(c);
            va.push_back(0.1);
        }
        ci.push_back(i);
        va.push_back(2.0);
        rp.push_back((int)ci.size());
    }
}

static rbs_options opts(int select) {
    rbs_options o{};
    o.select = select;
    o.device = -1;
    o.host_only = 1;
    o.max_rhs = 1;
    o.mixed = 1;
    o.ir_tol = 1e-13;
    o.ir_max_iter = 8;
    o.spin_limit = 1 << 22;
    return o;
}

int main(int argc, char **argv) {
    int bad = 0;
    std::vector<int> rp, ci;
    std::vector<double> va;
    band(1 << 18, 64, 5.0, 1, rp, ci, va);
    const int n = (int)rp.size() - 1, nnz = rp[(size_t)n];
    for (int sel : {RBS_SELECT_AUTO, RBS_SELECT_TUNE}) {
        std::string err;
        Plan P, Q;
        bad |= analyse_host(P, rp.data(), ci.data(), va.data(), n, nnz, RBS_FMT_CSR, RBS_FORWARD, 3, opts(sel), err, nullptr);
        // the lower CSR read as the CSC of its transpose: a backward system
        bad |= analyse_host(Q, rp.data(), ci.data(), va.data(), n, nnz, RBS_FMT_CSC, RBS_BACKWARD, 2, opts(sel), err, nullptr);
        if (!err.empty()) std::printf("%s\n", err.c_str());
    }
    std::vector<int> bp(1, 0), bi, segs;
    std::vector<double> bv;
    for (int s = 0; s < 40; ++s) {
        std::vector<int> r, c;
        std::vector<double> v;
        band(2000 + 300 * s, 32, 3.0, 100 + s, r, c, v);
        const int r0 = (int)bp.size() - 1;
        segs.push_back(r0);
        for (size_t i = 0; i + 1 < r.size(); ++i) {
            for (int k = r[i]; k < r[i + 1]; ++k) {
                bi.push_back(c[(size_t)k] + r0);
                bv.push_back(v[(size_t)k]);
            }
            bp.push_back((int)bi.size());
        }
    }
    const int N = (int)bp.size() - 1, Z = (int)bi.size();
    for (int sel : {RBS_SELECT_AUTO, RBS_SELECT_TUNE}) {
        std::string err;
        Plan P, Q;
        bad |= analyse_host(P, bp.data(), bi.data(), bv.data(), N, Z, RBS_FMT_CSR, RBS_FORWARD, 0, opts(sel), err, &segs);
        if (P.lc_rec64.empty()) bad = 1;
        // the FP32 pool copy uploaded for mixed precision (converted on host threads)
        const bulk_vector<float> v32 = to_f32(P.val_pool);
        if (v32.size() != P.val_pool.size()) bad = 1;
        for (size_t i = 0; i < v32.size(); ++i)
            if (v32[i] != (float)P.val_pool[i]) bad = 1;
        // the plan file round trip (its digest is computed on host threads)
        const char *path = argc > 1 ? argv[1] : "analysis_driver.rbs";
        bad |= plan_save(P, path, err);
        bad |= plan_load(Q, path, err);
        if (Q.lc_rec64 != P.lc_rec64 || Q.col_pool != P.col_pool || Q.val_pool != P.val_pool || Q.ell_col != P.ell_col)
            bad = 1;
        std::remove(path);
        if (!err.empty()) std::printf("%s\n", err.c_str());
    }
    std::printf("analysis driver: %s\n", bad ? "FAILED" : "ok");
    return bad ? 1 : 0;
}
