// cli.cpp -- the sptrsv driver, a drop-in for recblock-sptrsv's main.cu.
//
//   sptrsv -d <device> -rhs <k> -lv <levels|-1> -forward|-backward -mtx <file.mtx>
//
// Same flags in the same fixed order (main.cu:51-132).  Like main.cu it
// reads the Matrix Market file into CSR (symmetric and Hermitian files are
// expanded, mmio_highlevel.h:137-296), keeps the strict lower (forward) or
// upper (backward) pattern with values rand()%10+1 and a unit diagonal
// (main.cu:157-198), draws x_ref = rand()%10+1 and b = T x_ref
// (main.cu:211-229), transposes to CSC (main.cu:236), applies the automatic
// lv rule (main.cu:245-254) and calls recblocking_solver_cuda, then checks
// sum|x - x_ref| / sum|x_ref| < 1e-4 (main.cu:296-317).  The file parsing,
// triangle extraction and transposition run on the device (rbs_mtx_*); the
// rand() draws and b stay on the host in main.cu's order.
// Differences: the random seed is time(NULL) unless RBS_SEED is set; -d
// also selects the CUDA device; -rhs k > 1 solves k columns (the reference
// hard-codes one); a wrong flag prints the usage and exits with status 2
// instead of returning 0 silently.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <algorithm>
#include <string>
#include <vector>

#include "rbs.h"

namespace {

int usage() {
    fprintf(stderr, "usage: sptrsv -d <device> -rhs <k> -lv <levels|-1> -forward|-backward -mtx <file.mtx>\n");
    return 2;
}

}  // namespace

int main(int argc, char **argv) {
    printf("---------------------------------------------------------------------------------------------\n");
    printf("PRECISION = 64-bit Double Precision\n");
    if (argc < 10) return usage();
    if (strcmp(argv[1], "-d") || strcmp(argv[3], "-rhs") || strcmp(argv[5], "-lv")) return usage();
    int device_id = atoi(argv[2]), rhs = atoi(argv[4]), lv = atoi(argv[6]);
    int substitution;
    if (!strcmp(argv[7], "-forward")) substitution = RBS_FORWARD;
    else if (!strcmp(argv[7], "-backward")) substitution = RBS_BACKWARD;
    else return usage();
    const char *filename = argv[9];
    printf("device_id = %i\nrhs = %i\nsubstitution = %i\n", device_id, rhs, substitution);
    printf("-------------- %s --------------\n", filename);
    const char *seed_env = getenv("RBS_SEED");
    srand(seed_env ? (unsigned)strtoul(seed_env, nullptr, 10) : (unsigned)time(nullptr));

    int ndev = 0;
    rbs_options ropt;
    rbs_options_default(&ropt);
    if (cudaGetDeviceCount(&ndev) == cudaSuccess && device_id >= 0 && device_id < ndev) {
        cudaSetDevice(device_id);
        ropt.device = device_id;
    }
    // mmio_info + mmio_data (main.cu:120-141) on the device
    rbs_mtx *A = nullptr;
    if (rbs_mtx_read(filename, &ropt, &A) != RBS_OK) {
        fprintf(stderr, "sptrsv: %s\n", rbs_last_error());
        return 1;
    }
    rbs_mtx_info inf;
    rbs_mtx_info_get(A, &inf);
    printf("input matrix A: ( %i, %i ) nnz = %i\n", inf.m, inf.n, (int)inf.nnz);
    if (inf.m != inf.n) {
        printf("we need square matrix. Exit!\n");
        rbs_mtx_free(A);
        return 1;
    }
    const int m = inf.m, n = inf.n;
    const long long nstrict = substitution == RBS_FORWARD ? inf.nnz_lower : inf.nnz_upper;
    const int nnz = (int)(m + nstrict);
    // main.cu:157-198: strict triangle of A's pattern with values drawn by
    // rand() % 10 + 1 in row-major order, unit diagonal; built on the device
    // as CSR (for b) and as its stable transposition (the solver's CSC,
    // main.cu:231-238)
    std::vector<double> sv((size_t)nstrict);
    for (auto &v : sv) v = rand() % 10 + 1;
    int *d_rp, *d_ci, *d_cp, *d_ri;
    double *d_sv, *d_tv, *d_va, *d_x, *d_b;
    const int k = rhs > 0 ? rhs : 1;
    cudaMalloc(&d_sv, sizeof(double) * std::max<size_t>(sv.size(), 1));
    cudaMalloc(&d_rp, sizeof(int) * (m + 1));
    cudaMalloc(&d_ci, sizeof(int) * nnz);
    cudaMalloc(&d_tv, sizeof(double) * nnz);
    cudaMalloc(&d_cp, sizeof(int) * (n + 1));
    cudaMalloc(&d_ri, sizeof(int) * nnz);
    cudaMalloc(&d_va, sizeof(double) * nnz);
    cudaMalloc(&d_x, sizeof(double) * (size_t)n * k);
    cudaMalloc(&d_b, sizeof(double) * (size_t)m * k);
    cudaMemcpy(d_sv, sv.data(), sizeof(double) * sv.size(), cudaMemcpyHostToDevice);
    if (rbs_mtx_triangle(A, substitution, RBS_FMT_CSR, d_sv, d_rp, d_ci, d_tv) != RBS_OK ||
        rbs_mtx_triangle(A, substitution, RBS_FMT_CSC, d_sv, d_cp, d_ri, d_va) != RBS_OK) {
        fprintf(stderr, "sptrsv: %s\n", rbs_last_error());
        rbs_mtx_free(A);
        return 1;
    }
    rbs_mtx_free(A);
    std::vector<int> trp((size_t)m + 1), tci((size_t)nnz);
    std::vector<double> tva((size_t)nnz);
    cudaMemcpy(trp.data(), d_rp, sizeof(int) * (m + 1), cudaMemcpyDeviceToHost);
    cudaMemcpy(tci.data(), d_ci, sizeof(int) * nnz, cudaMemcpyDeviceToHost);
    cudaMemcpy(tva.data(), d_tv, sizeof(double) * nnz, cudaMemcpyDeviceToHost);
    // main.cu:211-229
    std::vector<double> x_ref((size_t)n * k), b((size_t)m * k, 0.0), x((size_t)n * k, 0.0);
    for (auto &v : x_ref) v = rand() % 10 + 1;
    for (int r = 0; r < k; ++r)
        for (int i = 0; i < m; ++i)
            for (int j = trp[i]; j < trp[i + 1]; ++j) b[(size_t)r * m + i] += tva[j] * x_ref[(size_t)r * n + tci[j]];
    if (lv == -1) lv = rbs_auto_lv(m, device_id);
    while (lv > 0 && (1 << lv) > m) --lv;
    printf("lv = %i\n", lv);
    cudaMemcpy(d_b, b.data(), sizeof(double) * (size_t)m * k, cudaMemcpyHostToDevice);

    double cal_time = 0, preprocess_time = 0;
    if (k == 1) {
        recblocking_solver_cuda(d_cp, d_ri, d_va, m, n, nnz, d_x, d_b, substitution, lv, &cal_time, &preprocess_time);
    } else {
        rbs_options o;
        rbs_options_default(&o);
        o.max_rhs = k;
        o.lv_device_id = device_id;
        rbs_plan *plan = nullptr;
        if (rbs_analyse_device(d_cp, d_ri, d_va, m, nnz, RBS_FMT_CSC, substitution, lv, &o, &plan) == RBS_OK) {
            rbs_stats st;
            if (rbs_solve(plan, d_b, d_x, k, m, RBS_PREC_FP64, &st) == RBS_OK) cal_time = st.ms;
            rbs_plan_free(plan);
        }
    }
    const char *e = rbs_last_error();
    if (e && *e) {
        fprintf(stderr, "sptrsv: %s\n", e);
        return 1;
    }
    cudaMemcpy(x.data(), d_x, sizeof(double) * (size_t)n * k, cudaMemcpyDeviceToHost);
    printf("preprocess usetime = %.3lf ms\n", preprocess_time);
    printf("computation usetime = %.3lf ms\n", cal_time);
    printf("Performance = %.3lf gflops\n", (2.0 * nnz * k) / (cal_time * 1e6));
    for (void *p : {(void *)d_sv, (void *)d_rp, (void *)d_ci, (void *)d_tv, (void *)d_cp, (void *)d_ri,
                    (void *)d_va, (void *)d_x, (void *)d_b})
        cudaFree(p);
    double ref = 0, res = 0;
    for (size_t i = 0; i < x.size(); ++i) {
        ref += fabs(x_ref[i]);
        res += fabs(x[i] - x_ref[i]);
    }
    res = ref == 0 ? res : res / ref;
    if (res < 1e-4 && res >= 0) printf("x check passed! |x-xref|/|xref| = %8.2e\n", res);
    else printf(" x check _NOT_ passed! |x-xref|/|xref| = %8.2e\n", res);
    return 0;
}
