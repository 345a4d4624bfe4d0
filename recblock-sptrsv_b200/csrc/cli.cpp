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
// sum|x - x_ref| / sum|x_ref| < 1e-4 (main.cu:296-317).
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
#include <string>
#include <vector>

#include "rbs.h"

namespace {

int usage() {
    fprintf(stderr, "usage: sptrsv -d <device> -rhs <k> -lv <levels|-1> -forward|-backward -mtx <file.mtx>\n");
    return 2;
}

struct Csr {
    int m = 0, n = 0;
    std::vector<int> rp, ci;
    std::vector<double> va;
};

// Matrix Market coordinate reader with the expansion rules of
// mmio_highlevel.h:137-296: 1-based -> 0-based, symmetric/Hermitian files
// mirrored (diagonal once), columns kept in file order inside a row.
bool read_mtx(const char *path, Csr &A, std::string &err) {
    FILE *f = fopen(path, "r");
    if (!f) {
        err = std::string("cannot open ") + path;
        return false;
    }
    char line[4096];
    if (!fgets(line, sizeof line, f) || strncmp(line, "%%MatrixMarket", 14) != 0) {
        err = "missing %%MatrixMarket banner";
        fclose(f);
        return false;
    }
    char obj[64] = {0}, fmt[64] = {0}, field[64] = {0}, sym[64] = {0};
    sscanf(line + 14, "%63s %63s %63s %63s", obj, fmt, field, sym);
    for (char *p : {obj, fmt, field, sym})
        for (; *p; ++p) *p = (char)tolower(*p);
    if (strcmp(fmt, "coordinate") != 0) {
        err = "only coordinate Matrix Market files are supported";
        fclose(f);
        return false;
    }
    bool pattern = !strcmp(field, "pattern"), complex_ = !strcmp(field, "complex");
    bool symmetric = !strcmp(sym, "symmetric") || !strcmp(sym, "hermitian");
    long long nz = 0;
    int m = 0, n = 0;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '%') continue;
        if (sscanf(line, "%d %d %lld", &m, &n, &nz) == 3) break;
    }
    std::vector<int> I, J;
    std::vector<double> V;
    I.reserve(nz);
    J.reserve(nz);
    V.reserve(nz);
    for (long long k = 0; k < nz; ++k) {
        int i, j;
        double v = 1.0, im = 0;
        if (pattern) {
            if (fscanf(f, "%d %d", &i, &j) != 2) break;
        } else if (complex_) {
            if (fscanf(f, "%d %d %lg %lg", &i, &j, &v, &im) != 4) break;
        } else {
            if (fscanf(f, "%d %d %lg", &i, &j, &v) != 3) break;
        }
        I.push_back(i - 1);
        J.push_back(j - 1);
        V.push_back(v);
    }
    fclose(f);
    if ((long long)I.size() != nz) {
        err = "truncated Matrix Market file";
        return false;
    }
    A.m = m;
    A.n = n;
    std::vector<int> cnt((size_t)m + 1, 0);
    for (size_t k = 0; k < I.size(); ++k) {
        if (I[k] < 0 || I[k] >= m || J[k] < 0 || J[k] >= n) {
            err = "entry out of range";
            return false;
        }
        cnt[I[k]]++;
        if (symmetric && I[k] != J[k]) cnt[J[k]]++;
    }
    A.rp.assign((size_t)m + 1, 0);
    for (int i = 0; i < m; ++i) A.rp[i + 1] = A.rp[i] + cnt[i];
    A.ci.resize(A.rp[m]);
    A.va.resize(A.rp[m]);
    std::vector<int> fill(A.rp.begin(), A.rp.end() - 1);
    for (size_t k = 0; k < I.size(); ++k) {
        int d = fill[I[k]]++;
        A.ci[d] = J[k];
        A.va[d] = V[k];
        if (symmetric && I[k] != J[k]) {
            d = fill[J[k]]++;
            A.ci[d] = I[k];
            A.va[d] = V[k];
        }
    }
    return true;
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

    Csr A;
    std::string err;
    if (!read_mtx(filename, A, err)) {
        fprintf(stderr, "sptrsv: %s\n", err.c_str());
        return 1;
    }
    printf("input matrix A: ( %i, %i ) nnz = %i\n", A.m, A.n, A.rp[A.m]);
    if (A.m != A.n) {
        printf("we need square matrix. Exit!\n");
        return 1;
    }
    const int m = A.m, n = A.n;
    // main.cu:150-198: strict triangle of A's pattern, random values, unit diagonal
    std::vector<int> trp((size_t)m + 1, 0), tci;
    std::vector<double> tva;
    tci.reserve(A.rp[m] + m);
    tva.reserve(A.rp[m] + m);
    for (int i = 0; i < m; ++i) {
        if (substitution == RBS_BACKWARD) {
            tci.push_back(i);
            tva.push_back(1.0);
        }
        for (int j = A.rp[i]; j < A.rp[i + 1]; ++j) {
            int c = A.ci[j];
            if (substitution == RBS_FORWARD ? c < i : c > i) {
                tci.push_back(c);
                tva.push_back(rand() % 10 + 1);
            }
        }
        if (substitution == RBS_FORWARD) {
            tci.push_back(i);
            tva.push_back(1.0);
        }
        trp[i + 1] = (int)tci.size();
    }
    const int nnz = trp[m];
    const int k = rhs > 0 ? rhs : 1;
    // main.cu:211-229
    std::vector<double> x_ref((size_t)n * k), b((size_t)m * k, 0.0), x((size_t)n * k, 0.0);
    for (auto &v : x_ref) v = rand() % 10 + 1;
    for (int r = 0; r < k; ++r)
        for (int i = 0; i < m; ++i)
            for (int j = trp[i]; j < trp[i + 1]; ++j) b[(size_t)r * m + i] += tva[j] * x_ref[(size_t)r * n + tci[j]];
    // main.cu:231-238 CSR -> CSC (stable)
    std::vector<int> ccp((size_t)n + 1, 0), cri(nnz);
    std::vector<double> cva(nnz);
    for (int j = 0; j < nnz; ++j) ccp[tci[j] + 1]++;
    for (int c = 0; c < n; ++c) ccp[c + 1] += ccp[c];
    {
        std::vector<int> fill(ccp.begin(), ccp.end() - 1);
        for (int i = 0; i < m; ++i)
            for (int j = trp[i]; j < trp[i + 1]; ++j) {
                int d = fill[tci[j]]++;
                cri[d] = i;
                cva[d] = tva[j];
            }
    }
    if (lv == -1) lv = rbs_auto_lv(m, device_id);
    while (lv > 0 && (1 << lv) > m) --lv;
    printf("lv = %i\n", lv);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) == cudaSuccess && device_id >= 0 && device_id < ndev) cudaSetDevice(device_id);

    int *d_cp, *d_ri;
    double *d_va, *d_x, *d_b;
    cudaMalloc(&d_cp, sizeof(int) * (n + 1));
    cudaMalloc(&d_ri, sizeof(int) * nnz);
    cudaMalloc(&d_va, sizeof(double) * nnz);
    cudaMalloc(&d_x, sizeof(double) * (size_t)n * k);
    cudaMalloc(&d_b, sizeof(double) * (size_t)m * k);
    cudaMemcpy(d_cp, ccp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(d_ri, cri.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice);
    cudaMemcpy(d_va, cva.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice);
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
    cudaFree(d_cp);
    cudaFree(d_ri);
    cudaFree(d_va);
    cudaFree(d_x);
    cudaFree(d_b);
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
