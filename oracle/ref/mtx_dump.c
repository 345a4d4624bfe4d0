/* mtx_dump.c -- golden-vector harness around the reference's OWN Matrix
 * Market reader.  Built by oracle/Makefile against the reference sources
 * where they lie (-I <reference>/recblock-sptrsv); the binary goes to
 * oracle/_ref/.  Calls mmio_info and mmio_data (mmio_highlevel.h:7-296)
 * exactly as main.cu:120-141 does and writes to stdout:
 *   int32 m, n, nnz, isSymmetric; int32 rowptr[m+1]; int32 colidx[nnz];
 *   f64 val[nnz].
 * With --time first, prints instead the wall milliseconds of the two calls
 * (the reference's CPU reading path, timed as the baseline). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mmio_highlevel.h"

static double now_ms(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1e3 + t.tv_nsec * 1e-6;
}

int main(int argc, char **argv) {
    const int timing = argc == 3 && !strcmp(argv[1], "--time");
    if (argc != 2 && !timing) {
        fprintf(stderr, "usage: mtx_dump [--time] <file.mtx>\n");
        return 2;
    }
    char *path = argv[argc - 1];
    int m = 0, n = 0, nnz = 0, sym = 0;
    const double t0 = now_ms();
    if (mmio_info(&m, &n, &nnz, &sym, path) != 0) return 3;
    int *rp = (int *)malloc(sizeof(int) * (size_t)(m + 1));
    int *ci = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    double *va = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    if (mmio_data(rp, ci, va, path) != 0) return 4;
    if (timing) {
        printf("%.3f\n", now_ms() - t0);
        return 0;
    }
    int hdr[4] = {m, n, nnz, sym};
    fwrite(hdr, 4, 4, stdout);
    fwrite(rp, 4, (size_t)(m + 1), stdout);
    fwrite(ci, 4, (size_t)nnz, stdout);
    fwrite(va, 8, (size_t)nnz, stdout);
    free(rp);
    free(ci);
    free(va);
    return 0;
}
