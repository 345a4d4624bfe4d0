/*
 * csrsv2_shim.h -- force-included when compiling the reference's analysis
 * headers for the golden-vector harness (oracle/ref/ref_dump.cu).
 *
 * cuSPARSE 12 removed csrsv2Info_t and the cusparse{D,S}csrsv2_* routines
 * that recblock-sptrsv's method 1 uses (utils_sptrsv_cuda.h:25,
 * recblocking_preprocess.h:572-593).  The harness only needs the integer
 * analysis, so these stand-ins accept the calls and do nothing.  No solve is
 * ever run through them.
 */
#pragma once
#include <cusparse.h>

typedef struct rbs_shim_csrsv2_info *csrsv2Info_t;

static inline cusparseStatus_t cusparseCreateCsrsv2Info(csrsv2Info_t *info) {
    *info = 0;
    return CUSPARSE_STATUS_SUCCESS;
}
static inline cusparseStatus_t cusparseDcsrsv2_bufferSize(cusparseHandle_t, cusparseOperation_t, int, int,
                                                          const cusparseMatDescr_t, double *, const int *,
                                                          const int *, csrsv2Info_t, int *size) {
    *size = 0;
    return CUSPARSE_STATUS_SUCCESS;
}
static inline cusparseStatus_t cusparseScsrsv2_bufferSize(cusparseHandle_t, cusparseOperation_t, int, int,
                                                          const cusparseMatDescr_t, float *, const int *,
                                                          const int *, csrsv2Info_t, int *size) {
    *size = 0;
    return CUSPARSE_STATUS_SUCCESS;
}
static inline cusparseStatus_t cusparseDcsrsv2_analysis(cusparseHandle_t, cusparseOperation_t, int, int,
                                                        const cusparseMatDescr_t, const double *, const int *,
                                                        const int *, csrsv2Info_t, cusparseSolvePolicy_t, void *) {
    return CUSPARSE_STATUS_SUCCESS;
}
static inline cusparseStatus_t cusparseScsrsv2_analysis(cusparseHandle_t, cusparseOperation_t, int, int,
                                                        const cusparseMatDescr_t, const float *, const int *,
                                                        const int *, csrsv2Info_t, cusparseSolvePolicy_t, void *) {
    return CUSPARSE_STATUS_SUCCESS;
}
static inline cusparseStatus_t cusparseXcsrsv2_zeroPivot(cusparseHandle_t, csrsv2Info_t, int *) {
    return CUSPARSE_STATUS_SUCCESS;
}
