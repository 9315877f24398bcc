/*
 * ref_shim_cusparse.h -- ORACLE TEST INFRASTRUCTURE (never shipped, never measured).
 *
 * The reference's cudaSpmv.cu (test_gcucsr, cudaSpmv.cu:629-704) calls the legacy
 * cuSPARSE entry point cusparseCsrmvEx with cusparseAlgMode_t / CUSPARSE_ALG1
 * (cudaSpmv.cu:635,663,675).  CUDA 12 removed those names, so the reference does not
 * compile unchanged against CUDA 12.9.  This header declares the removed names so that
 * the reference translation unit compiles; the stand-ins only report
 * CUSPARSE_STATUS_NOT_SUPPORTED.  The oracle never calls test_gcucsr: it only uses the
 * reference's host converters (getFormatData*) and CPU SpMV (ncsr).
 */
#ifndef GS_ORACLE_REF_SHIM_CUSPARSE_H
#define GS_ORACLE_REF_SHIM_CUSPARSE_H

#include <cusparse.h>

typedef enum { CUSPARSE_ALG0 = 0, CUSPARSE_ALG1 = 1 } cusparseAlgMode_t;

static inline cusparseStatus_t cusparseCsrmvEx_bufferSize(
    cusparseHandle_t, cusparseAlgMode_t, cusparseOperation_t, int, int, int,
    const void *, cudaDataType, const cusparseMatDescr_t, const void *, cudaDataType,
    const int *, const int *, const void *, cudaDataType, const void *, cudaDataType,
    void *, cudaDataType, cudaDataType, size_t *bufferSize)
{
    if (bufferSize) *bufferSize = 0;
    return CUSPARSE_STATUS_NOT_SUPPORTED;
}

static inline cusparseStatus_t cusparseCsrmvEx(
    cusparseHandle_t, cusparseAlgMode_t, cusparseOperation_t, int, int, int,
    const void *, cudaDataType, const cusparseMatDescr_t, const void *, cudaDataType,
    const int *, const int *, const void *, cudaDataType, const void *, cudaDataType,
    void *, cudaDataType, cudaDataType, void *)
{
    return CUSPARSE_STATUS_NOT_SUPPORTED;
}

#endif
