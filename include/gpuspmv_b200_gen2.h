/*
 * gpuspmv_b200_gen2.h -- drop-in for the reference's second API generation,
 * gpuSpmv_header.h (the one its gpuSpmv_main.cu includes).
 *
 * That generation reuses names of the first (matrixReading, getFormatDataAXT, ...) with
 * other struct layouts, so the library exports it under gs2_* symbols; this header declares
 * the second generation's structs under their own names and maps every name of that API
 * onto the gs2_* symbols with macros.  A program written against gpuSpmv_header.h includes
 * this header instead (or gpuspmv_b200.h with GS_API_GEN2 defined) and links
 * libgpuspmv_b200.  Define GS2_NO_ALIASES to get only the gs2_* names (the library itself
 * does, since it also defines the first generation).
 *
 * Behaviour: the same as the first generation's drop-in (GPU converters filling the same
 * host arrays, timed sm_100a kernels, errors reported instead of exit()), with this
 * generation's arrays and names:
 *   - mode "NOC" is the first generation's "UNC" (identical layouts, gpuSpmv_header.h:
 *     1120-1191); "COM" exists for tileH = 1 only, with a header word at every tile
 *     boundary (gpuSpmv_header.h:1193-1227); for COM with tileH > 1 the reference fills no
 *     array (gpuSpmv_header.h:1289-1301) and neither does this library;
 *   - con has nrows entries for every mode (gpuSpmv_header.h:1086-1115);
 *   - AXC has no hbs (HBRICK_SIZE = 32) and no mapx.
 */
#ifndef GPUSPMV_B200_GEN2_H
#define GPUSPMV_B200_GEN2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef GS_UIN_DEFINED
#define GS_UIN_DEFINED
typedef unsigned int UIN;
typedef double FPT;
#endif

/* gpuSpmv_header.h:252 */
typedef struct { UIN nrows; UIN nnz; UIN rmin; FPT rave; UIN rmax; FPT rsd; UIN bw; FPT *val;
                 UIN *row; UIN *col; UIN *rl; } gs2_matCSR;
/* gpuSpmv_header.h:375 */
typedef struct { char name[18]; double mfp; double beta; double ct; } gs2_formatData;
/* gpuSpmv_header.h:440 */
typedef struct { double aErr; double rErr; UIN pos; } gs2_err;
/* gpuSpmv_header.h:469 */
typedef struct { char name[24]; double et; double flops; gs2_err sErr; } gs2_res;
/* gpuSpmv_header.h:675 */
typedef struct { UIN nrows; UIN nnz; UIN lenAX; UIN lenBRP; FPT *ax; UIN *brp; } gs2_matAXC;
/* gpuSpmv_header.h:865 */
typedef struct { UIN nrows; UIN nnz; UIN chunkNum; UIN lenVC; UIN *permi; UIN *nmc; UIN *chp;
                 FPT *val; UIN *col; } gs2_matK1;
/* gpuSpmv_header.h:1082 */
typedef struct { UIN nrows; UIN nnz; char mode[8]; UIN tileHW; UIN tileH; UIN logTH;
                 UIN tileN; UIN lenAX; UIN lenSEC; UIN lenCON; UIN log; FPT *ax; UIN *sec;
                 UIN *con; } gs2_matAXT;

/* gpuSpmv_header.h:256, 322 (the .sta file is named after the path up to its first '.') */
gs2_matCSR gs2_matrixReading(const char *matFileName);
void gs2_printMatrixStats(const char *matFileName, gs2_matCSR *matCSR);
/* gpuSpmv_header.h:379, 398, 414, 444 */
gs2_formatData gs2_getFormatDataCSR(const gs2_matCSR matCSR);
void gs2_initVec(const UIN len, FPT *vec);
void gs2_cf_CSR(const gs2_matCSR matCSR, const FPT *vec, FPT *res);
void gs2_getErrors(const UIN len, const FPT *ar, const FPT *ac, gs2_err *sErr);
/* gpuSpmv_header.h:473, 516, 597 */
gs2_res gs2_test_cf_CSR(const gs2_matCSR matCSR, const FPT *vec, const FPT *ref);
gs2_res gs2_test_gk_CSR(const UIN cudaBlockSize, const gs2_matCSR matCSR, const FPT *vec,
                        const FPT *ref);
gs2_res gs2_test_gcu_CSR(const gs2_matCSR matCSR, const FPT *vec, const FPT *ref);
/* gpuSpmv_header.h:722, 803 */
gs2_formatData gs2_getFormatDataAXC(const UIN ompNumThreads, const gs2_matCSR matCSR,
                                    const FPT *vec, gs2_matAXC *matAXC);
gs2_res gs2_test_gk_AXC(const UIN cudaBlockSize, const gs2_matAXC matAXC, const FPT *ref);
/* gpuSpmv_header.h:934, 1021 */
gs2_formatData gs2_getFormatDataK1(const UIN cudaBlockSize, const gs2_matCSR matCSR,
                                   const FPT *vec, gs2_matK1 *matK1);
gs2_res gs2_test_gk_K1(const UIN cudaBlockSize, const gs2_matK1 matK1, const FPT *vec,
                       const FPT *ref);
/* gpuSpmv_header.h:1231, 1376, 1464, 1621 */
gs2_formatData gs2_getFormatDataAXT(const UIN ompNT, const UIN bs, const UIN thw, const UIN th,
                                    const char *mode, const gs2_matCSR matCSR, const FPT *vec,
                                    gs2_matAXT *matAXT);
gs2_res gs2_test_gk_AXT_NOC_H1(const UIN cudaBlockSize, const gs2_matAXT matAXT,
                               const FPT *ref);
gs2_res gs2_test_gk_AXT_NOC(const UIN cudaBlockSize, const gs2_matAXT matAXT, const FPT *ref);
gs2_res gs2_test_gk_AXT_COM_H1(const UIN cudaBlockSize, const gs2_matAXT matAXT,
                               const FPT *ref);

#ifdef __cplusplus
}
#endif

#ifndef GS2_NO_ALIASES
typedef gs2_matCSR str_matCSR;
typedef gs2_formatData str_formatData;
typedef gs2_err str_err;
typedef gs2_res str_res;
typedef gs2_matAXC str_matAXC;
typedef gs2_matK1 str_matK1;
typedef gs2_matAXT str_matAXT;
#define matrixReading gs2_matrixReading
#define printMatrixStats gs2_printMatrixStats
#define getFormatDataCSR gs2_getFormatDataCSR
#define initVec gs2_initVec
#define cf_CSR gs2_cf_CSR
#define getErrors gs2_getErrors
#define test_cf_CSR gs2_test_cf_CSR
#define test_gk_CSR gs2_test_gk_CSR
#define test_gcu_CSR gs2_test_gcu_CSR
#define getFormatDataAXC gs2_getFormatDataAXC
#define test_gk_AXC gs2_test_gk_AXC
#define getFormatDataK1 gs2_getFormatDataK1
#define test_gk_K1 gs2_test_gk_K1
#define getFormatDataAXT gs2_getFormatDataAXT
#define test_gk_AXT_NOC_H1 gs2_test_gk_AXT_NOC_H1
#define test_gk_AXT_NOC gs2_test_gk_AXT_NOC
#define test_gk_AXT_COM_H1 gs2_test_gk_AXT_COM_H1
#endif

#endif /* GPUSPMV_B200_GEN2_H */
