/*
 * gpuspmv_b200_gen0.h -- drop-in for the brick formats of the reference's first API
 * generation, spmv_header.h (the one its spmv_main.cu includes): AXCv0, AXCv1, AXBv0 and
 * AXBv1, the segmented-scan formats with bricks of HBRICK_SIZE = 16 values.
 *
 * That generation's base structs differ from the later ones (str_matCSR without name,
 * rowStart and rowEnd; a 12-character format name; str_res without ot), so the library
 * exports it under gs0_* symbols; this header declares the structs under their own names and
 * maps that API's names onto the gs0_* symbols with macros.  A program written against
 * spmv_header.h's brick formats includes this header and links libgpuspmv_b200.  Define
 * GS0_NO_ALIASES to get only the gs0_* names.
 *
 * The four formats are layouts the engine already builds (the correspondence is pinned
 * against spmv_header.h compiled unchanged, tests/test_oracle.py):
 *   AXCv0 = AXC with half-brick 16               (brp, ax;           spmv_header.h:665-760)
 *   AXCv1 = AXT UNC, tileH 1, tileHW 16          (brp = con, rwp = sec; :851-960)
 *   AXBv0 = AXT COM, tileH 1, tileHW 16, a header word every 32 positions
 *                                                (hdr0 = sec;         :1649-1727)
 *   AXBv1 = the same with a header word every cudaBlockSize positions, hdr1 padded with
 *           zeros to a multiple of 32 words     (:2299-2390)
 * The converters run on the GPU and fill the same calloc'd host arrays as the reference's
 * (x baked into ax); the entry points time the engine's sm_100a kernels for those layouts
 * (the tile kernel for AXCv0 / AXCv1, the row-stream kernel for AXBv0 / AXBv1) and score y
 * against ref with the reference's error summary.  The reference's several kernels per
 * format (gk_AXCv1_0..4, gk_AXBv0_0..3: the same product, unrolled differently) share one
 * engine kernel each; every entry point keeps its own result name.  gs_dropin_last_y
 * (gpuspmv_b200.h) returns the y of the last of them.
 *
 * Differences a caller sees: errors print and return a result named "error" instead of
 * exit(); AXBv1 takes only a cudaBlockSize that is a power of two in 32..1024 (the
 * reference's header packing needs it, spmv_header.h:2355-2364); a row 0 whose single element
 * sits at position 0 (header word 0) is summed, where the reference's AXB kernels skip
 * header words equal to 0 (spmv_header.h:1760).
 */
#ifndef GPUSPMV_B200_GEN0_H
#define GPUSPMV_B200_GEN0_H

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

/* spmv_header.h:247 */
typedef struct { UIN nrows; UIN nnz; UIN rmin; FPT rave; UIN rmax; FPT rsd; UIN bw; FPT *val;
                 UIN *row; UIN *col; UIN *rl; } gs0_matCSR;
/* spmv_header.h:370 */
typedef struct { char name[12]; double mfp; double beta; double ct; } gs0_formatData;
/* spmv_header.h:435 */
typedef struct { double aErr; double rErr; UIN pos; } gs0_err;
/* spmv_header.h:464 */
typedef struct { char name[24]; double et; double flops; gs0_err sErr; } gs0_res;
/* spmv_header.h:665 */
typedef struct { UIN nrows; UIN nnz; UIN lenAX; UIN lenBRP; FPT *ax; UIN *brp; } gs0_matAXCv0;
/* spmv_header.h:851 */
typedef struct { UIN nrows; UIN nnz; UIN lenAX; UIN lenBRP; UIN lenRWP; FPT *ax; UIN *brp;
                 UIN *rwp; } gs0_matAXCv1;
/* spmv_header.h:1649 */
typedef struct { UIN nrows; UIN nnz; UIN brickNum; UIN lenAX; UIN lenHDR; FPT *ax; UIN *hdr0; }
    gs0_matAXBv0;
/* spmv_header.h:2299 */
typedef struct { UIN nrows; UIN nnz; UIN brickNum; UIN lenAX; UIN lenHDR; UIN blockLog; FPT *ax;
                 UIN *hdr1; } gs0_matAXBv1;

/* Converters (spmv_header.h:711, 916, 1690, 2340).  rl must hold the row lengths
 * (printMatrixStats fills it in the reference's programs). */
gs0_formatData gs0_getFormatDataAXCv0(const UIN numThreads, const gs0_matCSR matCSR,
                                      const FPT *vec, gs0_matAXCv0 *matAXC);
gs0_formatData gs0_getFormatDataAXCv1(const UIN numThreads, const gs0_matCSR matCSR,
                                      const FPT *vec, gs0_matAXCv1 *matAXC);
gs0_formatData gs0_getFormatDataAXBv0(const gs0_matCSR matCSR, const FPT *vec,
                                      gs0_matAXBv0 *matAXB);
gs0_formatData gs0_getFormatDataAXBv1(const UIN cudaBlockSize, const gs0_matCSR matCSR,
                                      const FPT *vec, gs0_matAXBv1 *matAXB);

/* Entry points (spmv_header.h:794, 1023, 1121, 1252, 1408, 1590, 1775, 1905, 2060, 2240,
 * 2474): NUM_ITE timed launches (gs_set_num_ite), y scored against ref. */
gs0_res gs0_testGpuSpmvAXCv0(const UIN cudaBlockSize, const gs0_matAXCv0 matAXC, const FPT *ref);
gs0_res gs0_testGpuSpmvAXCv1_0(const UIN cudaBlockSize, const gs0_matAXCv1 matAXC,
                               const FPT *ref);
gs0_res gs0_testGpuSpmvAXCv1_1(const UIN cudaBlockSize, const gs0_matAXCv1 matAXC,
                               const FPT *ref);
gs0_res gs0_testGpuSpmvAXCv1_2(const UIN cudaBlockSize, const gs0_matAXCv1 matAXC,
                               const FPT *ref);
gs0_res gs0_testGpuSpmvAXCv1_3(const UIN cudaBlockSize, const gs0_matAXCv1 matAXC,
                               const FPT *ref);
gs0_res gs0_testGpuSpmvAXCv1_4(const UIN cudaBlockSize, const gs0_matAXCv1 matAXC,
                               const FPT *ref);
gs0_res gs0_testGpuSpmvAXBv0_0(const UIN cudaBlockSize, const gs0_matAXBv0 matAXB,
                               const FPT *ref);
gs0_res gs0_testGpuSpmvAXBv0_1(const UIN cudaBlockSize, const gs0_matAXBv0 matAXB,
                               const FPT *ref);
gs0_res gs0_testGpuSpmvAXBv0_2(const UIN cudaBlockSize, const gs0_matAXBv0 matAXB,
                               const FPT *ref);
gs0_res gs0_testGpuSpmvAXBv0_3(const UIN cudaBlockSize, const gs0_matAXBv0 matAXB,
                               const FPT *ref);
gs0_res gs0_testGpuSpmvAXBv1_0(const UIN cudaBlockSize, const gs0_matAXBv1 matAXB,
                               const FPT *ref);

#ifdef __cplusplus
}
#endif

#ifndef GS0_NO_ALIASES
typedef gs0_matCSR str_matCSR;
typedef gs0_formatData str_formatData;
typedef gs0_err str_err;
typedef gs0_res str_res;
typedef gs0_matAXCv0 str_matAXCv0;
typedef gs0_matAXCv1 str_matAXCv1;
typedef gs0_matAXBv0 str_matAXBv0;
typedef gs0_matAXBv1 str_matAXBv1;
#define getFormatDataAXCv0 gs0_getFormatDataAXCv0
#define getFormatDataAXCv1 gs0_getFormatDataAXCv1
#define getFormatDataAXBv0 gs0_getFormatDataAXBv0
#define getFormatDataAXBv1 gs0_getFormatDataAXBv1
#define testGpuSpmvAXCv0 gs0_testGpuSpmvAXCv0
#define testGpuSpmvAXCv1_0 gs0_testGpuSpmvAXCv1_0
#define testGpuSpmvAXCv1_1 gs0_testGpuSpmvAXCv1_1
#define testGpuSpmvAXCv1_2 gs0_testGpuSpmvAXCv1_2
#define testGpuSpmvAXCv1_3 gs0_testGpuSpmvAXCv1_3
#define testGpuSpmvAXCv1_4 gs0_testGpuSpmvAXCv1_4
#define testGpuSpmvAXBv0_0 gs0_testGpuSpmvAXBv0_0
#define testGpuSpmvAXBv0_1 gs0_testGpuSpmvAXBv0_1
#define testGpuSpmvAXBv0_2 gs0_testGpuSpmvAXBv0_2
#define testGpuSpmvAXBv0_3 gs0_testGpuSpmvAXBv0_3
#define testGpuSpmvAXBv1_0 gs0_testGpuSpmvAXBv1_0
#endif

#endif /* GPUSPMV_B200_GEN0_H */
