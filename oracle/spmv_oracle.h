/*
 * spmv_oracle.h -- ORACLE TEST INFRASTRUCTURE (the CPU restatement, "port").
 *
 * A plain-C restatement of the reference's hot-path algorithms (cudaSpmv.cu): the CPU CSR
 * SpMV, row statistics, and the CSR -> K1 / AXC / AXT converters, plus CPU emulations of
 * what each format's SpMV computes.  Only tests/, the smoke check and the bench's
 * CPU-baseline leg use it, and only as the checker; the product never links it.
 *
 * Converter outputs are produced in two forms:
 *   - the reference layout with x baked in ("ax": per tile row, thw values then thw x[col]),
 *     bit-for-bit what getFormatDataAXC / getFormatDataAXT write;
 *   - the engine's native streams: slot s of a tile layout holds value nval[s] and column
 *     ncol[s], where slot s corresponds to ax[(s/w)*2w + s%w] (value half) and
 *     ax[(s/w)*2w + w + s%w] (x half), w = tileHW (AXT) or hbs (AXC).
 *     With x[i] = i (the reference's init_vec) the x half equals (double)ncol exactly.
 */
#ifndef GS_SPMV_ORACLE_H
#define GS_SPMV_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint32_t u32;

/* cudaSpmv.cu:451-466 (ncsr) / spmv_header.h:409-425 (cpuSpmvCSR): sequential row sums. */
void orc_csr_spmv(u32 n, const u32 *row, const u32 *col, const double *val, const double *x,
                  double *y);
/* Same product with long-double accumulation plus the per-row bound sum |a_ij||x_j|. */
void orc_csr_spmv_truth(u32 n, const u32 *row, const u32 *col, const double *val,
                        const double *x, double *y_true, double *abs_ax);
/* Multi-RHS CSR product, X is ncols x k row-major, Y is n x k row-major (float64). */
void orc_csr_spmm(u32 n, u32 k, const u32 *row, const u32 *col, const double *val,
                  const double *X, double *Y);

/* cudaSpmv.cu:332-358 (printMatrixStats without the file): rl, rmin, rave, rmax, rsd, bw. */
void orc_row_stats(u32 n, const u32 *row, const u32 *col, u32 *rl, double *out5);

/* cudaSpmv.cu:474-495 (get_errors). */
void orc_get_errors(u32 n, const double *ar, const double *ac, double *aErr, double *rErr,
                    u32 *pos);

/* ---------------- K1 (cudaSpmv.cu:708-867) ---------------- */
u32 orc_k1_chunknum(u32 n);
/* Stable descending sort of rows by length (qsort + orderFunction, cudaSpmv.cu:716-737). */
void orc_k1_perm(u32 n, const u32 *rl, u32 *permi);
/* nmc / chp (cudaSpmv.cu:741-754); returns lenVC. */
u32 orc_k1_nmc_chp(u32 n, const u32 *rl, const u32 *permi, u32 *nmc, u32 *chp);
/* column-major scatter (cudaSpmv.cu:758-778); kval/kcol must be zeroed by the caller. */
void orc_k1_fill(u32 n, const u32 *row, const u32 *col, const double *val, const u32 *permi,
                 const u32 *chp, double *kval, u32 *kcol);
/* gk1 semantics (cudaSpmv.cu:851-867), reading every stored slot of each sorted row. */
void orc_k1_spmv(u32 n, const u32 *permi, const u32 *nmc, const u32 *chp, const double *kval,
                 const u32 *kcol, const double *x, double *y);

/* ---------------- AXC (cudaSpmv.cu:933-1096) ---------------- */
/* brp prefix (cudaSpmv.cu:937-948); returns lenAX. */
u32 orc_axc_brp(u32 n, u32 hbs, const u32 *rl, u32 *brp);
/* ax (cudaSpmv.cu:952-979, may be NULL), native streams (may be NULL), mapx
 * (cudaSpmv.cu:983-999, may be NULL).  Outputs must be zeroed by the caller. */
void orc_axc_fill(u32 n, u32 hbs, const u32 *row, const u32 *col, const double *val,
                  const double *x, const u32 *brp, double *ax, double *nval, u32 *ncol,
                  u32 *mapx);

/* ---------------- AXT (cudaSpmv.cu:1154-1566) ---------------- */
typedef struct {
    u32 tileN, lenAX, lenSEC, lenCON, log, logTH;
} orc_axt_dims;

/* Length pass + con (cudaSpmv.cu:1158-1235, 1401-1405, 1504-1536).  mode 0 = UNC, 1 = COM.
 * con must hold n+1 entries (zeroed).  Returns 0, or -1 for an invalid parameter set. */
int orc_axt_dims_con(u32 n, const u32 *rl, u32 thw, u32 th, u32 bs, int mode, u32 *con,
                     orc_axt_dims *d);
/* Fill pass (cudaSpmv.cu:1239-1387): ax (baked with x; may be NULL), native streams
 * (may be NULL) and sec.  Outputs must be zeroed by the caller. */
void orc_axt_fill(u32 n, const u32 *row, const u32 *col, const double *val, const double *x,
                  u32 thw, u32 th, u32 bs, int mode, const u32 *con, const orc_axt_dims *d,
                  double *ax, double *nval, u32 *ncol, u32 *sec);

/* What the AXT kernels compute (cudaSpmv.cu:1570-2209), restated on the native streams
 * with the row of every slot recovered from the format's own metadata (sec / headers);
 * y is overwritten.  Returns 0 or -1 on malformed metadata. */
int orc_axt_spmv(u32 n, u32 thw, u32 th, u32 bs, int mode, const orc_axt_dims *d,
                 const u32 *sec, const double *nval, const u32 *ncol, const double *x,
                 double *y);
/* Same on the baked layout (x taken from ax). */
int orc_axt_spmv_baked(u32 n, u32 thw, u32 th, u32 bs, int mode, const orc_axt_dims *d,
                       const u32 *sec, const double *ax, double *y);

#ifdef __cplusplus
}
#endif
#endif
