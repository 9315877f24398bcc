/*
 * ref_wrap.cu -- ORACLE TEST INFRASTRUCTURE.  Only tests/, the smoke check and the
 * bench's CPU-baseline leg load the library built from this file; the product never does.
 *
 * This translation unit compiles the reference's canonical source, cudaSpmv.cu, UNCHANGED
 * (the file is #included from where it lies; the build recipe passes its path as
 * REF_CUDASPMV), renames its main() to ref_main(), and exposes C entry points around the
 * reference's own host functions so that Python (ctypes) can call them:
 *
 *   ref_ncsr           -> ncsr               (cudaSpmv.cu:451-466, OpenMP CPU CSR SpMV)
 *   ref_init_vec       -> init_vec           (cudaSpmv.cu:440-447, x[i] = i)
 *   ref_get_errors     -> get_errors         (cudaSpmv.cu:474-495)
 *   ref_stats          -> printMatrixStats   (cudaSpmv.cu:332-381, fills rl[], writes .sta)
 *   ref_k1_*           -> getFormatDataK1    (cudaSpmv.cu:782-846)
 *   ref_axc_*          -> getFormatDataAXC   (cudaSpmv.cu:1004-1062)
 *   ref_axt_*          -> getFormatDataAXT   (cudaSpmv.cu:1391-1566)
 *   ref_gpu_*          -> test_gcsr, test_gk1, test_gaxc, test_gaxtuh, test_gaxtuh1hw16w,
 *                         test_gaxtch1, test_gaxtch (the reference's own GPU products,
 *                         cudaSpmv.cu:547-2285)
 *   ref_struct_layout  -> sizeof / offsetof of the reference's host-API structs
 *
 * No reference code is copied here: the wrappers only marshal arguments into the
 * reference's own structs (str_matCSR, str_matK1, str_matAXC, str_matAXT) and back out.
 */
#include <stdint.h>
#define main ref_main
#include REF_CUDASPMV
#undef main

namespace {

struct RefCSR {
    str_matCSR m;
};

/* Build a str_matCSR view of caller arrays; rl[] is the row length as the reference
 * defines it (cudaSpmv.cu:339: rl = row[i+1] - row[i]). */
static str_matCSR make_csr(UIN nrows, UIN nnz, const FPT *val, const UIN *col,
                           const UIN *row, UIN *rl)
{
    str_matCSR m;
    memset(&m, 0, sizeof(m));
    strcpy(m.name, "oracle");
    m.nrows = nrows;
    m.nnz = nnz;
    m.val = (FPT *)val;
    m.col = (UIN *)col;
    m.row = (UIN *)row;
    m.rl = rl;
    for (UIN i = 0; i < nrows; i++) rl[i] = row[i + 1] - row[i];
    return m;
}

}  // namespace

extern "C" {

void ref_ncsr(UIN ompNT, UIN nrows, UIN nnz, const FPT *val, const UIN *col,
              const UIN *row, const FPT *vec, FPT *res)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl);
    ncsr(ompNT, m, vec, res);
    free(rl);
}

void ref_init_vec(UIN ompNT, UIN len, FPT *vec) { init_vec(ompNT, len, vec); }

void ref_get_errors(UIN len, const FPT *ar, const FPT *ac, double *aErr, double *rErr,
                    UIN *pos)
{
    str_err e;
    get_errors(len, ar, ac, &e);
    *aErr = e.aErr;
    *rErr = e.rErr;
    *pos = e.pos;
}

/* printMatrixStats writes "<path up to the first '.'>.sta"; callers pass a scratch path. */
void ref_stats(const char *path, UIN nrows, UIN nnz, const FPT *val, const UIN *col,
               const UIN *row, UIN *rl_out, double *out5)
{
    str_matCSR m;
    memset(&m, 0, sizeof(m));
    m.nrows = nrows;
    m.nnz = nnz;
    m.val = (FPT *)val;
    m.col = (UIN *)col;
    m.row = (UIN *)row;
    m.rl = rl_out;
    printMatrixStats(path, &m);
    out5[0] = m.rmin;
    out5[1] = m.rave;
    out5[2] = m.rmax;
    out5[3] = m.rsd;
    out5[4] = m.bw;
}

/* ---------------- K1 ---------------- */
void *ref_k1(UIN nrows, UIN nnz, const FPT *val, const UIN *col, const UIN *row,
             const FPT *vec, double *fd3)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl);
    str_matK1 *k = (str_matK1 *)calloc(1, sizeof(str_matK1));
    str_formatData fd = getFormatDataK1(CHUNK_SIZE, m, vec, k);
    fd3[0] = fd.mfp;
    fd3[1] = fd.beta;
    fd3[2] = fd.ct;
    free(rl);
    return k;
}
void ref_k1_dims(void *h, UIN *d4)
{
    str_matK1 *k = (str_matK1 *)h;
    d4[0] = k->nrows; d4[1] = k->nnz; d4[2] = k->chunkNum; d4[3] = k->lenVC;
}
void ref_k1_copy(void *h, UIN *permi, UIN *nmc, UIN *chp, FPT *val, UIN *col)
{
    str_matK1 *k = (str_matK1 *)h;
    memcpy(permi, k->permi, (size_t)(k->chunkNum + 1) * CHUNK_SIZE * sizeof(UIN));
    memcpy(nmc, k->nmc, (size_t)k->chunkNum * sizeof(UIN));
    memcpy(chp, k->chp, (size_t)k->chunkNum * sizeof(UIN));
    memcpy(val, k->val, (size_t)k->lenVC * sizeof(FPT));
    memcpy(col, k->col, (size_t)k->lenVC * sizeof(UIN));
}
void ref_k1_free(void *h)
{
    str_matK1 *k = (str_matK1 *)h;
    free(k->permi); free(k->nmc); free(k->chp); free(k->val); free(k->col); free(k);
}

/* ---------------- AXC ---------------- */
void *ref_axc(UIN ompNT, UIN hbs, UIN nrows, UIN nnz, const FPT *val, const UIN *col,
              const UIN *row, const FPT *vec, double *fd3)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl);
    str_matAXC *a = (str_matAXC *)calloc(1, sizeof(str_matAXC));
    str_formatData fd = getFormatDataAXC(ompNT, hbs, m, vec, a);
    fd3[0] = fd.mfp;
    fd3[1] = fd.beta;
    fd3[2] = fd.ct;
    free(rl);
    return a;
}
void ref_axc_dims(void *h, UIN *d6)
{
    str_matAXC *a = (str_matAXC *)h;
    d6[0] = a->nrows; d6[1] = a->nnz; d6[2] = a->hbs; d6[3] = a->lenAX; d6[4] = a->lenBRP;
    d6[5] = a->lenMAPX;
}
void ref_axc_copy(void *h, FPT *ax, UIN *brp, UIN *mapx)
{
    str_matAXC *a = (str_matAXC *)h;
    memcpy(ax, a->ax, (size_t)a->lenAX * sizeof(FPT));
    memcpy(brp, a->brp, (size_t)a->lenBRP * sizeof(UIN));
    memcpy(mapx, a->mapx, (size_t)a->lenMAPX * sizeof(UIN));
}
void ref_axc_free(void *h)
{
    str_matAXC *a = (str_matAXC *)h;
    free(a->ax); free(a->brp); free(a->mapx); free(a);
}

/* ---------------- AXT ---------------- */
void *ref_axt(UIN ompNT, UIN bs, UIN thw, UIN th, const char *mode, UIN nrows, UIN nnz,
              const FPT *val, const UIN *col, const UIN *row, const FPT *vec, double *fd3,
              char *name48)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl);
    str_matAXT *a = (str_matAXT *)calloc(1, sizeof(str_matAXT));
    str_formatData fd = getFormatDataAXT(ompNT, bs, thw, th, mode, m, vec, a);
    fd3[0] = fd.mfp;
    fd3[1] = fd.beta;
    fd3[2] = fd.ct;
    if (name48) memcpy(name48, fd.name, 48);
    free(rl);
    return a;
}
void ref_axt_dims(void *h, UIN *d11)
{
    str_matAXT *a = (str_matAXT *)h;
    d11[0] = a->nrows; d11[1] = a->nnz; d11[2] = a->tileHW; d11[3] = a->tileH;
    d11[4] = a->logTH; d11[5] = a->tileN; d11[6] = a->lenAX; d11[7] = a->lenSEC;
    d11[8] = a->lenCON; d11[9] = a->log; d11[10] = a->bs;
}
void ref_axt_copy(void *h, FPT *ax, UIN *sec, UIN *con)
{
    str_matAXT *a = (str_matAXT *)h;
    memcpy(ax, a->ax, (size_t)a->lenAX * sizeof(FPT));
    memcpy(sec, a->sec, (size_t)a->lenSEC * sizeof(UIN));
    memcpy(con, a->con, (size_t)(a->lenCON + 1) * sizeof(UIN));
}
void ref_axt_free(void *h)
{
    str_matAXT *a = (str_matAXT *)h;
    free(a->ax); free(a->sec); free(a->con); free(a);
}

/* ---------------- the reference's own GPU products, compiled for sm_100a ----------------
 * Each runs the reference's test function (device buffers, one launch timed by its cudaEvents
 * (NUM_ITE = 1), result copied back, buffers freed) and returns its str_res: et (seconds)
 * and the get_errors summary against `ref` in err3 = {aErr, rErr, pos}.  Only matrices
 * without all-empty 32-row chunks may go to gk1: its first load of a chunk
 * (cudaSpmv.cu:861) is unconditional. */
static double res_out(const str_res &r, double *err3)
{
    err3[0] = r.sErr.aErr;
    err3[1] = r.sErr.rErr;
    err3[2] = (double)r.sErr.pos;
    return r.et;
}
double ref_gpu_csr(UIN cbs, UIN nrows, UIN nnz, const FPT *val, const UIN *col,
                   const UIN *row, const FPT *vec, const FPT *ref, double *err3)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl);
    const str_res r = test_gcsr(cbs, m, vec, ref);             /* cudaSpmv.cu:547 */
    free(rl);
    return res_out(r, err3);
}
double ref_gpu_k1(void *h, UIN cbs, const FPT *vec, const FPT *ref, double *err3)
{
    return res_out(test_gk1(cbs, *(str_matK1 *)h, vec, ref), err3);    /* cudaSpmv.cu:871 */
}
double ref_gpu_axc(void *h, UIN cbs, const FPT *ref, double *err3)
{
    return res_out(test_gaxc(cbs, *(str_matAXC *)h, ref), err3);       /* cudaSpmv.cu:1100 */
}
/* tileH > 1, tileHW 32 */
double ref_gpu_axt_uh(void *h, UIN tpw, UIN cbs, const FPT *ref, double *err3)
{
    return res_out(test_gaxtuh(tpw, cbs, *(str_matAXT *)h, ref), err3); /* cudaSpmv.cu:1963 */
}
/* tileH 1, tileHW 16; wpw / 32 tiles per warp must be even (the kernel takes tiles in pairs) */
double ref_gpu_axt_uh1hw16(void *h, UIN wpw, UIN cbs, const FPT *ref, double *err3)
{
    return res_out(test_gaxtuh1hw16w(wpw, cbs, *(str_matAXT *)h, ref), err3); /* :1603 */
}

/* COM tileH = 1: gaxtch1 launched with cudaBlockSize equal to the layout's header block bs
 * (its segment offset o <= bs - 1 - tid indexes the block's shared array, cudaSpmv.cu:2087) */
double ref_gpu_axt_ch1(void *h, const FPT *ref, double *err3)
{
    const str_matAXT *m = (const str_matAXT *)h;
    return res_out(test_gaxtch1(m->bs, *m, ref), err3);                  /* cudaSpmv.cu:2101 */
}
/* COM tileH > 1, tileHW 32 */
double ref_gpu_axt_ch(void *h, UIN cbs, const FPT *ref, double *err3)
{
    return res_out(test_gaxtch(cbs, *(str_matAXT *)h, ref), err3);        /* cudaSpmv.cu:2213 */
}

/* sizeof and the offset of every field of the reference's host-API structs, in the order
 * of their declarations (cudaSpmv.cu:261, 385, 470, 499, 712, 933, 1154), as "name value"
 * lines; returns the number of characters written (0 if cap is too small). */
#define REF_SZ(T) n += snprintf(buf + n, cap > n ? cap - n : 0, #T " %zu\n", sizeof(T))
#define REF_OF(T, f) n += snprintf(buf + n, cap > n ? cap - n : 0, #T "." #f " %zu\n", offsetof(T, f))
size_t ref_struct_layout(char *buf, size_t cap)
{
    size_t n = 0;
    REF_SZ(str_matCSR);
    REF_OF(str_matCSR, name); REF_OF(str_matCSR, nrows); REF_OF(str_matCSR, nnz);
    REF_OF(str_matCSR, rmin); REF_OF(str_matCSR, rave); REF_OF(str_matCSR, rmax);
    REF_OF(str_matCSR, rsd); REF_OF(str_matCSR, bw); REF_OF(str_matCSR, val);
    REF_OF(str_matCSR, row); REF_OF(str_matCSR, rowStart); REF_OF(str_matCSR, rowEnd);
    REF_OF(str_matCSR, col); REF_OF(str_matCSR, rl);
    REF_SZ(str_formatData);
    REF_OF(str_formatData, name); REF_OF(str_formatData, mfp); REF_OF(str_formatData, beta);
    REF_OF(str_formatData, ct);
    REF_SZ(str_err);
    REF_OF(str_err, aErr); REF_OF(str_err, rErr); REF_OF(str_err, pos);
    REF_SZ(str_res);
    REF_OF(str_res, name); REF_OF(str_res, et); REF_OF(str_res, ot); REF_OF(str_res, flops);
    REF_OF(str_res, sErr);
    REF_SZ(str_matK1);
    REF_OF(str_matK1, nrows); REF_OF(str_matK1, nnz); REF_OF(str_matK1, chunkNum);
    REF_OF(str_matK1, lenVC); REF_OF(str_matK1, permi); REF_OF(str_matK1, nmc);
    REF_OF(str_matK1, chp); REF_OF(str_matK1, val); REF_OF(str_matK1, col);
    REF_SZ(str_matAXC);
    REF_OF(str_matAXC, nrows); REF_OF(str_matAXC, nnz); REF_OF(str_matAXC, hbs);
    REF_OF(str_matAXC, lenAX); REF_OF(str_matAXC, lenBRP); REF_OF(str_matAXC, lenMAPX);
    REF_OF(str_matAXC, ax); REF_OF(str_matAXC, brp); REF_OF(str_matAXC, mapx);
    REF_SZ(str_matAXT);
    REF_OF(str_matAXT, name); REF_OF(str_matAXT, nrows); REF_OF(str_matAXT, nnz);
    REF_OF(str_matAXT, mode); REF_OF(str_matAXT, tileHW); REF_OF(str_matAXT, tileH);
    REF_OF(str_matAXT, logTH); REF_OF(str_matAXT, tileN); REF_OF(str_matAXT, lenAX);
    REF_OF(str_matAXT, lenSEC); REF_OF(str_matAXT, lenCON); REF_OF(str_matAXT, log);
    REF_OF(str_matAXT, bs); REF_OF(str_matAXT, ax); REF_OF(str_matAXT, sec);
    REF_OF(str_matAXT, con);
    return n < cap ? n : 0;
}
#undef REF_SZ
#undef REF_OF

}  // extern "C"
