/*
 * ref_wrap_gen2.cu -- ORACLE TEST INFRASTRUCTURE.  Only tests/ load the library built from
 * this file; the product never does.
 *
 * Compiles the reference's second API generation, gpuSpmv_header.h, UNCHANGED (included
 * from where it lies; the recipe passes its path as REF_GEN2_HEADER) and exposes C entry
 * points around its own host functions:
 *
 *   ref2_stats       -> printMatrixStats  (gpuSpmv_header.h:322-371)
 *   ref2_cf_csr      -> cf_CSR            (gpuSpmv_header.h:414-428)
 *   ref2_axc_*       -> getFormatDataAXC  (gpuSpmv_header.h:722-773)
 *   ref2_k1_*        -> getFormatDataK1   (gpuSpmv_header.h:934-997)
 *   ref2_axt_*       -> getFormatDataAXT  (gpuSpmv_header.h:1231-1327), modes "NOC" / "COM"
 *
 * The wrappers only marshal arguments into the reference's structs and back out.
 */
#include <stdint.h>
#include REF_GEN2_HEADER

namespace {

str_matCSR make_csr(UIN nrows, UIN nnz, const FPT *val, const UIN *col, const UIN *row,
                    UIN *rl)
{
    str_matCSR m;
    memset(&m, 0, sizeof(m));
    m.nrows = nrows;
    m.nnz = nnz;
    m.val = (FPT *)val;
    m.col = (UIN *)col;
    m.row = (UIN *)row;
    m.rl = rl;
    for (UIN i = 0; i < nrows; i++) rl[i] = row[i + 1] - row[i];
    return m;
}

str_matAXC g_axc;
str_matK1 g_k1;
str_matAXT g_axt;
str_formatData g_fd;

}  // namespace

extern "C" {

void ref2_stats(const char *path, UIN nrows, UIN nnz, const FPT *val, const UIN *col,
                const UIN *row, UIN *rl_out, double *out5)
{
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl_out);
    printMatrixStats(path, &m);
    out5[0] = m.rmin;
    out5[1] = m.rave;
    out5[2] = m.rmax;
    out5[3] = m.rsd;
    out5[4] = m.bw;
}

void ref2_cf_csr(UIN nrows, UIN nnz, const FPT *val, const UIN *col, const UIN *row,
                 const FPT *vec, FPT *res)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl);
    cf_CSR(m, vec, res);
    free(rl);
}

/* formatData of the last conversion: name (18 bytes) and mfp, beta */
void ref2_fd(char *name18, double *mfp_beta)
{
    memcpy(name18, g_fd.name, sizeof(g_fd.name));
    mfp_beta[0] = g_fd.mfp;
    mfp_beta[1] = g_fd.beta;
}

/* ---- AXC: dims = {lenAX, lenBRP} */
void ref2_axc(UIN ompNT, UIN nrows, UIN nnz, const FPT *val, const UIN *col, const UIN *row,
              const FPT *vec, UIN *dims)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl);
    memset(&g_axc, 0, sizeof(g_axc));
    g_fd = getFormatDataAXC(ompNT, m, vec, &g_axc);
    free(rl);
    dims[0] = g_axc.lenAX;
    dims[1] = g_axc.lenBRP;
}

void ref2_axc_copy(FPT *ax, UIN *brp)
{
    memcpy(ax, g_axc.ax, (size_t)g_axc.lenAX * sizeof(FPT));
    memcpy(brp, g_axc.brp, (size_t)g_axc.lenBRP * sizeof(UIN));
    free(g_axc.ax);
    free(g_axc.brp);
}

/* ---- K1: dims = {chunkNum, lenVC} */
void ref2_k1(UIN cbs, UIN nrows, UIN nnz, const FPT *val, const UIN *col, const UIN *row,
             const FPT *vec, UIN *dims)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl);
    memset(&g_k1, 0, sizeof(g_k1));
    g_fd = getFormatDataK1(cbs, m, vec, &g_k1);
    free(rl);
    dims[0] = g_k1.chunkNum;
    dims[1] = g_k1.lenVC;
}

void ref2_k1_copy(UIN *permi, UIN *nmc, UIN *chp, FPT *val, UIN *col)
{
    memcpy(permi, g_k1.permi, (size_t)g_k1.chunkNum * CHUNK_SIZE * sizeof(UIN));
    memcpy(nmc, g_k1.nmc, (size_t)g_k1.chunkNum * sizeof(UIN));
    memcpy(chp, g_k1.chp, (size_t)g_k1.chunkNum * sizeof(UIN));
    memcpy(val, g_k1.val, (size_t)g_k1.lenVC * sizeof(FPT));
    memcpy(col, g_k1.col, (size_t)g_k1.lenVC * sizeof(UIN));
    free(g_k1.permi);
    free(g_k1.nmc);
    free(g_k1.chp);
    free(g_k1.val);
    free(g_k1.col);
}

/* ---- AXT: dims = {tileN, lenAX, lenSEC, lenCON, logTH, log} */
void ref2_axt(UIN ompNT, UIN bs, UIN thw, UIN th, const char *mode, UIN nrows, UIN nnz,
              const FPT *val, const UIN *col, const UIN *row, const FPT *vec, UIN *dims)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = make_csr(nrows, nnz, val, col, row, rl);
    memset(&g_axt, 0, sizeof(g_axt));
    g_fd = getFormatDataAXT(ompNT, bs, thw, th, mode, m, vec, &g_axt);
    free(rl);
    dims[0] = g_axt.tileN;
    dims[1] = g_axt.lenAX;
    dims[2] = g_axt.lenSEC;
    dims[3] = g_axt.lenCON;
    dims[4] = g_axt.logTH;
    dims[5] = g_axt.log;
}

void ref2_axt_copy(FPT *ax, UIN *sec, UIN *con)
{
    memcpy(ax, g_axt.ax, (size_t)g_axt.lenAX * sizeof(FPT));
    memcpy(sec, g_axt.sec, (size_t)g_axt.lenSEC * sizeof(UIN));
    memcpy(con, g_axt.con, (size_t)g_axt.lenCON * sizeof(UIN));
    free(g_axt.ax);
    free(g_axt.sec);
    free(g_axt.con);
}

}  // extern "C"
