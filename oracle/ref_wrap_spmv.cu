/*
 * ref_wrap_spmv.cu -- ORACLE TEST INFRASTRUCTURE.
 *
 * Compiles the reference's first-generation header spmv_header.h unchanged (path passed by
 * the build recipe as REF_SPMV_HEADER) and exposes its serial CPU CSR SpMV
 * cpuSpmvCSR (spmv_header.h:409-425) -- the single-core CPU path that spmv_main.cu times
 * (spmv_main.cu:79,149) -- as ref_cpuSpmvCSR.
 */
#include REF_SPMV_HEADER

extern "C" void ref_cpuSpmvCSR(UIN nrows, UIN nnz, const FPT *val, const UIN *col,
                               const UIN *row, const FPT *vec, FPT *res)
{
    str_matCSR m;
    memset(&m, 0, sizeof(m));
    m.nrows = nrows;
    m.nnz = nnz;
    m.val = (FPT *)val;
    m.col = (UIN *)col;
    m.row = (UIN *)row;
    cpuSpmvCSR(m, vec, res);
}
