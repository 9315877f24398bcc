/*
 * ref_wrap_spmv.cu -- ORACLE TEST INFRASTRUCTURE.
 *
 * Compiles the reference's first-generation header spmv_header.h unchanged (path passed by
 * the build recipe as REF_SPMV_HEADER) and exposes:
 *
 *   ref_cpuSpmvCSR  -> cpuSpmvCSR (spmv_header.h:409-425), the single-core CPU CSR SpMV that
 *                      spmv_main.cu times (spmv_main.cu:79,149);
 *   ref0_convert    -> getFormatDataAXCv0 / AXCv1 / AXBv0 / AXBv1 (spmv_header.h:711, 916,
 *                      1690, 2340), the brick formats of that generation: their arrays and
 *                      format data (name, mfp, beta) for comparison with the drop-in's;
 *   ref0_struct_layout -> sizeof / offsetof of that generation's structs.
 *
 * No reference code is copied here: the wrappers marshal arguments into the reference's own
 * structs and copy the arrays its converters return.
 */
#include REF_SPMV_HEADER

namespace {

str_matCSR view(UIN nrows, UIN nnz, const FPT *val, const UIN *col, const UIN *row, UIN *rl)
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

}  // namespace

extern "C" {

void ref_cpuSpmvCSR(UIN nrows, UIN nnz, const FPT *val, const UIN *col, const UIN *row,
                    const FPT *vec, FPT *res)
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

/* One brick format of the first generation.  kind: 0 AXCv0, 1 AXCv1, 2 AXBv0, 3 AXBv1
 * (cbs: the cudaBlockSize argument of getFormatDataAXBv1).  Returns the arrays in malloc'd
 * buffers: ax (lens[0] doubles) and up to two index arrays (lens[1], lens[2] words: AXCv0
 * brp; AXCv1 brp, rwp; AXBv0 hdr0; AXBv1 hdr1), lens[3] = AXBv1 blockLog; fd3 = mfp, beta,
 * ct; name receives the format name.  Free the buffers with ref0_free. */
void ref0_convert(int kind, UIN cbs, UIN nrows, UIN nnz, const FPT *val, const UIN *col,
                  const UIN *row, const FPT *vec, double *ax_lens_fd, FPT **ax, UIN **i1,
                  UIN **i2, UIN *lens, char *name)
{
    UIN *rl = (UIN *)malloc((size_t)(nrows ? nrows : 1) * sizeof(UIN));
    str_matCSR m = view(nrows, nnz, val, col, row, rl);
    str_formatData fd;
    *i1 = *i2 = NULL;
    lens[0] = lens[1] = lens[2] = lens[3] = 0;
    if (kind == 0) {
        str_matAXCv0 a;
        memset(&a, 0, sizeof(a));
        fd = getFormatDataAXCv0(1, m, vec, &a);
        *ax = a.ax; lens[0] = a.lenAX;
        *i1 = a.brp; lens[1] = a.lenBRP;
    } else if (kind == 1) {
        str_matAXCv1 a;
        memset(&a, 0, sizeof(a));
        fd = getFormatDataAXCv1(1, m, vec, &a);
        *ax = a.ax; lens[0] = a.lenAX;
        *i1 = a.brp; lens[1] = a.lenBRP;
        *i2 = a.rwp; lens[2] = a.lenRWP;
    } else if (kind == 2) {
        str_matAXBv0 a;
        memset(&a, 0, sizeof(a));
        fd = getFormatDataAXBv0(m, vec, &a);
        *ax = a.ax; lens[0] = a.lenAX;
        *i1 = a.hdr0; lens[1] = a.lenHDR;
    } else {
        str_matAXBv1 a;
        memset(&a, 0, sizeof(a));
        fd = getFormatDataAXBv1(cbs, m, vec, &a);
        *ax = a.ax; lens[0] = a.lenAX;
        *i1 = a.hdr1; lens[1] = a.lenHDR;
        lens[3] = a.blockLog;
    }
    ax_lens_fd[0] = fd.mfp;
    ax_lens_fd[1] = fd.beta;
    ax_lens_fd[2] = fd.ct;
    snprintf(name, 12, "%s", fd.name);
    free(rl);
}

void ref0_free(void *p) { free(p); }

/* sizeof and every field offset of the first generation's base and brick structs
 * (spmv_header.h:247, 370, 435, 464, 665, 851, 1649, 2299) as "name value" lines; returns
 * the characters written (0 if cap is too small). */
#define REF_SZ(T) n += snprintf(buf + n, cap > n ? cap - n : 0, #T " %zu\n", sizeof(T))
#define REF_OF(T, f) n += snprintf(buf + n, cap > n ? cap - n : 0, #T "." #f " %zu\n", offsetof(T, f))
size_t ref0_struct_layout(char *buf, size_t cap)
{
    size_t n = 0;
    REF_SZ(str_matCSR);
    REF_OF(str_matCSR, nrows); REF_OF(str_matCSR, nnz); REF_OF(str_matCSR, rmin);
    REF_OF(str_matCSR, rave); REF_OF(str_matCSR, rmax); REF_OF(str_matCSR, rsd);
    REF_OF(str_matCSR, bw); REF_OF(str_matCSR, val); REF_OF(str_matCSR, row);
    REF_OF(str_matCSR, col); REF_OF(str_matCSR, rl);
    REF_SZ(str_formatData);
    REF_OF(str_formatData, name); REF_OF(str_formatData, mfp); REF_OF(str_formatData, beta);
    REF_OF(str_formatData, ct);
    REF_SZ(str_err);
    REF_OF(str_err, aErr); REF_OF(str_err, rErr); REF_OF(str_err, pos);
    REF_SZ(str_res);
    REF_OF(str_res, name); REF_OF(str_res, et); REF_OF(str_res, flops); REF_OF(str_res, sErr);
    REF_SZ(str_matAXCv0);
    REF_OF(str_matAXCv0, nrows); REF_OF(str_matAXCv0, nnz); REF_OF(str_matAXCv0, lenAX);
    REF_OF(str_matAXCv0, lenBRP); REF_OF(str_matAXCv0, ax); REF_OF(str_matAXCv0, brp);
    REF_SZ(str_matAXCv1);
    REF_OF(str_matAXCv1, nrows); REF_OF(str_matAXCv1, nnz); REF_OF(str_matAXCv1, lenAX);
    REF_OF(str_matAXCv1, lenBRP); REF_OF(str_matAXCv1, lenRWP); REF_OF(str_matAXCv1, ax);
    REF_OF(str_matAXCv1, brp); REF_OF(str_matAXCv1, rwp);
    REF_SZ(str_matAXBv0);
    REF_OF(str_matAXBv0, nrows); REF_OF(str_matAXBv0, nnz); REF_OF(str_matAXBv0, brickNum);
    REF_OF(str_matAXBv0, lenAX); REF_OF(str_matAXBv0, lenHDR); REF_OF(str_matAXBv0, ax);
    REF_OF(str_matAXBv0, hdr0);
    REF_SZ(str_matAXBv1);
    REF_OF(str_matAXBv1, nrows); REF_OF(str_matAXBv1, nnz); REF_OF(str_matAXBv1, brickNum);
    REF_OF(str_matAXBv1, lenAX); REF_OF(str_matAXBv1, lenHDR); REF_OF(str_matAXBv1, blockLog);
    REF_OF(str_matAXBv1, ax); REF_OF(str_matAXBv1, hdr1);
    return n < cap ? n : 0;
}
#undef REF_SZ
#undef REF_OF

}  // extern "C"
