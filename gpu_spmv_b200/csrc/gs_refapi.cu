// gs_refapi.cu -- the drop-in layer: the reference program's host API (cudaSpmv.cu) with
// the same names, struct layouts and argument meaning, backed by the engine.
//
// Differences from the reference, all deliberate:
//  * converters run on the GPU (device scans / sort / scatter) and return the same host
//    arrays bit for bit; fd.ct is the device conversion time;
//  * entry points never exit(): failures print a message, return a result named "error"
//    (times 0) and leave the reason in gs_last_error();
//  * AXT entry points accept any tileHW (the reference's kernels hard-code 16/8/4/32) and
//    take the launch shape (wpw, tpw, cudaBlockSize) only for the result name;
//  * the AXT/AXC kernels write every y entry once, so y needs no memset between launches
//    (the reference memsets it outside its timing window, cudaSpmv.cu:1631);
//  * COM headers are decoded so that a header word equal to 0 (row 0, offset 0) still
//    counts -- gaxtch1 drops it (cudaSpmv.cu:2089).
#include <cusparse.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <vector>

#include "gs_internal.cuh"

extern "C" UIN gs_get_num_ite(void);

namespace {

using gs::DevBuf;

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~Timer() { cudaEventDestroy(a); cudaEventDestroy(b); }
};

str_res error_res(const char *name, const char *what)
{
    str_res r;
    memset(&r, 0, sizeof(r));
    strcpy(r.name, "error");
    fflush(stdout);
    printf("%s: %s\n", name, what);
    fflush(stdout);
    return r;
}

str_formatData error_fd(const char *name)
{
    str_formatData fd;
    memset(&fd, 0, sizeof(fd));
    strcpy(fd.name, "error");
    fflush(stdout);
    printf("%s: %s\n", name, gs_last_error());
    fflush(stdout);
    return fd;
}

template <class T> gs_status h2d(DevBuf &b, const T *h, size_t n)
{
    GS_TRY(b.alloc(n * sizeof(T)));
    if (n) GS_CUDA(cudaMemcpy(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return GS_OK;
}

template <class T> T *d2h_calloc(const void *d, size_t n)
{
    T *h = static_cast<T *>(calloc(n ? n : 1, sizeof(T)));
    if (h && n) cudaMemcpy(h, d, n * sizeof(T), cudaMemcpyDeviceToHost);
    return h;
}

// y of the calling thread's last test_* product that ran (host copy, row order)
thread_local std::vector<FPT> g_last_y;

// Times gs_get_num_ite() launches of `launch` (legacy default stream, CUDA events around
// each launch, as the reference's test_* loops do), then scores y against ref.
str_res timed(const char *name, UIN nrows, UIN nnz, const std::function<gs_status()> &launch,
              const DevBuf &dy, const FPT *ref)
{
    const UIN ite = gs_get_num_ite();
    Timer t;
    float tt = 0.f;
    for (UIN i = 0; i < ite; i++) {
        cudaEventRecord(t.a, 0);
        gs_status st = launch();
        cudaEventRecord(t.b, 0);
        cudaEventSynchronize(t.b);
        if (st != GS_OK) return error_res(name, gs_last_error());
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t.a, t.b);
        tt += ms;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return error_res(name, cudaGetErrorString(e));
    str_res sr;
    memset(&sr, 0, sizeof(sr));
    snprintf(sr.name, sizeof(sr.name), "%s", name);
    sr.et = ((double)tt / (double)ite) * 1e-3;
    sr.ot = 0.0;
    sr.flops = (2.0 * (double)nnz) / sr.et;
    FPT *res = d2h_calloc<FPT>(dy.p, nrows);
    get_errors(nrows, ref, res, &sr.sErr);
    if (res) g_last_y.assign(res, res + nrows);
    free(res);
    return sr;
}

// rpos[r] = src[r] / div  (UNC tileH=1 con, AXC brp -> first slot of each row)
__global__ void k_div_table(uint32_t n1, const uint32_t *src, uint32_t div, uint32_t *rpos)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n1) rpos[i] = src[i] / div;
}

// UNC tileH>1: rpos[r] = th * (first tile column of r), from con[r] = t*2*ths + c;
// rpos[n] = tileN * th * thw (trailing unused columns count as padding of the last row).
__global__ void k_unc_table(uint32_t n, const uint32_t *con, uint32_t thw, uint32_t th,
                            uint32_t tileN, uint32_t *rpos)
{
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t ths = thw * th;
    if (r < n) rpos[r] = th * ((con[r] / (2 * ths)) * thw + con[r] % thw);
    if (r == n) rpos[n] = tileN * ths;
}

// COM: recover row lengths from the header words.  Position p (CSR order) is a segment
// start iff it opens a segment block (p % blk == 0, blk = bs for tileH=1, th for tileH>1:
// the reference always writes a header there) or its header word is non-zero; the
// segment covers offset+1 positions of row hdr >> log.
__global__ void k_com_rowlen(uint32_t nnz, uint32_t n, const uint32_t *sec, uint32_t thw,
                             uint32_t th, uint32_t blk, uint32_t log, uint32_t *rl,
                             uint32_t *flag)
{
    const uint32_t ths = thw * th;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz;
         p += gridDim.x * blockDim.x) {
        uint32_t slot = p;
        if (th > 1) {
            const uint32_t t = p / ths, rem = p - t * ths, c = rem / th;
            slot = t * ths + (rem - c * th) * thw + c;
        }
        const uint32_t h = sec[slot];
        if (p % blk == 0 || h != 0) {
            const uint32_t r = h >> log, o = h & (blk - 1);
            if (r >= n) { atomicOr(flag, 1u); continue; }
            atomicAdd(rl + r, o + 1);
        }
    }
}

__global__ void k_narrow(uint32_t n1, const uint64_t *a, uint32_t *b)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n1) b[i] = (uint32_t)a[i];
}

gs_status com_rpos(const str_matAXT &m, const DevBuf &dsec, DevBuf &rpos)
{
    const uint32_t blk = m.tileH == 1 ? m.bs : m.tileH;
    if (blk == 0 || (blk & (blk - 1)) != 0 || (1u << m.log) != blk)
        return gs::fail(GS_ERR_UNSUPPORTED,
                        "COM headers decode only for a power-of-two %s (got %u, log %u)",
                        m.tileH == 1 ? "bs" : "tileH", blk, m.log);
    DevBuf rl, flag, P;
    GS_TRY(rl.alloc_zero((size_t)m.nrows * 4 + 4, 0));
    GS_TRY(flag.alloc_zero(4, 0));
    k_com_rowlen<<<1184, 256>>>(m.nnz, m.nrows, dsec.as<uint32_t>(), m.tileHW, m.tileH, blk,
                                m.log, rl.as<uint32_t>(), flag.as<uint32_t>());
    GS_CHECK_LAUNCH();
    uint32_t hf = 0;
    GS_CUDA(cudaMemcpy(&hf, flag.p, 4, cudaMemcpyDeviceToHost));
    if (hf) return gs::fail(GS_ERR_INVALID, "COM header names a row beyond nrows");
    GS_TRY(P.alloc(((size_t)m.nrows + 1) * 8));
    gs::CountSpec cs{gs::CountKind::Array};
    cs.arr = rl.as<uint32_t>();
    uint64_t total = 0;
    GS_TRY(gs::exclusive_scan(cs, m.nrows, P.as<uint64_t>(), &total, 0));
    if (total != m.nnz)
        return gs::fail(GS_ERR_INVALID, "COM headers cover %llu positions, nnz is %u",
                        (unsigned long long)total, m.nnz);
    GS_TRY(rpos.alloc(((size_t)m.nrows + 1) * 4));
    k_narrow<<<(m.nrows + 256) / 256, 256>>>(m.nrows + 1, P.as<uint64_t>(), rpos.as<uint32_t>());
    GS_CHECK_LAUNCH();
    return GS_OK;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------ I/O and statistics
str_matCSR matrixReading(const char *matFileName)
{
    str_matCSR m;
    memset(&m, 0, sizeof(m));
    if (!matFileName) return m;
    snprintf(m.name, sizeof(m.name), "%s", matFileName);
    const char *kind = strstr(matFileName, ".csr") ? "csr" : (strstr(matFileName, ".bin") ? "bin" : nullptr);
    if (!kind) {
        printf("\nmatrixReading detected that %s has NOT .csr or .bin extension\n\n", matFileName);
        gs::fail(GS_ERR_INVALID, "%s has neither a .csr nor a .bin extension", matFileName);
        return m;
    }
    FILE *fh = fopen(matFileName, kind[0] == 'c' ? "r" : "rb");
    if (!fh) {
        printf("\nmatrixReading is unable to open .%s file\n\n", kind);
        gs::fail(GS_ERR_INVALID, "cannot open %s", matFileName);
        return m;
    }
    bool ok = true;
    UIN n = 0, nnz = 0;
    if (kind[0] == 'c') {
        ok = fscanf(fh, "%u %u", &n, &nnz) == 2;
    } else {
        ok = fread(&n, sizeof(UIN), 1, fh) == 1 && fread(&nnz, sizeof(UIN), 1, fh) == 1;
    }
    if (ok) {
        m.nrows = n;
        m.nnz = nnz;
        m.val = (FPT *)malloc((size_t)(nnz ? nnz : 1) * sizeof(FPT));
        m.col = (UIN *)malloc((size_t)(nnz ? nnz : 1) * sizeof(UIN));
        m.row = (UIN *)malloc(((size_t)n + 1) * sizeof(UIN));
        m.rl = (UIN *)malloc((size_t)(n ? n : 1) * sizeof(UIN));
        ok = m.val && m.col && m.row && m.rl;
    }
    if (ok && kind[0] == 'c') {
        for (UIN i = 0; ok && i < nnz; i++) ok = fscanf(fh, "%lf %u", &m.val[i], &m.col[i]) == 2;
        for (UIN i = 0; ok && i <= n; i++) ok = fscanf(fh, "%u", &m.row[i]) == 1;
    } else if (ok) {
        ok = fread(m.val, sizeof(FPT), nnz, fh) == nnz && fread(m.col, sizeof(UIN), nnz, fh) == nnz &&
             fread(m.row, sizeof(UIN), (size_t)n + 1, fh) == (size_t)n + 1;
    }
    fclose(fh);
    if (!ok) {
        printf("\nmatrixReading failed to parse %s\n\n", matFileName);
        gs::fail(GS_ERR_INVALID, "malformed matrix file %s", matFileName);
        free(m.val); free(m.col); free(m.row); free(m.rl);
        memset(&m, 0, sizeof(m));
    }
    return m;
}

int matrixWritingBin(const char *matFileName, const str_matCSR *m)
{
    if (!matFileName || !m) return -1;
    FILE *fh = fopen(matFileName, "wb");
    if (!fh) return -1;
    bool ok = fwrite(&m->nrows, sizeof(UIN), 1, fh) == 1 && fwrite(&m->nnz, sizeof(UIN), 1, fh) == 1 &&
              fwrite(m->val, sizeof(FPT), m->nnz, fh) == m->nnz &&
              fwrite(m->col, sizeof(UIN), m->nnz, fh) == m->nnz &&
              fwrite(m->row, sizeof(UIN), (size_t)m->nrows + 1, fh) == (size_t)m->nrows + 1;
    return (fclose(fh) == 0 && ok) ? 0 : -1;
}

}  // extern "C"

// Statistics of cudaSpmv.cu:332-381 (and gpuSpmv_header.h:322-371, the same numbers and
// file) written to "<name>.sta": name = the path up to the first '.' of its last component
// (first API generation) or of the whole path (second: strtok on the full name).
static void stats_core(const char *matFileName, str_matCSR *m, bool dot_anywhere)
{
    UIN rmin = 1000000000u, rmax = 0, bw = 0;
    double s1 = 0.0, s2 = 0.0;
    for (UIN i = 0; i < m->nrows; i++) {
        const UIN l = m->row[i + 1] - m->row[i];
        m->rl[i] = l;
        s1 += l;
        s2 += (double)(UIN)(l * l);  // 32-bit square, as cudaSpmv.cu:342
        rmin = l < rmin ? l : rmin;
        rmax = l > rmax ? l : rmax;
        for (UIN j = m->row[i]; j < m->row[i + 1]; j++) {
            int d = abs((int)i - (int)m->col[j]);
            if ((UIN)d > bw) bw = (UIN)d;
        }
    }
    s1 /= (double)m->nrows;
    s2 /= (double)m->nrows;
    const double sd = sqrt(s2 - s1 * s1);
    m->rmin = rmin;
    m->rave = s1;
    m->rmax = rmax;
    m->rsd = sd;
    m->bw = bw;
    // "<file name up to its first '.'>.sta", next to the matrix file
    char path[512];
    snprintf(path, sizeof(path), "%s", matFileName ? matFileName : "matrix");
    char *slash = dot_anywhere ? nullptr : strrchr(path, '/');
    char *dot = strchr(slash ? slash + 1 : path, '.');
    if (dot) *dot = 0;
    strncat(path, ".sta", sizeof(path) - strlen(path) - 1);
    FILE *fh = fopen(path, "w+");
    if (!fh) return;
    fprintf(fh, "------------------------------------\n");
    fprintf(fh, "matrix's statistics\n");
    fprintf(fh, "------------------------------------\n");
    fprintf(fh, "name:  %28s\n", matFileName ? matFileName : "");
    fprintf(fh, "nrows: %28d\n", m->nrows);
    fprintf(fh, "nnz:   %28d\n", m->nnz);
    fprintf(fh, "rmin:  %28d\n", m->rmin);
    fprintf(fh, "rave:  %28.2lf\n", m->rave);
    fprintf(fh, "rmax:  %28d\n", m->rmax);
    fprintf(fh, "rsd:   %28.2lf\n", m->rsd);
    fprintf(fh, "rsdp:  %28.2lf\n", (sd / s1) * 100);
    fprintf(fh, "bw:    %28d\n", m->bw);
    fclose(fh);
}

extern "C" {

UIN gs_dropin_last_y(FPT *out, UIN cap)
{
    const UIN n = (UIN)g_last_y.size();
    if (out && cap >= n && n) memcpy(out, g_last_y.data(), (size_t)n * sizeof(FPT));
    return n;
}

void printMatrixStats(const char *matFileName, str_matCSR *m) { stats_core(matFileName, m, false); }

str_formatData getFormatDataCSR(str_matCSR *m)
{
    str_formatData fd;
    memset(&fd, 0, sizeof(fd));
    m->rowStart = (UIN *)calloc(m->nrows ? m->nrows : 1, sizeof(UIN));
    m->rowEnd = (UIN *)calloc(m->nrows ? m->nrows : 1, sizeof(UIN));
    struct timespec t1, t2;
    clock_gettime(CLOCK_MONOTONIC, &t1);
    for (UIN i = 0; i < m->nrows; i++) {
        m->rowStart[i] = m->row[i];
        m->rowEnd[i] = m->row[i + 1];
    }
    clock_gettime(CLOCK_MONOTONIC, &t2);
    strcpy(fd.name, "fcsr");
    fd.mfp = (double)m->nnz * sizeof(FPT) + (double)m->nnz * sizeof(UIN) +
             ((double)m->nrows + 1) * sizeof(UIN) + (double)m->nrows * sizeof(FPT);
    fd.beta = (double)m->nnz / (double)m->nnz;
    fd.ct = (double)(t2.tv_sec - t1.tv_sec) + (double)(t2.tv_nsec - t1.tv_nsec) * 1e-9;
    return fd;
}

void init_vec(const UIN ompNT, const UIN len, FPT *vec)
{
    (void)ompNT;
    for (UIN i = 0; i < len; i++) vec[i] = (FPT)i;
}

void get_errors(const UIN len, const FPT *ar, const FPT *ac, str_err *e)
{
    double md = 0.0, mv = 0.0;
    UIN pos = 0;
    for (UIN i = 0; i < len; i++) {
        const double v = fabs(ar[i]);
        if (v > mv) mv = v;
        const double d = fabs(fabs(ac[i]) - v);
        if (d > md) { md = d; pos = i; }
    }
    e->aErr = md;
    e->rErr = md / mv;
    e->pos = pos;
}

void ncsr(const UIN ompNT, const str_matCSR m, const FPT *vec, FPT *res)
{
    (void)ompNT;
    DevBuf row, col, val, x, y;
    if (h2d(row, m.row, (size_t)m.nrows + 1) || h2d(col, m.col, m.nnz) ||
        h2d(val, m.val, m.nnz) || h2d(x, vec, m.nrows) || y.alloc((size_t)m.nrows * 8) ||
        gs_csr_spmv_f64(m.nrows, m.nrows, m.nnz, row.as<UIN>(), col.as<UIN>(), val.as<double>(),
                        x.as<double>(), y.as<double>(), nullptr) ||
        cudaMemcpy(res, y.p, (size_t)m.nrows * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
        fflush(stdout);
        printf("ncsr: %s\n", gs_last_error());
        fflush(stdout);
    }
}

// ------------------------------------------------------------------ converters
static gs_status upload_csr(const str_matCSR &m, DevBuf &row, DevBuf &col, DevBuf &val)
{
    GS_TRY(h2d(row, m.row, (size_t)m.nrows + 1));
    GS_TRY(h2d(col, m.col, m.nnz));
    GS_TRY(h2d(val, m.val, m.nnz));
    return GS_OK;
}

str_formatData getFormatDataK1(const UIN blockSize, const str_matCSR m, const FPT *vec,
                               str_matK1 *k)
{
    (void)blockSize;
    (void)vec;
    DevBuf row, col, val;
    gs_matrix A;
    gs_convert_params p{};
    p.format = GS_FMT_K1;
    p.vtype = GS_F64;
    p.itype = GS_IDX_U32;
    p.keep_layout = 1;
    if (upload_csr(m, row, col, val) ||
        gs::convert(&A, p, m.nrows, m.nrows, m.nnz, row.as<UIN>(), col.as<UIN>(), val.p, GS_F64,
                    nullptr, nullptr, 0))
        return error_fd("getFormatDataK1");
    k->nrows = m.nrows;
    k->nnz = m.nnz;
    k->chunkNum = A.chunkNum;
    k->lenVC = A.lenVC;
    k->permi = d2h_calloc<UIN>(A.permi.p, ((size_t)A.chunkNum + 1) * 32);
    k->nmc = d2h_calloc<UIN>(A.nmc.p, A.chunkNum);
    k->chp = d2h_calloc<UIN>(A.chp.p, A.chunkNum);
    k->val = d2h_calloc<FPT>(A.val.p, A.lenVC);
    k->col = d2h_calloc<UIN>(A.col.p, A.lenVC);
    str_formatData fd;
    memset(&fd, 0, sizeof(fd));
    strcpy(fd.name, "fk1");
    fd.mfp = A.mfp;
    fd.beta = A.beta;
    fd.ct = A.conv_ms * 1e-3;
    return fd;
}

str_formatData getFormatDataAXC(const UIN ompNT, const UIN hbs, const str_matCSR m,
                                const FPT *vec, str_matAXC *a)
{
    (void)ompNT;
    DevBuf row, col, val, x, ax;
    gs_matrix A;
    gs_convert_params p{};
    p.format = GS_FMT_AXC;
    p.hbs = hbs;
    p.vtype = GS_F64;
    p.itype = GS_IDX_U32;
    p.keep_layout = 1;
    if (upload_csr(m, row, col, val) || h2d(x, vec, m.nrows) ||
        gs::convert(&A, p, m.nrows, m.nrows, m.nnz, row.as<UIN>(), col.as<UIN>(), val.p, GS_F64,
                    x.as<double>(), &ax, 0))
        return error_fd("getFormatDataAXC");
    a->nrows = m.nrows;
    a->nnz = m.nnz;
    a->hbs = hbs;
    a->lenAX = A.lenAX;
    a->lenBRP = A.lenBRP;
    a->lenMAPX = A.lenMAPX;
    a->ax = d2h_calloc<FPT>(ax.p, A.lenAX);
    a->brp = d2h_calloc<UIN>(A.brp.p, A.lenBRP);
    a->mapx = d2h_calloc<UIN>(A.mapx.p, A.lenMAPX);
    str_formatData fd;
    memset(&fd, 0, sizeof(fd));
    strcpy(fd.name, "faxc");
    fd.mfp = A.mfp;
    fd.beta = A.beta;
    fd.ct = A.conv_ms * 1e-3;
    return fd;
}

str_formatData getFormatDataAXT(const UIN ompNT, const UIN bs, const UIN thw, const UIN th,
                                const char *mode, const str_matCSR m, const FPT *vec,
                                str_matAXT *a)
{
    (void)ompNT;
    const bool unc = mode && (strcmp(mode, "UNC") == 0 || strcmp(mode, "NOC") == 0);
    const bool com = mode && strcmp(mode, "COM") == 0;
    if (!unc && !com) {
        gs::fail(GS_ERR_INVALID, "mode must be \"UNC\" (or \"NOC\") or \"COM\"");
        return error_fd("getFormatDataAXT");
    }
    DevBuf row, col, val, x, ax;
    gs_matrix A;
    gs_convert_params p{};
    p.format = GS_FMT_AXT;
    p.tileHW = thw;
    p.tileH = th;
    p.bs = bs;
    p.mode = unc ? GS_AXT_UNC : GS_AXT_COM;
    p.vtype = GS_F64;
    p.itype = GS_IDX_U32;
    p.keep_layout = 1;
    if (upload_csr(m, row, col, val) || h2d(x, vec, m.nrows) ||
        gs::convert(&A, p, m.nrows, m.nrows, m.nnz, row.as<UIN>(), col.as<UIN>(), val.p, GS_F64,
                    x.as<double>(), &ax, 0))
        return error_fd("getFormatDataAXT");
    snprintf(a->name, sizeof(a->name), "%s", m.name);
    a->nrows = m.nrows;
    a->nnz = m.nnz;
    snprintf(a->mode, sizeof(a->mode), "%s", mode);
    a->tileHW = thw;
    a->tileH = th;
    a->logTH = A.logTH;
    a->tileN = A.tileN;
    a->lenAX = A.lenAX;
    a->lenSEC = A.lenSEC;
    a->lenCON = A.lenCON;
    a->log = A.log;
    a->bs = bs;
    a->ax = d2h_calloc<FPT>(ax.p, A.lenAX);
    a->sec = d2h_calloc<UIN>(A.sec.p, A.lenSEC);
    a->con = d2h_calloc<UIN>(A.con.p, (size_t)A.lenCON + 1);
    str_formatData fd;
    memset(&fd, 0, sizeof(fd));
    if (unc && th == 1) snprintf(fd.name, sizeof(fd.name), "faxtuh1hw%u", thw);
    else if (unc) snprintf(fd.name, sizeof(fd.name), "faxtuh%uhw%u", th, thw);
    else if (th == 1) snprintf(fd.name, sizeof(fd.name), "faxtch1hw%ubs%u", thw, bs);
    else snprintf(fd.name, sizeof(fd.name), "faxtch%uhw%u", th, thw);
    fd.mfp = A.mfp;
    fd.beta = A.beta;
    fd.ct = A.conv_ms * 1e-3;
    return fd;
}

// ------------------------------------------------------------------ entry points
str_res test_gcsr(const UIN cudaBlockSize, const str_matCSR m, const FPT *vec, const FPT *ref)
{
    (void)cudaBlockSize;
    DevBuf row, col, val, x, y;
    gs::RowsPlan P;
    uint32_t V = gs::kDirectV;
    if (upload_csr(m, row, col, val) || h2d(x, vec, m.nrows) || y.alloc((size_t)m.nrows * 8) ||
        gs::direct_lane_positions(row.as<UIN>(), col.as<UIN>(), m.nrows, m.nnz, &V, 0) ||
        gs::build_rows_plan(row.as<UIN>(), nullptr, m.nrows, V, P, 0))
        return error_res("gcsr", gs_last_error());
    gs::RowsArgs a = gs::rows_args(P);
    a.val = val.p;
    a.col = col.p;
    a.x = x.p;
    a.y = y.p;
    a.nslots = m.nnz;
    return timed("gcsr", m.nrows, m.nnz, [&]() {
        return gs::launch_rows(a, GS_F64, GS_IDX_U32, GS_F64, 0, false, false, false, 0);
    }, y, ref);
}

str_res test_gcucsr(const str_matCSR m, const FPT *vec, const FPT *ref)
{
    DevBuf row, col, val, x, y, buf;
    if (upload_csr(m, row, col, val) || h2d(x, vec, m.nrows) || y.alloc((size_t)m.nrows * 8))
        return error_res("gcucsr", gs_last_error());
    cusparseHandle_t h = nullptr;
    cusparseSpMatDescr_t A = nullptr;
    cusparseDnVecDescr_t vx = nullptr, vy = nullptr;
    const double one = 1.0, zero = 0.0;
    size_t bsz = 0;
    if (cusparseCreate(&h) != CUSPARSE_STATUS_SUCCESS ||
        cusparseCreateCsr(&A, m.nrows, m.nrows, m.nnz, row.p, col.p, val.p, CUSPARSE_INDEX_32I,
                          CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F) !=
            CUSPARSE_STATUS_SUCCESS ||
        cusparseCreateDnVec(&vx, m.nrows, x.p, CUDA_R_64F) != CUSPARSE_STATUS_SUCCESS ||
        cusparseCreateDnVec(&vy, m.nrows, y.p, CUDA_R_64F) != CUSPARSE_STATUS_SUCCESS ||
        cusparseSpMV_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, A, vx, &zero, vy,
                                CUDA_R_64F, CUSPARSE_SPMV_ALG_DEFAULT, &bsz) !=
            CUSPARSE_STATUS_SUCCESS ||
        buf.alloc(bsz)) {
        if (vy) cusparseDestroyDnVec(vy);
        if (vx) cusparseDestroyDnVec(vx);
        if (A) cusparseDestroySpMat(A);
        if (h) cusparseDestroy(h);
        return error_res("gcucsr", "cuSPARSE set-up failed");
    }
    str_res r = timed("gcucsr", m.nrows, m.nnz, [&]() -> gs_status {
        return cusparseSpMV(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, A, vx, &zero, vy,
                            CUDA_R_64F, CUSPARSE_SPMV_ALG_DEFAULT, buf.p) == CUSPARSE_STATUS_SUCCESS
                   ? GS_OK
                   : gs::fail(GS_ERR_CUDA, "cusparseSpMV failed");
    }, y, ref);
    cusparseDestroyDnVec(vy);
    cusparseDestroyDnVec(vx);
    cusparseDestroySpMat(A);
    cusparseDestroy(h);
    return r;
}

str_res test_gk1(const UIN cudaBlockSize, const str_matK1 k, const FPT *vec, const FPT *ref)
{
    (void)cudaBlockSize;
    DevBuf permi, nmc, chp, val, col, x, y, uc, ub, part, cnt;
    uint32_t units = 0;
    if (h2d(permi, k.permi, ((size_t)k.chunkNum + 1) * 32) || h2d(nmc, k.nmc, k.chunkNum) ||
        h2d(chp, k.chp, k.chunkNum) || h2d(val, k.val, k.lenVC) || h2d(col, k.col, k.lenVC) ||
        h2d(x, vec, k.nrows) || y.alloc((size_t)k.nrows * 8) ||
        gs::build_k1_plan(nmc.as<UIN>(), k.chunkNum, uc, ub, part, cnt, &units, 0))
        return error_res("gk1", gs_last_error());
    gs::K1Args a{};
    a.nrows = k.nrows;
    a.chunkNum = k.chunkNum;
    a.permi = permi.as<UIN>();
    a.nmc = nmc.as<UIN>();
    a.chp = chp.as<UIN>();
    a.klen = nullptr;  // struct carries no row lengths: read each chunk's padded width
    a.val = val.p;
    a.col = col.p;
    a.x = x.p;
    a.y = y.p;
    a.unit_chunk = uc.as<UIN>();
    a.unit_base = ub.as<UIN>();
    a.units = units;
    a.partial = part.as<double>();
    a.count = cnt.as<UIN>();
    return timed("gk1", k.nrows, k.nnz, [&]() {
        return gs::launch_k1(a, GS_F64, GS_IDX_U32, GS_F64, false, 0);
    }, y, ref);
}

// align: rows start on multiples of `align` positions (UNC tiles / columns, AXC bricks),
// 0 for the compact COM layouts.
static str_res run_baked(const char *name, UIN nrows, UIN nnz, const FPT *hax, UIN lenAX,
                         DevBuf &rpos, bool tiled, UIN thw, UIN th, UIN axw, UIN align,
                         const FPT *ref)
{
    DevBuf ax, y;
    gs::RowsPlan P;
    if (!tiled && align == axw && (axw == 4 || axw == 8 || axw == 16 || axw == 32)) {
        // whole [axw values | axw x] tiles per row (UNC tileH = 1, AXC): the tile kernel,
        // its plan built over tiles (row r starts at tile rpos[r] / axw), in windows of one
        // 32-tile chunk (a tile is 2 axw values: small matrices still get many warps)
        DevBuf rtile;
        if (h2d(ax, hax, lenAX) || y.alloc((size_t)nrows * 8) ||
            rtile.alloc(((size_t)nrows + 1) * 4))
            return error_res(name, gs_last_error());
        k_div_table<<<(nrows + 256) / 256, 256>>>(nrows + 1, rpos.as<UIN>(), axw,
                                                  rtile.as<UIN>());
        if (gs::build_rows_plan(rtile.as<UIN>(), nullptr, nrows, 1, P, 0))
            return error_res(name, gs_last_error());
        gs::RowsArgs a = gs::rows_args(P);
        a.val = ax.p;
        a.y = y.p;
        return timed(name, nrows, nnz, [&]() { return gs::launch_tiles(a, axw, true, 0); }, y,
                     ref);
    }
    uint32_t V = tiled ? th : gs::kDirectV;
    bool aligned = false;
    if (tiled) aligned = align != 0 && (th == 2 || th == 4 || th == 8 || th == 16);
    else if (align) V = gs::aligned_lane_positions(align, &aligned);
    if (h2d(ax, hax, lenAX) || y.alloc((size_t)nrows * 8) ||
        gs::build_rows_plan(rpos.as<UIN>(), nullptr, nrows, V, P, 0, tiled))
        return error_res(name, gs_last_error());
    P.aligned = aligned;
    gs::RowsArgs a = gs::rows_args(P);
    a.val = ax.p;
    a.col = nullptr;
    a.x = nullptr;
    a.y = y.p;
    if (tiled) {
        a.thw = thw;
        a.th = th;
    }
    a.axw = axw;
    a.nslots = lenAX / 2;
    return timed(name, nrows, nnz, [&]() {
        return gs::launch_rows(a, GS_F64, GS_IDX_U32, GS_F64, 0, tiled, true, false, 0);
    }, y, ref);
}

str_res test_gaxc(const UIN cudaBlockSize, const str_matAXC m, const FPT *ref)
{
    (void)cudaBlockSize;
    DevBuf brp, rpos;
    if (m.hbs == 0) return error_res("gaxc", "hbs is 0");
    if (h2d(brp, m.brp, m.lenBRP) || rpos.alloc(((size_t)m.nrows + 1) * 4))
        return error_res("gaxc", gs_last_error());
    k_div_table<<<(m.nrows + 256) / 256, 256>>>(m.nrows + 1, brp.as<UIN>(), 2, rpos.as<UIN>());
    return run_baked("gaxc", m.nrows, m.nnz, m.ax, m.lenAX, rpos, false, m.hbs, 1, m.hbs, m.hbs,
                     ref);
}

static str_res test_unc1(const char *base, UIN wpw, const str_matAXT m, const FPT *ref)
{
    char name[48];
    snprintf(name, sizeof(name), "%s%u", base, wpw);
    if (strcmp(m.mode, "UNC") != 0 && strcmp(m.mode, "NOC") != 0)
        return error_res(name, "matrix is not an UNC AXT layout");
    if (m.tileH != 1) return error_res(name, "tileH must be 1");
    DevBuf con, rpos;
    if (h2d(con, m.con, (size_t)m.lenCON + 1) || rpos.alloc(((size_t)m.nrows + 1) * 4))
        return error_res(name, gs_last_error());
    k_div_table<<<(m.nrows + 256) / 256, 256>>>(m.nrows + 1, con.as<UIN>(), 2, rpos.as<UIN>());
    return run_baked(name, m.nrows, m.nnz, m.ax, m.lenAX, rpos, false, m.tileHW, 1, m.tileHW,
                     m.tileHW, ref);
}

str_res test_gaxtuh1hw16w(const UIN wpw, const UIN cbs, const str_matAXT m, const FPT *ref)
{
    (void)cbs;
    return test_unc1("gaxtuh1hw16w", wpw, m, ref);
}
str_res test_gaxtuh1hw08w(const UIN wpw, const UIN cbs, const str_matAXT m, const FPT *ref)
{
    (void)cbs;
    return test_unc1("gaxtuh1hw08w", wpw, m, ref);
}
str_res test_gaxtuh1hw04w(const UIN wpw, const UIN cbs, const str_matAXT m, const FPT *ref)
{
    (void)cbs;
    return test_unc1("gaxtuh1hw04w", wpw, m, ref);
}

str_res test_gaxtuh(const UIN tpw, const UIN cbs, const str_matAXT m, const FPT *ref)
{
    (void)cbs;
    char name[48];
    snprintf(name, sizeof(name), "gaxtuh%utpw%u", m.tileH, tpw);
    if (strcmp(m.mode, "UNC") != 0 && strcmp(m.mode, "NOC") != 0)
        return error_res(name, "matrix is not an UNC AXT layout");
    if (m.tileH < 2) return error_res(name, "tileH must be > 1");
    DevBuf con, rpos;
    if (h2d(con, m.con, (size_t)m.lenCON + 1) || rpos.alloc(((size_t)m.nrows + 1) * 4))
        return error_res(name, gs_last_error());
    k_unc_table<<<(m.nrows + 256) / 256, 256>>>(m.nrows, con.as<UIN>(), m.tileHW, m.tileH,
                                                m.tileN, rpos.as<UIN>());
    return run_baked(name, m.nrows, m.nnz, m.ax, m.lenAX, rpos, true, m.tileHW, m.tileH,
                     m.tileHW, m.tileH, ref);
}

static str_res test_com(const char *name, const str_matAXT m, const FPT *ref)
{
    if (strcmp(m.mode, "COM") != 0) return error_res(name, "matrix is not a COM AXT layout");
    DevBuf sec, rpos;
    if (h2d(sec, m.sec, m.lenSEC) || com_rpos(m, sec, rpos)) return error_res(name, gs_last_error());
    return run_baked(name, m.nrows, m.nnz, m.ax, m.lenAX, rpos, m.tileH > 1, m.tileHW, m.tileH,
                     m.tileHW, 0, ref);
}

str_res test_gaxtch1(const UIN cudaBlockSize, const str_matAXT m, const FPT *ref)
{
    (void)cudaBlockSize;
    char name[48];
    snprintf(name, sizeof(name), "gaxtch1bs%u", m.bs);
    if (m.tileH != 1) return error_res(name, "tileH must be 1");
    return test_com(name, m, ref);
}

str_res test_gaxtch(const UIN cudaBlockSize, const str_matAXT m, const FPT *ref)
{
    (void)cudaBlockSize;
    char name[48];
    snprintf(name, sizeof(name), "gaxtch%u", m.tileH);
    if (m.tileH < 2) return error_res(name, "tileH must be > 1");
    return test_com(name, m, ref);
}

}  // extern "C"

// ======================================================================================
// Second API generation (gpuSpmv_header.h), exported as gs2_* (gpuspmv_b200_gen2.h).
// Each call maps the second generation's structs onto the first generation's and reuses its
// converters and entry points; only the arrays that differ are made here: COM tileH = 1
// header words at every tile boundary and con for every row (gpuSpmv_header.h:1086-1115,
// 1193-1227).
// ======================================================================================
#define GS2_NO_ALIASES
#include "gpuspmv_b200_gen2.h"

namespace {

// con[r] = ax position of the start of row r (gpuSpmv_header.h:1097-1101 with positions =
// row length, COM); COM tileH = 1 (sec != nullptr): header word at every element that
// starts a row or a tile, (row << log) | min(elements left in the row - 1, 31 - p % thw)
// with the reference's unsigned arithmetic.
__global__ void k_gen2_com(UIN n, const UIN *row, UIN thw, UIN th, UIN log, UIN *sec,
                           UIN *con)
{
    const UIN r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const UIN ths = thw * th, p0 = row[r];
    const UIN t = (p0 + ths) / ths - 1;
    con[r] = t * (2 * ths) + (p0 % th) * (2 * thw) + ((p0 + th) / th - 1 - t * thw);
    if (!sec) return;
    const UIN len = row[r + 1] - p0;
    for (UIN e = 0; e < len; e++) {
        const UIN p = p0 + e, c = p % thw;
        if (c == 0 || e == 0) {
            const UIN q1 = len - e - 1, q2 = 31u - c;
            sec[p] = (r << log) | (q1 > q2 ? q2 : q1);
        }
    }
}

// rpos[r] = CSR position of row r's first element from con (COM tileH = 1), rpos[n] = nnz
__global__ void k_gen2_com_rpos(UIN n, UIN nnz, const UIN *con, UIN thw, UIN *rpos)
{
    const UIN r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) rpos[r] = (con[r] / (2 * thw)) * thw + con[r] % (2 * thw);
    if (r == n) rpos[n] = nnz;
}

str_matCSR gen1_view(const gs2_matCSR &m)
{
    str_matCSR v;
    memset(&v, 0, sizeof(v));
    strcpy(v.name, "gen2");
    v.nrows = m.nrows;
    v.nnz = m.nnz;
    v.rmin = m.rmin;
    v.rave = m.rave;
    v.rmax = m.rmax;
    v.rsd = m.rsd;
    v.bw = m.bw;
    v.val = m.val;
    v.row = m.row;
    v.col = m.col;
    v.rl = m.rl;
    return v;
}

gs2_res gen2_res(const str_res &r, const char *name)
{
    gs2_res o;
    memset(&o, 0, sizeof(o));
    snprintf(o.name, sizeof(o.name), "%s", strcmp(r.name, "error") ? name : "error");
    o.et = r.et;
    o.flops = r.flops;
    o.sErr.aErr = r.sErr.aErr;
    o.sErr.rErr = r.sErr.rErr;
    o.sErr.pos = r.sErr.pos;
    return o;
}

gs2_formatData gen2_fd(const char *name, double mfp, double beta, double ct)
{
    gs2_formatData fd;
    memset(&fd, 0, sizeof(fd));
    const size_t len = std::min(strlen(name), sizeof(fd.name) - 1);  // name[18]
    memcpy(fd.name, name, len);
    fd.mfp = mfp;
    fd.beta = beta;
    fd.ct = ct;
    return fd;
}

gs2_formatData gen2_error_fd()
{
    gs2_formatData fd;
    memset(&fd, 0, sizeof(fd));
    strcpy(fd.name, "error");
    return fd;
}

// first-generation view of a second-generation AXT with con[n] appended (lenCON = n here,
// n + 1 entries there); `ext` owns the copy
str_matAXT gen1_axt(const gs2_matAXT &m, const char *mode, std::vector<UIN> &ext)
{
    str_matAXT v;
    memset(&v, 0, sizeof(v));
    strcpy(v.name, "gen2");
    v.nrows = m.nrows;
    v.nnz = m.nnz;
    snprintf(v.mode, sizeof(v.mode), "%s", mode);
    v.tileHW = m.tileHW;
    v.tileH = m.tileH;
    v.logTH = m.logTH;
    v.tileN = m.tileN;
    v.lenAX = m.lenAX;
    v.lenSEC = m.lenSEC;
    v.lenCON = m.lenCON;
    v.log = m.log;
    v.bs = 1u << m.log;
    v.ax = m.ax;
    v.sec = m.sec;
    ext.assign(m.con, m.con + m.lenCON);
    ext.push_back(m.lenAX);
    v.con = ext.data();
    return v;
}

}  // namespace

extern "C" {

gs2_matCSR gs2_matrixReading(const char *matFileName)
{
    const str_matCSR r = matrixReading(matFileName);
    gs2_matCSR m;
    memset(&m, 0, sizeof(m));
    m.nrows = r.nrows;
    m.nnz = r.nnz;
    m.val = r.val;
    m.row = r.row;
    m.col = r.col;
    m.rl = r.rl;
    return m;
}

void gs2_printMatrixStats(const char *matFileName, gs2_matCSR *m)
{
    str_matCSR v = gen1_view(*m);
    stats_core(matFileName, &v, true);
    m->rmin = v.rmin;
    m->rave = v.rave;
    m->rmax = v.rmax;
    m->rsd = v.rsd;
    m->bw = v.bw;
}

gs2_formatData gs2_getFormatDataCSR(const gs2_matCSR m)
{
    return gen2_fd("CSR",
                   (double)m.nnz * sizeof(FPT) + (double)m.nnz * sizeof(UIN) +
                       ((double)m.nrows + 1) * sizeof(UIN) + (double)m.nrows * sizeof(FPT),
                   (double)m.nnz / (double)m.nnz, 0.0);
}

void gs2_initVec(const UIN len, FPT *vec) { init_vec(1, len, vec); }

void gs2_cf_CSR(const gs2_matCSR m, const FPT *vec, FPT *res) { ncsr(1, gen1_view(m), vec, res); }

void gs2_getErrors(const UIN len, const FPT *ar, const FPT *ac, gs2_err *e)
{
    str_err r;
    get_errors(len, ar, ac, &r);
    e->aErr = r.aErr;
    e->rErr = r.rErr;
    e->pos = r.pos;
}

gs2_res gs2_test_cf_CSR(const gs2_matCSR m, const FPT *vec, const FPT *ref)
{
    return gen2_res(test_gcsr(0, gen1_view(m), vec, ref), "cf_CSR");
}

gs2_res gs2_test_gk_CSR(const UIN cudaBlockSize, const gs2_matCSR m, const FPT *vec,
                        const FPT *ref)
{
    return gen2_res(test_gcsr(cudaBlockSize, gen1_view(m), vec, ref), "gk_CSR");
}

gs2_res gs2_test_gcu_CSR(const gs2_matCSR m, const FPT *vec, const FPT *ref)
{
    return gen2_res(test_gcucsr(gen1_view(m), vec, ref), "gcu_CSR");
}

gs2_formatData gs2_getFormatDataAXC(const UIN ompNumThreads, const gs2_matCSR m,
                                    const FPT *vec, gs2_matAXC *a)
{
    str_matAXC a1;
    memset(&a1, 0, sizeof(a1));
    const str_formatData fd = getFormatDataAXC(ompNumThreads, 32, gen1_view(m), vec, &a1);
    if (!strcmp(fd.name, "error")) return gen2_error_fd();
    free(a1.mapx);
    a->nrows = a1.nrows;
    a->nnz = a1.nnz;
    a->lenAX = a1.lenAX;
    a->lenBRP = a1.lenBRP;
    a->ax = a1.ax;
    a->brp = a1.brp;
    return gen2_fd("AXC", (double)a->lenAX * sizeof(FPT) + (double)a->lenBRP * sizeof(UIN),
                   (double)a->nnz / (double)(a->lenAX >> 1), fd.ct);
}

gs2_res gs2_test_gk_AXC(const UIN cudaBlockSize, const gs2_matAXC a, const FPT *ref)
{
    str_matAXC v;
    memset(&v, 0, sizeof(v));
    v.nrows = a.nrows;
    v.nnz = a.nnz;
    v.hbs = 32;
    v.lenAX = a.lenAX;
    v.lenBRP = a.lenBRP;
    v.ax = a.ax;
    v.brp = a.brp;
    return gen2_res(test_gaxc(cudaBlockSize, v, ref), "gk_AXC");
}

gs2_formatData gs2_getFormatDataK1(const UIN cudaBlockSize, const gs2_matCSR m, const FPT *vec,
                                   gs2_matK1 *k)
{
    str_matK1 k1;
    memset(&k1, 0, sizeof(k1));
    const str_formatData fd = getFormatDataK1(cudaBlockSize, gen1_view(m), vec, &k1);
    if (!strcmp(fd.name, "error")) return gen2_error_fd();
    static_assert(sizeof(str_matK1) == sizeof(gs2_matK1), "K1 structs of both generations");
    memcpy(k, &k1, sizeof(k1));
    return gen2_fd("K1",
                   (double)k->chunkNum * sizeof(UIN) * 2 + (double)k->lenVC * sizeof(FPT) +
                       (double)k->lenVC * sizeof(UIN) + (double)k->chunkNum * 32 * sizeof(UIN) +
                       (double)k->nrows * sizeof(FPT),
                   (double)k->nnz / (double)k->lenVC, fd.ct);
}

gs2_res gs2_test_gk_K1(const UIN cudaBlockSize, const gs2_matK1 k, const FPT *vec,
                       const FPT *ref)
{
    str_matK1 k1;
    memcpy(&k1, &k, sizeof(k1));
    return gen2_res(test_gk1(cudaBlockSize, k1, vec, ref), "gk_K1");
}

gs2_formatData gs2_getFormatDataAXT(const UIN ompNT, const UIN bs, const UIN thw, const UIN th,
                                    const char *mode, const gs2_matCSR m, const FPT *vec,
                                    gs2_matAXT *a)
{
    const bool noc = mode && !strcmp(mode, "NOC"), com = mode && !strcmp(mode, "COM");
    if (!noc && !com) {
        gs::fail(GS_ERR_INVALID, "mode must be \"NOC\" or \"COM\"");
        printf("getFormatDataAXT: mode must be \"NOC\" or \"COM\"\n");
        return gen2_error_fd();
    }
    memset(a, 0, sizeof(*a));
    a->nrows = m.nrows;
    a->nnz = m.nnz;
    snprintf(a->mode, sizeof(a->mode), "%s", mode);
    a->tileHW = thw;
    a->tileH = th;
    for (UIN i = 0; i < 10; i++)
        if ((th >> i) == 1) a->logTH = i;
    if (com)
        for (UIN i = 1; i < 10; i++)
            if ((bs >> i) == 1) {
                a->log = i;
                break;
            }
    a->lenCON = m.nrows;
    double ct = 0.0;
    if (noc || th == 1) {
        str_matAXT t;
        memset(&t, 0, sizeof(t));
        const str_formatData fd =
            getFormatDataAXT(ompNT, bs, thw, th, noc ? "UNC" : "COM", gen1_view(m), vec, &t);
        if (!strcmp(fd.name, "error")) return gen2_error_fd();
        ct = fd.ct;
        a->tileN = t.tileN;
        a->lenAX = t.lenAX;
        a->lenSEC = t.lenSEC;
        a->ax = t.ax;
        a->sec = t.sec;
        a->con = t.con;  // the same values for rows < n (NOC); rebuilt below for COM
    } else {
        // COM with tileH > 1: lengths only, no array filled (gpuSpmv_header.h:1289-1301)
        uint64_t cols = 0;
        for (UIN r = 0; r < m.nrows; r++) cols += (m.row[r + 1] - m.row[r] + th - 1) / th;
        a->tileN = (UIN)((cols + thw - 1) / thw);
        a->lenAX = a->tileN * 2 * thw * th;
        a->lenSEC = a->tileN * thw * th;
        a->ax = (FPT *)calloc(a->lenAX ? a->lenAX : 1, sizeof(FPT));
        a->sec = (UIN *)calloc(a->lenSEC ? a->lenSEC : 1, sizeof(UIN));
    }
    if (com) {
        free(a->con);
        a->con = (UIN *)calloc((size_t)m.nrows + 1, sizeof(UIN));
        DevBuf row, sec, con;
        const bool fill_sec = th == 1;
        gs_status st = h2d(row, m.row, (size_t)m.nrows + 1);
        if (!st && fill_sec) st = sec.alloc_zero((size_t)a->lenSEC * 4, 0);
        if (!st) st = con.alloc(((size_t)m.nrows + 1) * 4);
        if (st) return gen2_error_fd();
        if (m.nrows)
            k_gen2_com<<<(m.nrows + 255) / 256, 256>>>(m.nrows, row.as<UIN>(), thw, th, a->log,
                                                       fill_sec ? sec.as<UIN>() : nullptr,
                                                       con.as<UIN>());
        if (cudaDeviceSynchronize() != cudaSuccess) return gen2_error_fd();
        if (fill_sec && a->lenSEC)
            cudaMemcpy(a->sec, sec.p, (size_t)a->lenSEC * 4, cudaMemcpyDeviceToHost);
        if (m.nrows) cudaMemcpy(a->con, con.p, (size_t)m.nrows * 4, cudaMemcpyDeviceToHost);
    }
    char name[32];
    snprintf(name, sizeof(name), "AXT_%s_H%u_HW%u", mode, th, thw);
    return gen2_fd(name, (double)a->lenAX * sizeof(FPT) + (double)a->lenSEC * sizeof(UIN),
                   (double)a->nnz / (double)(a->lenAX >> 1), ct);
}

gs2_res gs2_test_gk_AXT_NOC_H1(const UIN cudaBlockSize, const gs2_matAXT a, const FPT *ref)
{
    (void)cudaBlockSize;
    char name[24];
    snprintf(name, sizeof(name), "gk_AXT_NOC_H1_HW%u", a.tileHW);
    std::vector<UIN> ext;
    return gen2_res(test_unc1("gk_AXT_NOC_H1", 0, gen1_axt(a, "UNC", ext), ref), name);
}

gs2_res gs2_test_gk_AXT_NOC(const UIN cudaBlockSize, const gs2_matAXT a, const FPT *ref)
{
    char name[24];
    snprintf(name, sizeof(name), "gk_AXT_NOC_H%u_HW%u", a.tileH, a.tileHW);
    std::vector<UIN> ext;
    return gen2_res(test_gaxtuh(0, cudaBlockSize, gen1_axt(a, "UNC", ext), ref), name);
}

gs2_res gs2_test_gk_AXT_COM_H1(const UIN cudaBlockSize, const gs2_matAXT a, const FPT *ref)
{
    (void)cudaBlockSize;
    char name[24];
    snprintf(name, sizeof(name), "gk_AXT_COM_H1_HW%u", a.tileHW);
    if (strcmp(a.mode, "COM") != 0 || a.tileH != 1) {
        gs2_res r;
        memset(&r, 0, sizeof(r));
        strcpy(r.name, "error");
        printf("%s: matrix is not a COM tileH=1 AXT layout\n", name);
        return r;
    }
    DevBuf con, rpos;
    str_res r1;
    if (h2d(con, a.con, a.nrows) || rpos.alloc(((size_t)a.nrows + 1) * 4)) {
        r1 = error_res(name, gs_last_error());
    } else {
        k_gen2_com_rpos<<<(a.nrows + 256) / 256, 256>>>(a.nrows, a.nnz, con.as<UIN>(), a.tileHW,
                                                        rpos.as<UIN>());
        r1 = run_baked(name, a.nrows, a.nnz, a.ax, a.lenAX, rpos, false, a.tileHW, 1, a.tileHW,
                       0, ref);
    }
    return gen2_res(r1, name);
}

}  // extern "C"

// ======================================================================================
// First API generation (spmv_header.h), its brick formats AXCv0, AXCv1, AXBv0 and AXBv1,
// exported as gs0_* (gpuspmv_b200_gen0.h).  Each is a layout the later generation's
// converters already build, with bricks of 16: AXCv0 = AXC hbs 16 (spmv_header.h:665-760),
// AXCv1 = AXT UNC tileH 1 tileHW 16 (brp = con, rwp = sec; :851-960), AXBv0 = AXT COM tileH 1
// tileHW 16 with a header word every 32 positions (hdr0 = sec; :1649-1727), AXBv1 = the same
// every cudaBlockSize positions with hdr1 padded to a multiple of 32 words (:2299-2390).
// ======================================================================================
#define GS0_NO_ALIASES
#include "gpuspmv_b200_gen0.h"

namespace {

constexpr UIN kGen0Brick = 16;  // HBRICK_SIZE of spmv_header.h (spmv_header.h:97-99)

str_matCSR gen1_view0(const gs0_matCSR &m)
{
    str_matCSR v;
    memset(&v, 0, sizeof(v));
    strcpy(v.name, "gen0");
    v.nrows = m.nrows;
    v.nnz = m.nnz;
    v.rmin = m.rmin;
    v.rave = m.rave;
    v.rmax = m.rmax;
    v.rsd = m.rsd;
    v.bw = m.bw;
    v.val = m.val;
    v.row = m.row;
    v.col = m.col;
    v.rl = m.rl;
    return v;
}

gs0_formatData gen0_fd(const char *name, double mfp, double beta, double ct)
{
    gs0_formatData fd;
    memset(&fd, 0, sizeof(fd));
    snprintf(fd.name, sizeof(fd.name), "%s", name);
    fd.mfp = mfp;
    fd.beta = beta;
    fd.ct = ct;
    return fd;
}

gs0_formatData gen0_error_fd()
{
    return gen0_fd("error", 0.0, 0.0, 0.0);
}

gs0_res gen0_res(const str_res &r, const char *name)
{
    gs0_res o;
    memset(&o, 0, sizeof(o));
    snprintf(o.name, sizeof(o.name), "%s", strcmp(r.name, "error") ? name : "error");
    o.et = r.et;
    o.flops = r.flops;
    o.sErr.aErr = r.sErr.aErr;
    o.sErr.rErr = r.sErr.rErr;
    o.sErr.pos = r.sErr.pos;
    return o;
}

// UNC tileH 1 tileHW 16 or COM tileH 1 tileHW 16 (header block bs) of a first-generation
// CSR, through the later generation's converter
str_formatData gen0_axt(const gs0_matCSR &m, const FPT *vec, const char *mode, UIN bs,
                        str_matAXT *t)
{
    memset(t, 0, sizeof(*t));
    return getFormatDataAXT(1, bs, kGen0Brick, 1, mode, gen1_view0(m), vec, t);
}

// first-generation views of the brick formats as later-generation structs, for the products
str_matAXC axc_view(const gs0_matAXCv0 &a)
{
    str_matAXC v;
    memset(&v, 0, sizeof(v));
    v.nrows = a.nrows;
    v.nnz = a.nnz;
    v.hbs = kGen0Brick;
    v.lenAX = a.lenAX;
    v.lenBRP = a.lenBRP;
    v.ax = a.ax;
    v.brp = a.brp;
    return v;
}

str_matAXT unc_view(const gs0_matAXCv1 &a)
{
    str_matAXT v;
    memset(&v, 0, sizeof(v));
    strcpy(v.name, "gen0");
    v.nrows = a.nrows;
    v.nnz = a.nnz;
    strcpy(v.mode, "UNC");
    v.tileHW = kGen0Brick;
    v.tileH = 1;
    v.tileN = a.lenRWP;
    v.lenAX = a.lenAX;
    v.lenSEC = a.lenRWP;
    v.lenCON = a.nrows;
    v.ax = a.ax;
    v.sec = a.rwp;
    v.con = a.brp;  // nrows + 1 entries
    return v;
}

str_matAXT com_view(UIN nrows, UIN nnz, UIN lenAX, UIN *hdr, UIN lenHDR, UIN log, FPT *ax)
{
    str_matAXT v;
    memset(&v, 0, sizeof(v));
    strcpy(v.name, "gen0");
    v.nrows = nrows;
    v.nnz = nnz;
    strcpy(v.mode, "COM");
    v.tileHW = kGen0Brick;
    v.tileH = 1;
    v.tileN = lenAX / (2 * kGen0Brick);
    v.lenAX = lenAX;
    v.lenSEC = lenHDR;
    v.log = log;
    v.bs = 1u << log;
    v.ax = ax;
    v.sec = hdr;
    return v;
}

gs0_res gen0_error_res(const char *name, const char *what)
{
    return gen0_res(error_res(name, what), name);
}

}  // namespace

extern "C" {

gs0_formatData gs0_getFormatDataAXCv0(const UIN numThreads, const gs0_matCSR m, const FPT *vec,
                                      gs0_matAXCv0 *a)
{
    if (!a) return gen0_error_fd();
    memset(a, 0, sizeof(*a));
    str_matAXC a1;
    memset(&a1, 0, sizeof(a1));
    const str_formatData fd = getFormatDataAXC(numThreads, kGen0Brick, gen1_view0(m), vec, &a1);
    if (!strcmp(fd.name, "error")) return gen0_error_fd();
    free(a1.mapx);
    a->nrows = a1.nrows;
    a->nnz = a1.nnz;
    a->lenAX = a1.lenAX;
    a->lenBRP = a1.lenBRP;
    a->ax = a1.ax;
    a->brp = a1.brp;
    // spmv_header.h:748-751
    return gen0_fd("AXCv0", (double)((size_t)a->lenAX * sizeof(FPT)) +
                               (double)((size_t)a->lenBRP * sizeof(UIN)),
                   (double)a->nnz / (double)(a->lenAX >> 1), fd.ct);
}

gs0_formatData gs0_getFormatDataAXCv1(const UIN numThreads, const gs0_matCSR m, const FPT *vec,
                                      gs0_matAXCv1 *a)
{
    (void)numThreads;
    if (!a) return gen0_error_fd();
    memset(a, 0, sizeof(*a));
    str_matAXT t;
    const str_formatData fd = gen0_axt(m, vec, "UNC", 256, &t);
    if (!strcmp(fd.name, "error")) return gen0_error_fd();
    a->nrows = t.nrows;
    a->nnz = t.nnz;
    a->lenAX = t.lenAX;
    a->lenBRP = t.nrows + 1;
    a->lenRWP = t.lenSEC;
    a->ax = t.ax;
    a->brp = t.con;
    a->rwp = t.sec;
    // spmv_header.h:965-968
    return gen0_fd("AXCv1", (double)((size_t)a->lenAX * sizeof(FPT)) +
                               (double)((size_t)a->lenRWP * sizeof(UIN)),
                   (double)a->nnz / (double)(a->lenAX >> 1), fd.ct);
}

gs0_formatData gs0_getFormatDataAXBv0(const gs0_matCSR m, const FPT *vec, gs0_matAXBv0 *a)
{
    if (!a) return gen0_error_fd();
    memset(a, 0, sizeof(*a));
    str_matAXT t;
    const str_formatData fd = gen0_axt(m, vec, "COM", 32, &t);
    if (!strcmp(fd.name, "error")) return gen0_error_fd();
    free(t.con);
    a->nrows = t.nrows;
    a->nnz = t.nnz;
    a->brickNum = t.tileN;
    a->lenAX = t.lenAX;
    a->lenHDR = t.lenSEC;
    a->ax = t.ax;
    a->hdr0 = t.sec;
    // spmv_header.h:1718-1721
    return gen0_fd("AXBv0", (double)((size_t)a->lenAX * sizeof(FPT)) +
                               (double)((size_t)a->lenHDR * sizeof(UIN)),
                   (double)a->nnz / (double)(a->lenAX >> 1), fd.ct);
}

gs0_formatData gs0_getFormatDataAXBv1(const UIN cudaBlockSize, const gs0_matCSR m,
                                      const FPT *vec, gs0_matAXBv1 *a)
{
    if (!a) return gen0_error_fd();
    memset(a, 0, sizeof(*a));
    UIN log = 0;
    for (UIN i = 5; i < 11; i++)
        if ((cudaBlockSize >> i) == 1) log = i;
    if (log == 0 || cudaBlockSize != (1u << log)) {
        gs::fail(GS_ERR_UNSUPPORTED, "AXBv1 takes a cudaBlockSize that is a power of two in "
                                     "32..1024 (got %u)", cudaBlockSize);
        return gen0_fd("error", 0.0, 0.0, 0.0);
    }
    str_matAXT t;
    const str_formatData fd = gen0_axt(m, vec, "COM", cudaBlockSize, &t);
    if (!strcmp(fd.name, "error")) return gen0_error_fd();
    free(t.con);
    // hdr1: the header words, padded with zeros to a multiple of 32 (spmv_header.h:2350)
    const size_t len = ((size_t)t.lenAX / 2 + 2 * kGen0Brick - 1) / (2 * kGen0Brick) *
                       (2 * kGen0Brick);
    UIN *hdr = static_cast<UIN *>(calloc(len ? len : 1, sizeof(UIN)));
    if (!hdr) {
        free(t.ax);
        free(t.sec);
        gs::fail(GS_ERR_ALLOC, "AXBv1 header allocation");
        return gen0_error_fd();
    }
    if (t.lenSEC) memcpy(hdr, t.sec, (size_t)t.lenSEC * sizeof(UIN));
    free(t.sec);
    a->nrows = t.nrows;
    a->nnz = t.nnz;
    a->brickNum = t.tileN;
    a->lenAX = t.lenAX;
    a->lenHDR = (UIN)len;
    a->blockLog = log;
    a->ax = t.ax;
    a->hdr1 = hdr;
    // spmv_header.h:2379-2382
    return gen0_fd("AXBv1", (double)((size_t)a->lenAX * sizeof(FPT)) +
                               (double)((size_t)a->lenHDR * sizeof(UIN)),
                   (double)a->nnz / (double)(a->lenAX >> 1), fd.ct);
}

gs0_res gs0_testGpuSpmvAXCv0(const UIN cudaBlockSize, const gs0_matAXCv0 a, const FPT *ref)
{
    return gen0_res(test_gaxc(cudaBlockSize, axc_view(a), ref), "gk_AXCv0");
}

static gs0_res axcv1(const char *name, const gs0_matAXCv1 &a, const FPT *ref)
{
    if (a.lenBRP != a.nrows + 1) return gen0_error_res(name, "lenBRP must be nrows + 1");
    return gen0_res(test_gaxtuh1hw16w(0, 0, unc_view(a), ref), name);
}
gs0_res gs0_testGpuSpmvAXCv1_0(const UIN c, const gs0_matAXCv1 a, const FPT *r)
{
    (void)c;
    return axcv1("gk_AXCv1_0", a, r);
}
gs0_res gs0_testGpuSpmvAXCv1_1(const UIN c, const gs0_matAXCv1 a, const FPT *r)
{
    (void)c;
    return axcv1("gk_AXCv1_1", a, r);
}
gs0_res gs0_testGpuSpmvAXCv1_2(const UIN c, const gs0_matAXCv1 a, const FPT *r)
{
    (void)c;
    return axcv1("gk_AXCv1_2", a, r);
}
gs0_res gs0_testGpuSpmvAXCv1_3(const UIN c, const gs0_matAXCv1 a, const FPT *r)
{
    (void)c;
    return axcv1("gk_AXCv1_3", a, r);
}
gs0_res gs0_testGpuSpmvAXCv1_4(const UIN c, const gs0_matAXCv1 a, const FPT *r)
{
    (void)c;
    return axcv1("gk_AXCv1_4", a, r);
}

static gs0_res axb(const char *name, UIN nrows, UIN nnz, UIN lenAX, UIN *hdr, UIN lenHDR,
                   UIN log, FPT *ax, const FPT *ref)
{
    if (lenHDR < lenAX / 2) return gen0_error_res(name, "header array shorter than lenAX / 2");
    return gen0_res(test_gaxtch1(0, com_view(nrows, nnz, lenAX, hdr, lenAX / 2, log, ax), ref),
                    name);
}
gs0_res gs0_testGpuSpmvAXBv0_0(const UIN c, const gs0_matAXBv0 a, const FPT *r)
{
    (void)c;
    return axb("gk_AXBv0_0", a.nrows, a.nnz, a.lenAX, a.hdr0, a.lenHDR, 5, a.ax, r);
}
gs0_res gs0_testGpuSpmvAXBv0_1(const UIN c, const gs0_matAXBv0 a, const FPT *r)
{
    (void)c;
    return axb("gk_AXBv0_1", a.nrows, a.nnz, a.lenAX, a.hdr0, a.lenHDR, 5, a.ax, r);
}
gs0_res gs0_testGpuSpmvAXBv0_2(const UIN c, const gs0_matAXBv0 a, const FPT *r)
{
    (void)c;
    return axb("gk_AXBv0_2", a.nrows, a.nnz, a.lenAX, a.hdr0, a.lenHDR, 5, a.ax, r);
}
gs0_res gs0_testGpuSpmvAXBv0_3(const UIN c, const gs0_matAXBv0 a, const FPT *r)
{
    (void)c;
    return axb("gk_AXBv0_3", a.nrows, a.nnz, a.lenAX, a.hdr0, a.lenHDR, 5, a.ax, r);
}
gs0_res gs0_testGpuSpmvAXBv1_0(const UIN c, const gs0_matAXBv1 a, const FPT *r)
{
    (void)c;
    if (a.blockLog < 5 || a.blockLog > 10)
        return gen0_error_res("gk_AXBv1_0", "blockLog must be 5..10");
    return axb("gk_AXBv1_0", a.nrows, a.nnz, a.lenAX, a.hdr1, a.lenHDR, a.blockLog, a.ax, r);
}

}  // extern "C"
