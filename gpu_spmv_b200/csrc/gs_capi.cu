// gs_capi.cu -- the native C ABI (gs_*): matrix handles, SpMV dispatch, status strings.
#include <cstdio>
#include <cstring>
#include <new>

#include "gs_internal.cuh"

namespace gs {
const char *last_error_text();
}

namespace {
UIN g_num_ite = 250;  // cudaSpmv.cu:96-98
}

extern "C" {

const char *gs_status_string(gs_status s)
{
    switch (s) {
    case GS_OK: return "GS_OK";
    case GS_ERR_INVALID: return "GS_ERR_INVALID";
    case GS_ERR_CUDA: return "GS_ERR_CUDA";
    case GS_ERR_ALLOC: return "GS_ERR_ALLOC";
    case GS_ERR_OVERFLOW: return "GS_ERR_OVERFLOW";
    case GS_ERR_UNSUPPORTED: return "GS_ERR_UNSUPPORTED";
    case GS_ERR_DEVICE: return "GS_ERR_DEVICE";
    default: return "GS_ERR_UNKNOWN";
    }
}

const char *gs_last_error(void) { return gs::last_error_text(); }

const char *gs_version(void) { return "gpuspmv_b200 1.0 (sm_100a)"; }

void gs_set_num_ite(UIN n) { g_num_ite = n ? n : 1; }
UIN gs_get_num_ite(void) { return g_num_ite; }

double gs_algorithmic_bytes(UIN nrows, UIN ncols, UIN nnz, UIN k, UIN s_v, UIN s_i, UIN s_x,
                            UIN s_y)
{
    return (double)nnz * (s_v + s_i) + 4.0 * ((double)nrows + 1) + (double)s_x * ncols * k +
           (double)s_y * nrows * k;
}

gs_status gs_matrix_create(gs_matrix **out, const gs_convert_params *params, UIN nrows,
                           UIN ncols, UIN nnz, const UIN *d_row, const UIN *d_col,
                           const void *d_val, gs_dtype val_type, gs_stream stream)
{
    gs::clear_error();
    if (!out || !params) return gs::fail(GS_ERR_INVALID, "NULL argument");
    *out = nullptr;
    gs_matrix *A = new (std::nothrow) gs_matrix();
    if (!A) return gs::fail(GS_ERR_ALLOC, "host allocation failed");
    gs_status st = gs::convert(A, *params, nrows, ncols, nnz, d_row, d_col, d_val, val_type,
                               nullptr, nullptr, gs::cs(stream));
    if (st != GS_OK) {
        cudaStreamSynchronize(gs::cs(stream));
        delete A;
        return st;
    }
    *out = A;
    return GS_OK;
}

gs_status gs_matrix_create_host(gs_matrix **out, const gs_convert_params *params, UIN nrows,
                                UIN ncols, UIN nnz, const UIN *h_row, const UIN *h_col,
                                const void *h_val, gs_dtype val_type, gs_stream stream)
{
    gs::clear_error();
    if (!out || !params || !h_row || (nnz && (!h_col || !h_val)))
        return gs::fail(GS_ERR_INVALID, "NULL argument");
    if (val_type != GS_F64 && val_type != GS_F32)
        return gs::fail(GS_ERR_UNSUPPORTED, "input CSR values must be FP64 or FP32");
    *out = nullptr;
    gs::DevBuf row, col, val;
    const size_t vsz = gs::dtype_size(val_type);
    GS_TRY(row.alloc(((size_t)nrows + 1) * 4));
    GS_TRY(col.alloc((size_t)nnz * 4));
    GS_TRY(val.alloc((size_t)nnz * vsz));
    cudaStream_t s = gs::cs(stream);
    GS_CUDA(cudaMemcpyAsync(row.p, h_row, ((size_t)nrows + 1) * 4, cudaMemcpyHostToDevice, s));
    if (nnz) {
        GS_CUDA(cudaMemcpyAsync(col.p, h_col, (size_t)nnz * 4, cudaMemcpyHostToDevice, s));
        GS_CUDA(cudaMemcpyAsync(val.p, h_val, (size_t)nnz * vsz, cudaMemcpyHostToDevice, s));
    }
    // the conversion synchronises before returning, so the staging buffers may go
    return gs_matrix_create(out, params, nrows, ncols, nnz, row.as<UIN>(), col.as<UIN>(),
                            val.p, val_type, stream);
}

gs_status gs_matrix_destroy(gs_matrix *A)
{
    if (A) {
        cudaDeviceSynchronize();  // no kernel may still read the buffers
        delete A;
    }
    return GS_OK;
}

gs_status gs_matrix_get_info(const gs_matrix *A, gs_matrix_info *i)
{
    if (!A || !i) return gs::fail(GS_ERR_INVALID, "NULL argument");
    memset(i, 0, sizeof(*i));
    i->format = A->p.format;
    i->nrows = A->nrows;
    i->ncols = A->ncols;
    i->nnz = A->nnz;
    i->tileHW = A->tileHW;
    i->tileH = A->tileH;
    i->logTH = A->logTH;
    i->tileN = A->tileN;
    i->lenAX = A->lenAX;
    i->lenSEC = A->lenSEC;
    i->lenCON = A->lenCON;
    i->log = A->log;
    i->bs = A->bs;
    i->mode = A->p.mode;
    i->hbs = A->hbs;
    i->lenBRP = A->lenBRP;
    i->lenMAPX = A->lenMAPX;
    i->chunkNum = A->chunkNum;
    i->lenVC = A->lenVC;
    i->nslots = A->nslots;
    i->vtype = A->p.vtype;
    i->itype = A->p.itype;
    i->d_val = A->val.p;
    i->d_col = A->col.p;
    i->d_colbase = A->colbase.as<UIN>();
    i->d_sec = A->sec.as<UIN>();
    i->d_con = A->con.as<UIN>();
    i->d_brp = A->brp.as<UIN>();
    i->d_mapx = A->mapx.as<UIN>();
    i->d_permi = A->permi.as<UIN>();
    i->d_nmc = A->nmc.as<UIN>();
    i->d_chp = A->chp.as<UIN>();
    i->d_rpos = A->rpos.as<UIN>();
    i->d_rlen = A->rlen.as<UIN>();
    i->conv_ms = A->conv_ms;
    i->mfp = A->mfp;
    i->beta = A->beta;
    i->lane_positions = (A->p.format == GS_FMT_K1 || A->tile_w) ? 0u : A->plan.V;
    i->tiles_per_step = 0;
    if (A->tiled && A->plan.aligned && A->p.tileHW == 32 && (A->p.tileH == 2 || A->p.tileH == 4))
        i->tiles_per_step = A->plan.grouped ? 2u : 1u;
    return GS_OK;
}

gs_status gs_spmv(const gs_matrix *A, const void *d_x, gs_dtype xtype, void *d_y,
                  gs_dtype ytype, UIN flags, gs_stream stream)
{
    if (!A || !d_x || !d_y) return gs::fail(GS_ERR_INVALID, "NULL argument");
    cudaStream_t s = gs::cs(stream);
    if (A->p.format == GS_FMT_K1) {
        const bool f64 = A->p.vtype == GS_F64;
        if (xtype != (f64 ? GS_F64 : GS_F32))
            return gs::fail(GS_ERR_UNSUPPORTED, f64 ? "FP64 matrices take FP64 x"
                                                    : "FP32/BF16 matrices take FP32 x");
        gs::K1Args a{};
        a.nrows = A->nrows;
        a.chunkNum = A->chunkNum;
        a.permi = A->permi.as<uint32_t>();
        a.nmc = A->nmc.as<uint32_t>();
        a.chp = A->chp.as<uint32_t>();
        a.klen = A->k1len.as<uint32_t>();
        a.val = A->val.p;
        a.col = A->col.p;
        a.ck = A->k1ck.as<uint32_t>();
        a.x = d_x;
        a.y = d_y;
        a.unit_chunk = A->k1unit_chunk.as<uint32_t>();
        a.unit_base = A->k1unit_base.as<uint32_t>();
        a.units = A->k1units;
        a.partial = A->k1partial.as<double>();
        a.count = A->k1count.as<uint32_t>();
        return gs::launch_k1(a, A->p.vtype, A->p.itype, ytype, (flags & GS_FLAG_ACC_F64) != 0,
                             s);
    }
    const bool f64 = A->p.vtype == GS_F64;
    if (f64 && xtype != GS_F64) return gs::fail(GS_ERR_UNSUPPORTED, "FP64 matrices take FP64 x");
    if (!f64 && xtype != GS_F32)
        return gs::fail(GS_ERR_UNSUPPORTED, "FP32/BF16 matrices take FP32 x");
    if (A->tile_w && f64 && ytype == GS_F64 && !(flags & (GS_FLAG_STRIPED | GS_FLAG_TMA))) {
        // whole tiles per row (UNC tileH = 1, AXC): the tile kernel over the tile plan
        gs::RowsArgs t = gs::rows_args(A->tplan);
        t.val = A->val.p;
        t.col = A->col.p;
        t.x = d_x;
        t.y = d_y;
        t.rbits = A->plan.padded ? A->plan.rbits.as<uint32_t>() : nullptr;
        return gs::launch_tiles(t, A->tile_w, false, s);
    }
    gs::RowsArgs a = gs::rows_args(A->plan);
    a.val = A->val.p;
    a.col = A->col.p;
    a.x = d_x;
    a.y = d_y;
    if (A->tiled) {
        a.thw = A->tileHW;
        a.th = A->tileH;
    }
    a.nslots = A->nslots;
    return gs::launch_rows(a, A->p.vtype, A->p.itype, ytype, flags, A->tiled != 0, false,
                           A->plan.padded, s);
}

gs_status gs_spmv_host(const gs_matrix *A, const void *h_x, void *d_xbuf, gs_dtype xtype,
                       void *h_y, void *d_ybuf, gs_dtype ytype, UIN flags, gs_stream stream)
{
    if (!A || !h_x || !h_y || !d_xbuf || !d_ybuf)
        return gs::fail(GS_ERR_INVALID, "NULL argument");
    cudaStream_t s = gs::cs(stream);
    GS_CUDA(cudaMemcpyAsync(d_xbuf, h_x, (size_t)A->ncols * gs::dtype_size(xtype),
                            cudaMemcpyHostToDevice, s));
    GS_TRY(gs_spmv(A, d_xbuf, xtype, d_ybuf, ytype, flags, stream));
    GS_CUDA(cudaMemcpyAsync(h_y, d_ybuf, (size_t)A->nrows * gs::dtype_size(ytype),
                            cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    return GS_OK;
}

gs_status gs_spmv_host_stream(const gs_matrix *Ac, const void *h_x, size_t x_stride,
                              gs_dtype xtype, void *h_y, size_t y_stride, gs_dtype ytype,
                              UIN count, UIN flags, gs_stream stream)
{
    if (!Ac || (count && (!h_x || !h_y))) return gs::fail(GS_ERR_INVALID, "NULL argument");
    if (!count) return GS_OK;
    gs_matrix *A = const_cast<gs_matrix *>(Ac);  // the pipeline is a cache of the handle
    HostPipe &P = A->pipe;
    const size_t xb = (size_t)A->ncols * gs::dtype_size(xtype);
    const size_t yb = (size_t)A->nrows * gs::dtype_size(ytype);
    if (!P.ready || P.x[0].bytes < xb || P.y[0].bytes < yb) {
        if (!P.in) {
            GS_CUDA(cudaStreamCreateWithFlags(&P.in, cudaStreamNonBlocking));
            GS_CUDA(cudaStreamCreateWithFlags(&P.out, cudaStreamNonBlocking));
            for (int b = 0; b < 2; b++) {
                GS_CUDA(cudaEventCreateWithFlags(&P.xready[b], cudaEventDisableTiming));
                GS_CUDA(cudaEventCreateWithFlags(&P.kdone[b], cudaEventDisableTiming));
                GS_CUDA(cudaEventCreateWithFlags(&P.ydone[b], cudaEventDisableTiming));
            }
        }
        for (int b = 0; b < 2; b++) {
            GS_TRY(P.x[b].alloc(xb));
            GS_TRY(P.y[b].alloc(yb));
        }
        P.ready = true;
    }
    cudaStream_t s = gs::cs(stream);
    const char *hx = static_cast<const char *>(h_x);
    char *hy = static_cast<char *>(h_y);
    const size_t xs = x_stride * gs::dtype_size(xtype), ys = y_stride * gs::dtype_size(ytype);
    // the first uses of each buffer wait for nothing earlier on the compute stream
    GS_CUDA(cudaEventRecord(P.kdone[0], s));
    GS_CUDA(cudaEventRecord(P.kdone[1], s));
    GS_CUDA(cudaEventRecord(P.ydone[0], s));
    GS_CUDA(cudaEventRecord(P.ydone[1], s));
    for (UIN k = 0; k < count; k++) {
        const int b = (int)(k & 1u);
        // in: x_k into buffer b once product k-2 (the last reader of b) is done
        GS_CUDA(cudaStreamWaitEvent(P.in, P.kdone[b], 0));
        GS_CUDA(cudaMemcpyAsync(P.x[b].p, hx + (size_t)k * xs, xb, cudaMemcpyHostToDevice, P.in));
        GS_CUDA(cudaEventRecord(P.xready[b], P.in));
        // compute: product k once x_k is in and y_{k-2} is out of buffer b
        GS_CUDA(cudaStreamWaitEvent(s, P.xready[b], 0));
        GS_CUDA(cudaStreamWaitEvent(s, P.ydone[b], 0));
        GS_TRY(gs_spmv(A, P.x[b].p, xtype, P.y[b].p, ytype, flags, stream));
        GS_CUDA(cudaEventRecord(P.kdone[b], s));
        // out: y_k to the host
        GS_CUDA(cudaStreamWaitEvent(P.out, P.kdone[b], 0));
        GS_CUDA(cudaMemcpyAsync(hy + (size_t)k * ys, P.y[b].p, yb, cudaMemcpyDeviceToHost, P.out));
        GS_CUDA(cudaEventRecord(P.ydone[b], P.out));
    }
    GS_CUDA(cudaStreamSynchronize(P.out));
    GS_CUDA(cudaStreamSynchronize(s));
    return GS_OK;
}

gs_status gs_matrix_device_status(const gs_matrix *A, UIN *word, int reset)
{
    if (!A || !word) return gs::fail(GS_ERR_INVALID, "NULL argument");
    *word = 0;
    if (!A->plan.status.p) return GS_OK;
    GS_CUDA(cudaDeviceSynchronize());
    GS_CUDA(cudaMemcpy(word, A->plan.status.p, 4, cudaMemcpyDeviceToHost));
    if (reset) GS_CUDA(cudaMemset(A->plan.status.p, 0, 4));
    return GS_OK;
}

gs_status gs_copy_to_host(void *h_dst, const void *d_src, size_t bytes)
{
    if (!bytes) return GS_OK;
    if (!h_dst || !d_src) return gs::fail(GS_ERR_INVALID, "NULL argument");
    GS_CUDA(cudaMemcpy(h_dst, d_src, bytes, cudaMemcpyDeviceToHost));
    return GS_OK;
}

gs_status gs_csr_spmv_f64(UIN nrows, UIN ncols, UIN nnz, const UIN *d_row, const UIN *d_col,
                          const double *d_val, const double *d_x, double *d_y,
                          gs_stream stream)
{
    (void)ncols;
    if (nrows == 0) return GS_OK;
    if (!d_row || !d_x || !d_y || (nnz && (!d_col || !d_val)))
        return gs::fail(GS_ERR_INVALID, "NULL argument");
    if ((reinterpret_cast<uintptr_t>(d_val) & 15u) || (reinterpret_cast<uintptr_t>(d_col) & 15u))
        return gs::fail(GS_ERR_INVALID, "val and col must be 16-byte aligned");
    cudaStream_t s = gs::cs(stream);
    gs::RowsPlan P;
    uint32_t V = gs::kDirectV;
    GS_TRY(gs::direct_lane_positions(d_row, d_col, nrows, nnz, &V, s));
    GS_TRY(gs::build_rows_plan(d_row, nullptr, nrows, V, P, s));
    gs::RowsArgs a = gs::rows_args(P);
    a.val = d_val;
    a.col = d_col;
    a.x = d_x;
    a.y = d_y;
    a.nslots = nnz;
    GS_TRY(gs::launch_rows(a, GS_F64, GS_IDX_U32, GS_F64, 0, false, false, false, s));
    GS_CUDA(cudaStreamSynchronize(s));  // the plan's buffers are released on return
    return GS_OK;
}

}  // extern "C"
