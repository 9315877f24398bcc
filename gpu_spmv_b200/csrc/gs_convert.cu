// gs_convert.cu -- CSR -> CSR / K1 / AXC / AXT conversion on the device.
//
// The layouts are the reference's, bit for bit:
//   K1   getFormatDataK1   cudaSpmv.cu:782-846  (permi 723-737, nmc/chp 741-754,
//                                                 val/col scatter 758-778)
//   AXC  getFormatDataAXC  cudaSpmv.cu:1004-1062 (brp 937-948, ax 952-979, mapx 983-999)
//   AXT  getFormatDataAXT  cudaSpmv.cu:1391-1566 (lengths/con 1158-1235,
//                                                 ax/sec 1239-1387)
// but they are produced with device scans (row offsets), a stable device radix sort (K1
// permutation) and one warp-per-row scatter pass, instead of the reference's serial host
// loops.  Each element's destination is computed in closed form from its row's offset:
//   UNC tileH=1 : slot = rowfirst + e                      (rowfirst = con[r]/2)
//   UNC tileH>1 : column C = C_r + e/th, tile row e%th     (C_r from the column scan)
//   COM         : element p of the CSR stream, slot p (tileH=1) or transposed in its tile
//   AXC         : slot = brp[r]/2 + e
// and slot s is the value half ax[(s/w)*2w + s%w] (x half w further) of the reference's
// interleaved array, w = tileHW or hbs.
//
// The engine stores value and column streams in slot order (its native form: x is
// gathered at SpMV time), plus the reference's metadata on request, plus -- for the
// drop-in converters -- the reference's x-baked ax.
#include <cstdio>
#include <cstring>

#include "gs_internal.cuh"

namespace gs {

namespace {

enum FillLayout : int { kDirect = 0, kUncTiled = 1, kCom = 2 };
enum SecMode : int { kSecNone = 0, kSecTile = 1, kSecColumn = 2, kSecHeader = 3 };

struct FillArgs {
    uint32_t n;
    const uint32_t *row, *col;
    const void *val;
    const uint32_t *rpos;
    int layout, sec_mode;
    uint32_t thw, th, bs, log;
    uint32_t *sec;
    void *oval;
    uint32_t *ocol;
    uint32_t *mapx;
    const double *xbake;
    double *ax;
    uint32_t axw;
};

template <class VIN, class VOUT> __device__ __forceinline__ VOUT cvt(VIN v);
template <> __device__ __forceinline__ double cvt<double, double>(double v) { return v; }
template <> __device__ __forceinline__ float cvt<double, float>(double v) { return __double2float_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 cvt<double, __nv_bfloat16>(double v) { return __double2bfloat16(v); }
template <> __device__ __forceinline__ double cvt<float, double>(float v) { return (double)v; }
template <> __device__ __forceinline__ float cvt<float, float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 cvt<float, __nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

template <class VIN, class VOUT>
__global__ void __launch_bounds__(256) k_fill(const FillArgs f)
{
    const int lane = threadIdx.x & 31;
    const uint32_t ths = f.thw * f.th;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const VIN *val = static_cast<const VIN *>(f.val);
    VOUT *oval = static_cast<VOUT *>(f.oval);
    uint32_t *ocol = f.ocol;
    for (uint32_t r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < f.n; r += warps) {
        const uint32_t b = f.row[r], len = f.row[r + 1] - b;
        for (uint32_t e = lane; e < len; e += 32) {
            const uint32_t p = b + e;
            const VIN v = val[p];
            const uint32_t c = f.col[p];
            uint32_t slot, C = 0, fr = 0;
            if (f.layout == kDirect) {
                slot = f.rpos[r] + e;
            } else if (f.layout == kUncTiled) {
                const uint32_t P = f.rpos[r] + e;  // rpos = th * (first tile column of r)
                C = P / f.th;
                fr = P - C * f.th;
                slot = (C / f.thw) * ths + fr * f.thw + C % f.thw;
            } else {
                if (f.th == 1) {
                    slot = p;
                } else {
                    const uint32_t t = p / ths, rem = p - t * ths, cc = rem / f.th;
                    slot = t * ths + (rem - cc * f.th) * f.thw + cc;
                }
            }
            if (oval) oval[slot] = cvt<VIN, VOUT>(v);
            if (ocol) ocol[slot] = c;
            if (f.sec_mode == kSecTile) {
                if (e % f.thw == 0) f.sec[slot / f.thw] = r;
            } else if (f.sec_mode == kSecColumn) {
                if (fr == 0) f.sec[(C / f.thw) * f.thw + C % f.thw] = r;
            } else if (f.sec_mode == kSecHeader) {
                const uint32_t fp = (f.th == 1) ? p % f.bs : p % f.th;
                const uint32_t lim = (f.th == 1) ? f.bs - 1 - fp : f.th - 1 - fp;
                if (e == 0 || fp == 0) {
                    const uint32_t q1 = len - e - 1;
                    f.sec[slot] = (r << f.log) | (q1 > lim ? lim : q1);
                }
            }
            if (f.mapx) f.mapx[slot] = c;
            if (f.ax) {
                const uint32_t ai = (slot / f.axw) * 2u * f.axw + slot % f.axw;
                f.ax[ai] = (double)v;
                f.ax[ai + f.axw] = f.xbake[c];
            }
        }
    }
}

// one warp per K1 work unit (a kK1Split-step piece of a 32-row chunk), lane = sorted row
// g of the chunk: its elements e of the piece -> k1_slot(chp[c], nmc[c], e, g % 32); a chunk
// of long rows is filled by as many warps as it has pieces
template <class VIN, class VOUT>
__global__ void k_fill_k1(uint32_t n, uint32_t units, const uint32_t *unit_chunk,
                          const uint32_t *unit_base, const uint32_t *row, const uint32_t *col,
                          const VIN *val, const uint32_t *permi, const uint32_t *chp,
                          const uint32_t *nmc, bool blocked, VOUT *oval, uint32_t *ocol)
{
    const uint32_t u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31u;
    if (u >= units) return;
    const uint32_t c = unit_chunk[u], j0 = (u - unit_base[c]) * kK1Split;
    const uint32_t g = 32u * c + lane;
    if (g >= n) return;
    const uint32_t r = permi[g], b = row[r], len = row[r + 1] - b;
    const uint32_t cb = chp[c], m = nmc[c], j1 = min(len, j0 + kK1Split);
    for (uint32_t e = j0; e < j1; e++) {
        const uint32_t pos = k1_slot(cb, m, e, lane, blocked);
        oval[pos] = cvt<VIN, VOUT>(val[b + e]);
        ocol[pos] = col[b + e];
    }
}

template <class VIN>
void launch_fill_k1(uint32_t n, uint32_t units, const uint32_t *unit_chunk,
                    const uint32_t *unit_base, const uint32_t *row, const uint32_t *col,
                    const VIN *val, const uint32_t *permi, const uint32_t *chp,
                    const uint32_t *nmc, bool blocked, gs_dtype vout, void *oval, uint32_t *ocol,
                    cudaStream_t s)
{
    if (!units) return;
    const unsigned b = (units + 7) / 8;
    if (vout == GS_F64)
        k_fill_k1<VIN, double><<<b, 256, 0, s>>>(n, units, unit_chunk, unit_base, row, col, val,
                                                 permi, chp, nmc, blocked,
                                                 static_cast<double *>(oval), ocol);
    else if (vout == GS_F32)
        k_fill_k1<VIN, float><<<b, 256, 0, s>>>(n, units, unit_chunk, unit_base, row, col, val,
                                                permi, chp, nmc, blocked,
                                                static_cast<float *>(oval), ocol);
    else
        k_fill_k1<VIN, __nv_bfloat16><<<b, 256, 0, s>>>(n, units, unit_chunk, unit_base, row,
                                                        col, val, permi, chp, nmc, blocked,
                                                        static_cast<__nv_bfloat16 *>(oval),
                                                        ocol);
}

// first tile of each row (and the tile count at [n]): rpos / w
__global__ void k_tile_starts(uint32_t n1, const uint32_t *rpos, uint32_t w, uint32_t *rt)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n1) rt[i] = rpos[i] / w;
}

__global__ void k_rowlen(uint32_t n, const uint32_t *row, uint32_t *rl)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rl[i] = row[i + 1] - row[i];
}

// tables from a 64-bit exclusive prefix P[0..n]:
//   mode 0 (UNC tileH=1): con = 2*w*P (r <= n), rpos = w*P
//   mode 1 (UNC tileH>1): con = (P/thw)*2*ths + P%thw (r < n), rpos = th*P (r <= n)
//   mode 2 (AXC)        : brp = 2*w*P (r <= n), rpos = w*P
__global__ void k_tables(uint32_t n, const uint64_t *P, int mode, uint32_t w, uint32_t thw,
                         uint32_t th, uint32_t *con, uint32_t *rpos)
{
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > n) return;
    const uint64_t p = P[r];
    if (mode == 0 || mode == 2) {
        if (con) con[r] = (uint32_t)(2ull * w * p);
        rpos[r] = (uint32_t)(w * p);
    } else {
        const uint64_t ths = (uint64_t)thw * th;
        if (con && r < n) con[r] = (uint32_t)((p / thw) * 2ull * ths + p % thw);
        rpos[r] = (uint32_t)(th * p);
    }
}

__global__ void k_k1_meta(uint32_t n, uint32_t chunkNum, const uint32_t *rl,
                          const uint32_t *permi, uint32_t *nmc, uint32_t *klen)
{
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n) {
        uint32_t l = rl[permi[g]];
        klen[g] = l;
        if ((g & 31) == 0) nmc[g >> 5] = l;
    }
}

__global__ void k_u64_to_u32(uint32_t n, const uint64_t *a, uint32_t *b)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (uint32_t)a[i];
}

// bit 0: row pointer not monotone / row[0] != 0 / row[n] != nnz; bit 1: column >= ncols
__global__ void k_validate(uint32_t n, uint32_t ncols, uint32_t nnz, const uint32_t *row,
                           const uint32_t *col, uint32_t *flag)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t bad = 0;
    if (i < n && row[i] > row[i + 1]) bad |= 1u;
    if (i == 0 && (row[0] != 0 || row[n] != nnz)) bad |= 1u;
    for (uint32_t p = i; p < nnz; p += gridDim.x * blockDim.x)
        if (col[p] >= ncols) { bad |= 2u; break; }
    if (bad) atomicOr(flag, bad);
}

inline unsigned blocks_for(uint64_t n, unsigned t = 256) { return (unsigned)((n + t - 1) / t); }

uint32_t ref_log_loop(uint32_t v, uint32_t from, uint32_t to_excl)
{
    for (uint32_t i = from; i < to_excl; i++)
        if ((v >> i) == 1) return i;
    return 0;
}

template <class VIN>
gs_status launch_fill(const FillArgs &f, gs_dtype vout, cudaStream_t s)
{
    const uint64_t want = ((uint64_t)f.n + 7) / 8;
    unsigned blocks = (unsigned)(want < 148u * 64u ? want : 148u * 64u);
    if (blocks == 0) return GS_OK;
    if (vout == GS_F64) k_fill<VIN, double><<<blocks, 256, 0, s>>>(f);
    else if (vout == GS_F32) k_fill<VIN, float><<<blocks, 256, 0, s>>>(f);
    else k_fill<VIN, __nv_bfloat16><<<blocks, 256, 0, s>>>(f);
    GS_CHECK_LAUNCH();
    return GS_OK;
}

}  // namespace

gs_status convert(gs_matrix *A, const gs_convert_params &p, uint32_t n, uint32_t ncols,
                  uint32_t nnz, const uint32_t *d_row, const uint32_t *d_col,
                  const void *d_val, gs_dtype val_type, const double *d_xbake,
                  DevBuf *ax_out, cudaStream_t s)
{
    if (n == 0) return fail(GS_ERR_INVALID, "matrix has no rows");
    if (!d_row || (nnz && (!d_col || !d_val)))
        return fail(GS_ERR_INVALID, "NULL CSR array");
    if (val_type != GS_F64 && val_type != GS_F32)
        return fail(GS_ERR_UNSUPPORTED, "input CSR values must be FP64 or FP32");
    if (p.itype == GS_IDX_U16 && p.vtype == GS_F64)
        return fail(GS_ERR_UNSUPPORTED, "16-bit columns need FP32 or BF16 values");
    const bool reduced = p.vtype != GS_F64;
    if (reduced && !(p.format == GS_FMT_CSR || p.format == GS_FMT_K1 ||
                     (p.format == GS_FMT_AXT && p.tileH == 1) || p.format == GS_FMT_AXC))
        return fail(GS_ERR_UNSUPPORTED,
                    "FP32/BF16 storage is available for CSR, K1, AXC and tileH=1 AXT layouts");
    if ((d_xbake || ax_out) && p.vtype != GS_F64)
        return fail(GS_ERR_UNSUPPORTED, "baked layouts are FP64");

    cudaEvent_t e0, e1;
    GS_CUDA(cudaEventCreate(&e0));
    GS_CUDA(cudaEventCreate(&e1));
    GS_CUDA(cudaEventRecord(e0, s));

    A->p = p;
    A->nrows = n;
    A->ncols = ncols;
    A->nnz = nnz;

    // ---- validate the CSR (structure and column range)
    {
        DevBuf flag;
        GS_TRY(flag.alloc_zero(4, s));
        k_validate<<<blocks_for(n + 1), 256, 0, s>>>(n, ncols, nnz, d_row, d_col,
                                                     flag.as<uint32_t>());
        GS_CHECK_LAUNCH();
        uint32_t hf = 0;
        GS_CUDA(cudaMemcpyAsync(&hf, flag.p, 4, cudaMemcpyDeviceToHost, s));
        GS_CUDA(cudaStreamSynchronize(s));
        if (hf & 1u)
            return fail(GS_ERR_INVALID, "row pointer array is not a valid CSR row pointer");
        if (hf & 2u) return fail(GS_ERR_INVALID, "column index >= ncols");
    }

    FillArgs f{};
    f.n = n;
    f.row = d_row;
    f.col = d_col;
    f.val = d_val;
    f.xbake = d_xbake;
    DevBuf P;  // 64-bit offsets
    const gs_format fmt = p.format;

    if (fmt == GS_FMT_K1) {
        if (p.vtype == GS_F64 && p.itype != GS_IDX_U32)
            return fail(GS_ERR_UNSUPPORTED, "FP64 K1 is stored with 32-bit columns");
        const uint32_t chunkNum = (n + 31) / 32;
        A->chunkNum = chunkNum;
        DevBuf rl;
        GS_TRY(rl.alloc((size_t)n * 4));
        k_rowlen<<<blocks_for(n), 256, 0, s>>>(n, d_row, rl.as<uint32_t>());
        GS_CHECK_LAUNCH();
        uint32_t maxlen = 0;
        GS_TRY(reduce_max_u32(rl.as<uint32_t>(), n, &maxlen, s));
        GS_TRY(A->permi.alloc_zero(((size_t)chunkNum + 1) * 32 * 4, s));
        GS_TRY(stable_sort_desc(rl.as<uint32_t>(), n, maxlen, A->permi.as<uint32_t>(), s));
        GS_TRY(A->nmc.alloc_zero((size_t)chunkNum * 4, s));
        GS_TRY(A->k1len.alloc((size_t)n * 4));
        k_k1_meta<<<blocks_for(n), 256, 0, s>>>(n, chunkNum, rl.as<uint32_t>(),
                                                A->permi.as<uint32_t>(), A->nmc.as<uint32_t>(),
                                                A->k1len.as<uint32_t>());
        GS_CHECK_LAUNCH();
        GS_TRY(P.alloc(((size_t)chunkNum + 1) * 8));
        CountSpec cs{CountKind::ArrayTimes};
        cs.arr = A->nmc.as<uint32_t>();
        cs.a = 32;
        uint64_t lenvc = 0;
        GS_TRY(exclusive_scan(cs, chunkNum, P.as<uint64_t>(), &lenvc, s));
        if (lenvc > 0xffffffffull) return fail(GS_ERR_OVERFLOW, "K1 lenVC exceeds 32 bits");
        A->lenVC = (uint32_t)lenvc;
        GS_TRY(A->chp.alloc((size_t)chunkNum * 4));
        k_u64_to_u32<<<blocks_for(chunkNum), 256, 0, s>>>(chunkNum, P.as<uint64_t>(),
                                                         A->chp.as<uint32_t>());
        GS_CHECK_LAUNCH();
        const bool u16 = p.itype == GS_IDX_U16;
        const size_t vsz = dtype_size(p.vtype), isz = u16 ? 2 : 4;
        GS_TRY(A->val.alloc_zero((size_t)A->lenVC * vsz, s));
        GS_TRY(A->col.alloc_zero((size_t)A->lenVC * isz, s));
        DevBuf col32;  // 32-bit columns before the 16-bit steps are taken
        if (u16) GS_TRY(col32.alloc_zero((size_t)A->lenVC * 4, s));
        uint32_t *ocol = u16 ? col32.as<uint32_t>() : A->col.as<uint32_t>();
        GS_TRY(build_k1_plan(A->nmc.as<uint32_t>(), chunkNum, A->k1unit_chunk, A->k1unit_base,
                             A->k1partial, A->k1count, &A->k1units, s));
        // 16-bit steps: lane-blocked slot order (k1_slot); otherwise the reference's
        if (val_type == GS_F64)
            launch_fill_k1<double>(n, A->k1units, A->k1unit_chunk.as<uint32_t>(),
                                   A->k1unit_base.as<uint32_t>(), d_row, d_col,
                                   static_cast<const double *>(d_val), A->permi.as<uint32_t>(),
                                   A->chp.as<uint32_t>(), A->nmc.as<uint32_t>(), u16, p.vtype,
                                   A->val.p, ocol, s);
        else
            launch_fill_k1<float>(n, A->k1units, A->k1unit_chunk.as<uint32_t>(),
                                  A->k1unit_base.as<uint32_t>(), d_row, d_col,
                                  static_cast<const float *>(d_val), A->permi.as<uint32_t>(),
                                  A->chp.as<uint32_t>(), A->nmc.as<uint32_t>(), u16, p.vtype,
                                  A->val.p, ocol, s);
        GS_CHECK_LAUNCH();
        if (u16) {
            K1Args a{};
            a.nrows = n;
            a.chunkNum = chunkNum;
            a.nmc = A->nmc.as<uint32_t>();
            a.chp = A->chp.as<uint32_t>();
            a.klen = A->k1len.as<uint32_t>();
            a.unit_chunk = A->k1unit_chunk.as<uint32_t>();
            a.unit_base = A->k1unit_base.as<uint32_t>();
            a.units = A->k1units;
            GS_TRY(A->k1ck.alloc((size_t)A->k1units * 32 * 4));
            GS_TRY(build_k1_deltas(a, col32.as<uint32_t>(), A->col.as<uint16_t>(),
                                   A->k1ck.as<uint32_t>(), s));
        }
        A->nslots = A->lenVC;
        A->mfp = (double)chunkNum * 4 + (double)chunkNum * 4 + (double)A->lenVC * vsz +
                 (double)A->lenVC * isz + (double)n * 4 + (double)n * 8 +
                 (u16 ? (double)A->k1units * 128 : 0.0);
        A->beta = (double)nnz / (double)A->lenVC;
    } else {
        // ---------------- row-stream layouts
        const uint32_t thw = p.tileHW, th = p.tileH;
        if (fmt == GS_FMT_AXT && (thw == 0 || th == 0))
            return fail(GS_ERR_INVALID, "tileHW and tileH must be >= 1");
        if (fmt == GS_FMT_AXC && p.hbs == 0) return fail(GS_ERR_INVALID, "hbs must be >= 1");
        GS_TRY(A->rpos.alloc(((size_t)n + 1) * 4));
        bool need_rlen = false;
        uint64_t nslots = 0;
        f.layout = kDirect;
        if (fmt == GS_FMT_CSR) {
            GS_CUDA(cudaMemcpyAsync(A->rpos.p, d_row, ((size_t)n + 1) * 4,
                                    cudaMemcpyDeviceToDevice, s));
            nslots = nnz;
            A->mfp = (double)nnz * 8 + (double)nnz * 4 + ((double)n + 1) * 4 + (double)n * 8;
            A->beta = (double)nnz / (double)nnz;
        } else if (fmt == GS_FMT_AXC) {
            const uint32_t hbs = p.hbs;
            A->hbs = hbs;
            GS_TRY(P.alloc(((size_t)n + 1) * 8));
            CountSpec cs{CountKind::RowTiles};
            cs.row = d_row;
            cs.a = hbs;
            uint64_t bricks = 0;
            GS_TRY(exclusive_scan(cs, n, P.as<uint64_t>(), &bricks, s));
            if (bricks * 2ull * hbs > 0xffffffffull)
                return fail(GS_ERR_OVERFLOW, "AXC lenAX exceeds 32 bits");
            A->lenAX = (uint32_t)(bricks * 2 * hbs);
            A->lenBRP = n + 1;
            A->lenMAPX = A->lenAX / 2 + 8;
            if (p.keep_layout) GS_TRY(A->brp.alloc(((size_t)n + 1) * 4));
            k_tables<<<blocks_for((uint64_t)n + 1), 256, 0, s>>>(
                n, P.as<uint64_t>(), 2, hbs, 0, 0, p.keep_layout ? A->brp.as<uint32_t>() : nullptr,
                A->rpos.as<uint32_t>());
            GS_CHECK_LAUNCH();
            nslots = A->lenAX / 2;
            need_rlen = true;
            if (p.keep_layout) GS_TRY(A->mapx.alloc_zero((size_t)A->lenMAPX * 4, s));
            f.mapx = p.keep_layout ? A->mapx.as<uint32_t>() : nullptr;
            f.axw = hbs;
            A->mfp = (double)A->lenAX * 8 + (double)A->lenBRP * 4;
            A->beta = (double)nnz / (double)(A->lenAX >> 1);
        } else if (fmt == GS_FMT_AXT) {
            const uint32_t ths = thw * th;
            A->tileHW = thw;
            A->tileH = th;
            A->bs = p.bs;
            A->lenCON = n;
            A->logTH = ref_log_loop(th, 0, 10);
            f.thw = thw;
            f.th = th;
            f.bs = p.bs;
            f.axw = thw;
            if (p.keep_layout) GS_TRY(A->con.alloc_zero(((size_t)n + 1) * 4, s));
            if (p.mode == GS_AXT_UNC && th == 1) {
                GS_TRY(P.alloc(((size_t)n + 1) * 8));
                CountSpec cs{CountKind::RowTiles};
                cs.row = d_row;
                cs.a = thw;
                uint64_t tiles = 0;
                GS_TRY(exclusive_scan(cs, n, P.as<uint64_t>(), &tiles, s));
                if (tiles * 2ull * thw > 0xffffffffull)
                    return fail(GS_ERR_OVERFLOW, "AXT lenAX exceeds 32 bits");
                A->tileN = (uint32_t)tiles;
                A->lenAX = (uint32_t)(tiles * 2 * thw);
                A->lenSEC = (uint32_t)tiles;
                k_tables<<<blocks_for((uint64_t)n + 1), 256, 0, s>>>(
                    n, P.as<uint64_t>(), 0, thw, 0, 0,
                    p.keep_layout ? A->con.as<uint32_t>() : nullptr, A->rpos.as<uint32_t>());
                GS_CHECK_LAUNCH();
                nslots = tiles * thw;
                need_rlen = true;
                f.layout = kDirect;
                f.sec_mode = p.keep_layout ? kSecTile : kSecNone;
            } else if (p.mode == GS_AXT_UNC) {
                GS_TRY(P.alloc(((size_t)n + 1) * 8));
                CountSpec cs{CountKind::RowTiles};
                cs.row = d_row;
                cs.a = th;
                uint64_t cols = 0;
                GS_TRY(exclusive_scan(cs, n, P.as<uint64_t>(), &cols, s));
                const uint64_t tiles = (cols + thw - 1) / thw;
                if (tiles * 2ull * ths > 0xffffffffull || cols * th > 0xffffffffull)
                    return fail(GS_ERR_OVERFLOW, "AXT lenAX exceeds 32 bits");
                A->tileN = (uint32_t)tiles;
                A->lenAX = (uint32_t)(tiles * 2 * ths);
                A->lenSEC = (uint32_t)(tiles * thw);
                k_tables<<<blocks_for((uint64_t)n + 1), 256, 0, s>>>(
                    n, P.as<uint64_t>(), 1, 0, thw, th,
                    p.keep_layout ? A->con.as<uint32_t>() : nullptr, A->rpos.as<uint32_t>());
                GS_CHECK_LAUNCH();
                nslots = tiles * ths;
                need_rlen = true;
                A->tiled = 1;
                f.layout = kUncTiled;
                f.sec_mode = p.keep_layout ? kSecColumn : kSecNone;
            } else if (p.mode == GS_AXT_COM) {
                const uint64_t w = (th == 1) ? thw : ths;
                const uint64_t tiles = ((uint64_t)nnz + w - 1) / w;
                if (tiles * 2ull * w > 0xffffffffull)
                    return fail(GS_ERR_OVERFLOW, "AXT lenAX exceeds 32 bits");
                A->tileN = (uint32_t)tiles;
                A->lenAX = (uint32_t)(tiles * 2 * w);
                A->lenSEC = (uint32_t)(tiles * w);
                A->log = (th == 1) ? ref_log_loop(p.bs, 1, 11) : ref_log_loop(th, 1, 10);
                if (p.keep_layout && th == 1 && p.bs == 0)
                    return fail(GS_ERR_INVALID, "COM tileH=1 needs bs >= 1");
                if (p.keep_layout && A->log < 32 && (uint64_t)(n - 1) > (0xffffffffull >> A->log))
                    return fail(GS_ERR_OVERFLOW,
                                "COM header (row << %u) overflows 32 bits for %u rows", A->log,
                                n);
                f.log = A->log;
                GS_CUDA(cudaMemcpyAsync(A->rpos.p, d_row, ((size_t)n + 1) * 4,
                                        cudaMemcpyDeviceToDevice, s));
                nslots = A->lenSEC;
                A->tiled = th > 1 ? 1 : 0;
                f.layout = kCom;
                f.sec_mode = p.keep_layout ? kSecHeader : kSecNone;
            } else {
                return fail(GS_ERR_INVALID, "unknown AXT mode %d", (int)p.mode);
            }
            if (p.keep_layout) {
                GS_TRY(A->sec.alloc_zero((size_t)A->lenSEC * 4, s));
                f.sec = A->sec.as<uint32_t>();
            }
            A->mfp = (double)A->lenAX * 8 + (double)A->lenSEC * 4;
            A->beta = (double)nnz / (double)(A->lenAX >> 1);
        } else {
            return fail(GS_ERR_INVALID, "unknown format %d", (int)fmt);
        }
        if (nslots > 0xffffffffull) return fail(GS_ERR_OVERFLOW, "slot count exceeds 32 bits");
        A->nslots = (uint32_t)nslots;
        if (need_rlen) {
            GS_TRY(A->rlen.alloc((size_t)n * 4));
            k_rowlen<<<blocks_for(n), 256, 0, s>>>(n, d_row, A->rlen.as<uint32_t>());
            GS_CHECK_LAUNCH();
        }
        // ---- value / column streams (32-bit columns first; narrowed below for U16)
        if (p.itype == GS_IDX_U16 && A->tiled)
            return fail(GS_ERR_UNSUPPORTED, "16-bit columns need tileH=1");
        GS_TRY(A->val.alloc_zero((size_t)A->nslots * dtype_size(p.vtype), s));
        DevBuf col32;
        DevBuf &c32 = (p.itype == GS_IDX_U16) ? col32 : A->col;
        GS_TRY(c32.alloc_zero((size_t)A->nslots * 4, s));
        f.rpos = (f.layout == kCom) ? d_row : A->rpos.as<uint32_t>();
        f.oval = A->val.p;
        f.ocol = c32.as<uint32_t>();
        if (ax_out) {
            GS_TRY(ax_out->alloc_zero((size_t)A->lenAX * 8, s));
            f.ax = ax_out->as<double>();
        }
        if (val_type == GS_F64) GS_TRY(launch_fill<double>(f, p.vtype, s));
        else GS_TRY(launch_fill<float>(f, p.vtype, s));
        // ---- execution plan of the row-stream kernel.  Rows of the UNC layouts start on a
        // tile column (tileH > 1) or a tile (tileH = 1), and AXC rows on a brick: the lane
        // width V is chosen to divide that alignment so the aligned kernel applies.
        uint32_t V = kDirectV;
        bool aligned = false;
        if (!reduced && !A->tiled && !need_rlen)  // FP64 CSR and COM tileH = 1
            GS_TRY(direct_lane_positions(d_row, d_col, n, nnz, &V, s));
        if (A->tiled) {
            V = th;
            aligned = fmt == GS_FMT_AXT && p.mode == GS_AXT_UNC &&
                      (th == 2 || th == 4 || th == 8 || th == 16);
        } else if ((fmt == GS_FMT_AXT && p.mode == GS_AXT_UNC) || fmt == GS_FMT_AXC) {
            const uint32_t align = fmt == GS_FMT_AXC ? p.hbs : thw;
            if (reduced) {  // reduced-precision kernels use 8 positions per lane
                aligned = align % 8 == 0;
            } else {
                V = aligned_lane_positions(align, &aligned);
                // rows padded to 32 or more: 4 positions per lane where the x gathers are
                // random (AXC hbs 32 on the power-law 457.5 -> 434-440 us: groups of 4 slots
                // read less padding), else 8 (the 27-point stencil: 325 against 433 us)
                if (aligned && V == 8 && align >= 32) {
                    bool rnd = false;
                    GS_TRY(random_columns(d_row, d_col, n, &rnd, s));
                    if (rnd) V = 4;
                }
            }
        }
        GS_TRY(build_rows_plan(A->rpos.as<uint32_t>(), need_rlen ? A->rlen.as<uint32_t>() : nullptr,
                               n, V, A->plan, s, A->tiled));
        A->plan.aligned = aligned;
        if (A->tiled && aligned && (th == 2 || th == 4))
            GS_TRY(random_columns(d_row, d_col, n, &A->plan.grouped, s));
        // FP64 whole-tile layouts: the same rows over tiles for the tile kernel (windows of
        // one 32-tile chunk).  Widths 4-16 only: at 32 a tile spans 16 lanes and 16 load
        // steps, too few gathers in flight per lane (power-law AXC hbs 32: 846 us on the
        // tile kernel, 516 us on the aligned row kernel; hw16 482 instead of 612 us)
        A->tile_w = 0;
        if (!A->tiled && !reduced && p.itype == GS_IDX_U32 &&
            ((fmt == GS_FMT_AXT && p.mode == GS_AXT_UNC) || fmt == GS_FMT_AXC)) {
            const uint32_t w = fmt == GS_FMT_AXC ? p.hbs : thw;
            if (w == 4 || w == 8 || w == 16) {
                DevBuf rt;
                GS_TRY(rt.alloc(((size_t)n + 1) * 4));
                k_tile_starts<<<blocks_for(n + 1), 256, 0, s>>>(n + 1, A->rpos.as<uint32_t>(), w,
                                                                rt.as<uint32_t>());
                GS_CHECK_LAUNCH();
                GS_TRY(build_rows_plan(rt.as<uint32_t>(), nullptr, n, 1, A->tplan, s));
                A->tile_w = w;
            }
        }
        if (p.itype == GS_IDX_U16) {
            GS_TRY(A->col.alloc_zero((size_t)A->nslots * 2, s));
            GS_TRY(build_u16_columns(col32.as<uint32_t>(), A->nslots, A->plan,
                                     A->col.as<uint16_t>(), s));
            A->colbase.reset();
        }
    }

    GS_CUDA(cudaEventRecord(e1, s));
    GS_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    GS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    A->conv_ms = ms;
    return GS_OK;
}

}  // namespace gs
