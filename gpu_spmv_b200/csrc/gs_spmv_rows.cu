// gs_spmv_rows.cu -- the row-stream SpMV kernel shared by CSR, AXC and every AXT layout.
//
// What it computes is the reference's SpMV for each of those formats:
//   gcsr          cudaSpmv.cu:531-543   (CSR, one thread per row)
//   gaxc          cudaSpmv.cu:1072-1096 (AXC bricks, one warp per row)
//   gaxtuh1hw16w/08w/04w cudaSpmv.cu:1570-1850 (AXT UNC tileH=1, tiles summed, atomics)
//   gaxtuh        cudaSpmv.cu:1939-1959 (AXT UNC tileH>1, column sums, atomics)
//   gaxtch1       cudaSpmv.cu:2041-2097 (AXT COM tileH=1, block scan over headers)
//   gaxtch        cudaSpmv.cu:2174-2209 (AXT COM tileH>1, per-column segment walk)
// but the decomposition is different and the same for all of them:
//
// * Every layout is described by a row table: rpos[r] = first position of row r in the
//   layout's position space, rlen[r] = number of real (non-padding) positions (or NULL
//   when rows are unpadded).  A position maps to a storage slot either directly (CSR,
//   AXC, tileH=1 AXT: the layout stores each row's elements contiguously) or through the
//   tile transpose of the tileH>1 layouts (position P -> tile P/(th*thw), tile row P%th,
//   tile column (P%(th*thw))/th), which is what makes lane-contiguous positions land in
//   warp-coalesced slots.
// * One warp owns RPU consecutive rows.  It walks their positions in windows of
//   32 lanes x V positions; each lane takes V consecutive positions (merge-path style):
//   vector loads of the value/column streams, independent x gathers (read-only path,
//   through L2), a sequential per-lane sum with row breaks, then one segmented warp scan
//   (5 shuffles) joins rows that cross lanes, and a carry joins rows that cross windows.
// * Padding positions are never multiplied and never loaded when a lane's whole share is
//   padding.  Every y entry is written exactly once (no atomics, no y pre-zeroing), so the
//   result is deterministic and one launch is the whole SpMV.
//
// Baked mode reads the reference layouts with x baked into ax (value half at
// ax[(s/w)*2w + s%w], x half w further), which is what the drop-in entry points receive.
#include <cuda_bf16.h>

#include <type_traits>

#include "gs_internal.cuh"

namespace gs {

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr unsigned kFull = 0xffffffffu;

template <class T> __device__ __forceinline__ T shfl_up(T v, int d) {
    return __shfl_up_sync(kFull, v, d);
}
template <class T> __device__ __forceinline__ T shfl_idx(T v, int l) {
    return __shfl_sync(kFull, v, l);
}

// exact product / sum without contraction into FMA (the reference's CPU loop multiplies
// and adds separately)
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// ---- streaming loads of V consecutive elements starting at an aligned index
template <class T, int V> struct VecLoad;
template <> struct VecLoad<double, 4> {
    __device__ __forceinline__ static void run(const double *p, double (&o)[4]) {
        double2 a = __ldcs(reinterpret_cast<const double2 *>(p));
        double2 b = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
};
template <> struct VecLoad<double, 8> {
    __device__ __forceinline__ static void run(const double *p, double (&o)[8]) {
        const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
        for (int i = 0; i < 4; i++) { double2 a = __ldcs(q + i); o[2 * i] = a.x; o[2 * i + 1] = a.y; }
    }
};
template <> struct VecLoad<float, 4> {
    __device__ __forceinline__ static void run(const float *p, float (&o)[4]) {
        float4 a = __ldcs(reinterpret_cast<const float4 *>(p));
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    }
};
template <> struct VecLoad<float, 8> {
    __device__ __forceinline__ static void run(const float *p, float (&o)[8]) {
        const float4 *q = reinterpret_cast<const float4 *>(p);
        float4 a = __ldcs(q), b = __ldcs(q + 1);
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
        o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
    }
};
template <> struct VecLoad<uint32_t, 4> {
    __device__ __forceinline__ static void run(const uint32_t *p, uint32_t (&o)[4]) {
        uint4 a = __ldcs(reinterpret_cast<const uint4 *>(p));
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    }
};
template <> struct VecLoad<uint32_t, 8> {
    __device__ __forceinline__ static void run(const uint32_t *p, uint32_t (&o)[8]) {
        const uint4 *q = reinterpret_cast<const uint4 *>(p);
        uint4 a = __ldcs(q), b = __ldcs(q + 1);
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
        o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
    }
};
template <> struct VecLoad<uint16_t, 4> {
    __device__ __forceinline__ static void run(const uint16_t *p, uint16_t (&o)[4]) {
        uint2 a = __ldcs(reinterpret_cast<const uint2 *>(p));
        o[0] = a.x & 0xffff; o[1] = a.x >> 16; o[2] = a.y & 0xffff; o[3] = a.y >> 16;
    }
};
template <> struct VecLoad<uint16_t, 8> {
    __device__ __forceinline__ static void run(const uint16_t *p, uint16_t (&o)[8]) {
        uint4 a = __ldcs(reinterpret_cast<const uint4 *>(p));
        uint32_t w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int i = 0; i < 4; i++) { o[2 * i] = w[i] & 0xffff; o[2 * i + 1] = w[i] >> 16; }
    }
};
template <> struct VecLoad<__nv_bfloat16, 4> {
    __device__ __forceinline__ static void run(const __nv_bfloat16 *p, __nv_bfloat16 (&o)[4]) {
        uint2 a = __ldcs(reinterpret_cast<const uint2 *>(p));
        uint32_t w[2] = {a.x, a.y};
#pragma unroll
        for (int i = 0; i < 2; i++) {
            o[2 * i] = __ushort_as_bfloat16((unsigned short)(w[i] & 0xffff));
            o[2 * i + 1] = __ushort_as_bfloat16((unsigned short)(w[i] >> 16));
        }
    }
};
template <> struct VecLoad<__nv_bfloat16, 8> {
    __device__ __forceinline__ static void run(const __nv_bfloat16 *p, __nv_bfloat16 (&o)[8]) {
        uint4 a = __ldcs(reinterpret_cast<const uint4 *>(p));
        uint32_t w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            o[2 * i] = __ushort_as_bfloat16((unsigned short)(w[i] & 0xffff));
            o[2 * i + 1] = __ushort_as_bfloat16((unsigned short)(w[i] >> 16));
        }
    }
};

template <class T> __device__ __forceinline__ T ld_stream(const T *p) { return __ldcs(p); }
template <> __device__ __forceinline__ __nv_bfloat16 ld_stream(const __nv_bfloat16 *p) {
    return __ushort_as_bfloat16(__ldcs(reinterpret_cast<const unsigned short *>(p)));
}

template <class T> __device__ __forceinline__ T to_acc(double v);
template <> __device__ __forceinline__ double to_acc<double>(double v) { return v; }
template <> __device__ __forceinline__ float to_acc<float>(double v) { return (float)v; }

template <class YT, class AT> __device__ __forceinline__ void store_y(YT *y, AT v) {
    *y = (YT)v;
}

// ---------------------------------------------------------------------------------------
// VT value storage, IT column storage (u32 or u16 offsets), XT x type, PT product type,
// AT accumulation type, YT output type.  VMAX positions per lane (compile time); the
// runtime lane share is VMAX for direct layouts and th (<= VMAX) for tiled ones.
template <class VT, class IT, class XT, class PT, class AT, class YT, int VMAX, bool TILED,
          bool BAKED, int RPU>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
k_rows(const RowsArgs a, const uint32_t nunits)
{
    __shared__ uint32_t s_rps[kWarpsPerBlock][RPU + 1];
    __shared__ uint32_t s_rre[kWarpsPerBlock][RPU];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    uint32_t *rps = s_rps[wib];
    uint32_t *rre = s_rre[wib];
    YT *y = static_cast<YT *>(a.y);
    const VT *val = static_cast<const VT *>(a.val);
    const IT *col = static_cast<const IT *>(a.col);
    const XT *x = static_cast<const XT *>(a.x);
    const double *ax = static_cast<const double *>(a.val);
    const uint32_t V = TILED ? a.th : (uint32_t)VMAX;
    const uint32_t WS = 32u * V;
    const uint32_t ths = a.th * a.thw;

    for (uint32_t u = blockIdx.x * kWarpsPerBlock + wib; u < nunits;
         u += gridDim.x * kWarpsPerBlock) {
        const uint32_t R0 = u * RPU;
        const int nr = (int)min((uint32_t)RPU, a.nrows - R0);
        // ---- row table of the unit
        for (int i = lane; i <= nr; i += 32) rps[i] = __ldg(a.rpos + R0 + i);
        __syncwarp();
        for (int i = lane; i < nr; i += 32) {
            uint32_t s0 = rps[i], s1 = rps[i + 1];
            rre[i] = a.rlen ? s0 + __ldg(a.rlen + R0 + i) : s1;
            if (s0 == s1) store_y<YT, AT>(y + R0 + i, (AT)0);  // empty row
        }
        __syncwarp();
        const uint32_t P0 = rps[0], P1 = rps[nr];
        const uint32_t cbase = (sizeof(IT) == 2) ? __ldg(a.colbase + u) : 0u;
        AT carry = (AT)0;
        uint32_t W = TILED ? (P0 / ths) * ths : (P0 / V) * V;
        for (; W < P1; W += WS) {
            const uint32_t qb = W + (uint32_t)lane * V;
            // ---- pass A: the row of each of the lane's positions, real or padding
            int ridx[VMAX];
            bool real[VMAX];
            bool anyreal = false;
            int cur = -1;
            if (qb + V > P0 && qb < P1) {
                const uint32_t qf = max(qb, P0);
                int lo = 0, hi = nr - 1;
                while (lo < hi) {
                    int mid = (lo + hi + 1) >> 1;
                    if (rps[mid] <= qf) lo = mid; else hi = mid - 1;
                }
                cur = lo;
            }
#pragma unroll
            for (int k = 0; k < VMAX; k++) {
                const uint32_t q = qb + k;
                ridx[k] = -1;
                real[k] = false;
                if (k < (int)V && cur >= 0 && q >= P0 && q < P1) {
                    while (cur + 1 < nr && rps[cur + 1] <= q) cur++;
                    ridx[k] = cur;
                    real[k] = q < rre[cur];
                    anyreal |= real[k];
                }
            }
            // ---- loads, gathers, products
            PT prod[VMAX];
#pragma unroll
            for (int k = 0; k < VMAX; k++) prod[k] = (PT)0;
            if constexpr (BAKED) {
#pragma unroll
                for (int k = 0; k < VMAX; k++) {
                    if (real[k]) {
                        uint32_t q = qb + k, s;
                        if constexpr (TILED) {
                            uint32_t t = q / ths, rem = q - t * ths, c = rem / a.th;
                            s = t * ths + (rem - c * a.th) * a.thw + c;
                        } else {
                            s = q;
                        }
                        uint32_t ai = (s / a.axw) * 2u * a.axw + s % a.axw;
                        prod[k] = (PT)mul_rn(__ldcs(ax + ai), __ldcs(ax + ai + a.axw));
                    }
                }
            } else if constexpr (!TILED) {
                if (anyreal) {
                    VT v[VMAX];
                    IT c[VMAX];
                    if (qb + VMAX <= a.nslots) {
                        VecLoad<VT, VMAX>::run(val + qb, v);
                        VecLoad<IT, VMAX>::run(col + qb, c);
                    } else {  // stream tail: element loads, never past the last slot
#pragma unroll
                        for (int k = 0; k < VMAX; k++) {
                            if (real[k]) {
                                v[k] = ld_stream(val + qb + k);
                                c[k] = ld_stream(col + qb + k);
                            }
                        }
                    }
                    XT xv[VMAX];
#pragma unroll
                    for (int k = 0; k < VMAX; k++)
                        xv[k] = real[k] ? __ldg(x + (cbase + (uint32_t)c[k])) : (XT)0;
#pragma unroll
                    for (int k = 0; k < VMAX; k++)
                        if (real[k])
                            prod[k] = mul_rn((PT)ValTraits<VT>::to_f64(v[k]), (PT)xv[k]);
                }
            } else {
                VT v[VMAX];
                IT c[VMAX];
#pragma unroll
                for (int k = 0; k < VMAX; k++) {
                    if (real[k]) {
                        uint32_t q = qb + k;
                        uint32_t t = q / ths, rem = q - t * ths, cc = rem / a.th;
                        uint32_t s = t * ths + (rem - cc * a.th) * a.thw + cc;
                        v[k] = ld_stream(val + s);
                        c[k] = ld_stream(col + s);
                    }
                }
                XT xv[VMAX];
#pragma unroll
                for (int k = 0; k < VMAX; k++)
                    xv[k] = real[k] ? __ldg(x + (cbase + (uint32_t)c[k])) : (XT)0;
#pragma unroll
                for (int k = 0; k < VMAX; k++)
                    if (real[k]) prod[k] = mul_rn((PT)ValTraits<VT>::to_f64(v[k]), (PT)xv[k]);
            }
            // ---- pass B: sequential lane sum with row breaks
            int first = -1, last = -1, nb = 0;
            bool starts = false;
            AT head = (AT)0, acc = (AT)0;
            uint32_t qlast = 0;
#pragma unroll
            for (int k = 0; k < VMAX; k++) {
                if (ridx[k] < 0) continue;
                const uint32_t q = qb + k;
                if (first < 0) {
                    first = last = ridx[k];
                    starts = (q == rps[first]);
                } else if (ridx[k] != last) {
                    if (nb == 0) head = acc;
                    else store_y<YT, AT>(y + R0 + last, acc);  // row entirely in this lane
                    nb++;
                    acc = (AT)0;
                    last = ridx[k];
                }
                if (real[k]) acc = add_rn(acc, (AT)prod[k]);
                qlast = q;
            }
            const bool has = first >= 0;
            const bool ends = has && (qlast + 1 == rps[last + 1]);
            // ---- segmented inclusive scan of the lanes' last segments
            const bool rf = has && (nb > 0 || starts);
            const unsigned rmask = __ballot_sync(kFull, rf);
            const unsigned le = rmask & (kFull >> (31 - lane));
            const int sstart = le ? 31 - __clz(le) : -1;
            AT S = acc;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                AT t = shfl_up(S, d);
                if (lane >= d && lane - d >= sstart) S = add_rn(S, t);
            }
            if (sstart < 0) S = add_rn(S, carry);
            AT E = shfl_up(S, 1);
            if (lane == 0) E = carry;
            if (has) {
                if (nb > 0) store_y<YT, AT>(y + R0 + first, starts ? head : add_rn(head, E));
                if (ends) store_y<YT, AT>(y + R0 + last, S);
            }
            carry = shfl_idx(S, 31);
        }
    }
}

template <class VT, class IT, class XT, class PT, class AT, class YT, int VMAX, bool TILED,
          bool BAKED>
gs_status launch_rpu(const RowsArgs &a, uint32_t rpu, cudaStream_t s)
{
    uint32_t nunits = (a.nrows + rpu - 1) / rpu;
    if (nunits == 0) return GS_OK;
    uint32_t blocks = (nunits + kWarpsPerBlock - 1) / kWarpsPerBlock;
    blocks = min(blocks, 148u * 64u);
    switch (rpu) {
    case 32:
        k_rows<VT, IT, XT, PT, AT, YT, VMAX, TILED, BAKED, 32>
            <<<blocks, kWarpsPerBlock * 32, 0, s>>>(a, nunits);
        break;
    case 64:
        k_rows<VT, IT, XT, PT, AT, YT, VMAX, TILED, BAKED, 64>
            <<<blocks, kWarpsPerBlock * 32, 0, s>>>(a, nunits);
        break;
    case 128:
        k_rows<VT, IT, XT, PT, AT, YT, VMAX, TILED, BAKED, 128>
            <<<blocks, kWarpsPerBlock * 32, 0, s>>>(a, nunits);
        break;
    default: return fail(GS_ERR_UNSUPPORTED, "rows per unit %u not supported", rpu);
    }
    GS_CHECK_LAUNCH();
    return GS_OK;
}

template <class VT, class IT, class XT, class PT, class AT, class YT, bool BAKED>
gs_status launch_shape(const RowsArgs &a, bool tiled, uint32_t lane_pos, uint32_t rpu,
                       cudaStream_t s)
{
    if constexpr (!std::is_same<VT, double>::value) {
        // reduced-precision storage: direct (tileH = 1) layouts, 8 positions per lane
        (void)lane_pos;
        if (tiled)
            return fail(GS_ERR_UNSUPPORTED, "FP32/BF16 storage needs a tileH=1 layout");
        return launch_rpu<VT, IT, XT, PT, AT, YT, 8, false, BAKED>(a, rpu, s);
    } else {
        if (tiled) {
            if (a.th <= 4) return launch_rpu<VT, IT, XT, PT, AT, YT, 4, true, BAKED>(a, rpu, s);
            if (a.th <= 8) return launch_rpu<VT, IT, XT, PT, AT, YT, 8, true, BAKED>(a, rpu, s);
            if (a.th <= 16)
                return launch_rpu<VT, IT, XT, PT, AT, YT, 16, true, BAKED>(a, rpu, s);
            return fail(GS_ERR_UNSUPPORTED, "tileH %u > 16 not supported by the kernels", a.th);
        }
        if (lane_pos == 8) return launch_rpu<VT, IT, XT, PT, AT, YT, 8, false, BAKED>(a, rpu, s);
        return launch_rpu<VT, IT, XT, PT, AT, YT, 4, false, BAKED>(a, rpu, s);
    }
}

}  // namespace

uint32_t choose_rpu(uint32_t nrows, uint64_t positions, uint32_t lane_pos)
{
    // aim for at least ~4 windows of work per warp unit
    double avg = nrows ? (double)positions / nrows : 0.0;
    double target = 4.0 * 32.0 * lane_pos;
    if (avg * 32 >= target) return 32;
    if (avg * 64 >= target) return 64;
    return 128;
}

gs_status launch_rows(const RowsArgs &a, gs_dtype vtype, gs_itype itype, gs_dtype ytype,
                      uint32_t flags, bool tiled, bool baked, uint32_t lane_pos, uint32_t rpu,
                      cudaStream_t s)
{
    if (tiled && (a.thw == 0 || 32 % a.thw != 0))
        return fail(GS_ERR_UNSUPPORTED, "tileH>1 kernels need tileHW dividing 32 (got %u)",
                    a.thw);
    if (baked) {
        if (vtype != GS_F64 || ytype != GS_F64)
            return fail(GS_ERR_UNSUPPORTED, "baked layouts are FP64 only");
        return launch_shape<double, uint32_t, double, double, double, double, true>(
            a, tiled, lane_pos, rpu, s);
    }
    const bool acc64 = (flags & GS_FLAG_ACC_F64) != 0;
    if (vtype == GS_F64) {
        if (ytype != GS_F64 || itype != GS_IDX_U32)
            return fail(GS_ERR_UNSUPPORTED, "FP64 matrices take FP64 y and 32-bit columns");
        return launch_shape<double, uint32_t, double, double, double, double, false>(
            a, tiled, lane_pos, rpu, s);
    }
#define GS_MIXED(VT_, IT_)                                                                 \
    do {                                                                                   \
        if (acc64 && ytype == GS_F64)                                                      \
            return launch_shape<VT_, IT_, float, float, double, double, false>(            \
                a, tiled, lane_pos, rpu, s);                                               \
        if (acc64)                                                                         \
            return launch_shape<VT_, IT_, float, float, double, float, false>(             \
                a, tiled, lane_pos, rpu, s);                                               \
        if (ytype == GS_F64)                                                               \
            return launch_shape<VT_, IT_, float, float, float, double, false>(             \
                a, tiled, lane_pos, rpu, s);                                               \
        return launch_shape<VT_, IT_, float, float, float, float, false>(a, tiled,         \
                                                                         lane_pos, rpu, s); \
    } while (0)
    if (vtype == GS_F32 && itype == GS_IDX_U32) GS_MIXED(float, uint32_t);
    if (vtype == GS_F32 && itype == GS_IDX_U16) GS_MIXED(float, uint16_t);
    if (vtype == GS_BF16 && itype == GS_IDX_U32) GS_MIXED(__nv_bfloat16, uint32_t);
    if (vtype == GS_BF16 && itype == GS_IDX_U16) GS_MIXED(__nv_bfloat16, uint16_t);
#undef GS_MIXED
    return fail(GS_ERR_UNSUPPORTED, "value type %d / index type %d not supported", (int)vtype,
                (int)itype);
}

}  // namespace gs
