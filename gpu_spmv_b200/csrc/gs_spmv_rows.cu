// gs_spmv_rows.cu -- the row-stream SpMV kernels shared by CSR, AXC and every AXT layout.
//
// What they compute is the reference's SpMV for each of those formats:
//   gcsr          cudaSpmv.cu:531-543   (CSR, one thread per row)
//   gaxc          cudaSpmv.cu:1072-1096 (AXC bricks, one warp per row)
//   gaxtuh1hw16w/08w/04w cudaSpmv.cu:1570-1850 (AXT UNC tileH=1, tiles summed, atomics)
//   gaxtuh        cudaSpmv.cu:1939-1959 (AXT UNC tileH>1, column sums, atomics)
//   gaxtch1       cudaSpmv.cu:2041-2097 (AXT COM tileH=1, block scan over headers)
//   gaxtch        cudaSpmv.cu:2174-2209 (AXT COM tileH>1, per-column segment walk)
// with one decomposition for all of them:
//
// * Position space.  Every layout is a sequence of positions in which each row occupies a
//   contiguous span (CSR and COM: the CSR element order; UNC and AXC: the padded rows).  A
//   position maps to a storage slot directly (tileH = 1 layouts) or through the tile
//   transpose of the tileH > 1 layouts (position P -> tile P/(th*thw), tile row P%th, tile
//   column (P%(th*thw))/th): the lane that owns th consecutive positions then reads one
//   slot of each tile row, and a warp's 32 lanes read 32 consecutive slots.
// * Plan (built once at conversion): a bitmap of row starts (1 bit per position), a
//   bitmap of real positions for padded layouts, and the running count of row starts per
//   window.  They replace the per-row pointers: a window's row structure is one popcount
//   scan across the warp.
// * Work: a warp owns a range of windows of 32 lanes x V positions; a lane takes V
//   consecutive positions: V independent x gathers through L2 (read-only path), a
//   sequential per-lane sum with row breaks, one segmented warp scan (5 shuffles) to join
//   rows that cross lanes, a carry for rows that cross windows.  A row belongs to the warp
//   in whose range it starts: the warp skips the leading continuation of the previous
//   warp's row and finishes its own last row past the end of its range.  Every y entry is
//   written once with a fixed summation order: no atomics, no y zero-fill, deterministic,
//   one launch per SpMV.
// * Staging.  k_rows loads the value/column streams with vectorised streaming loads
//   (direct layouts: 32 bytes per lane and request when the streams are 32-byte aligned)
//   or coalesced per-tile-row loads (tiled layouts).  k_rows_tma, for the
//   tiled layouts with 32-wide tiles, streams whole tiles into a per-warp ring of shared
//   memory stages with 1-D TMA bulk copies (cp.async.bulk, no multicast) completing on
//   mbarriers, several tiles ahead of the warp; the L1 then serves only the x gathers,
//   and lane c reads its tile column at a 32-slot stride (no bank conflicts).  Waits on
//   the mbarriers are bounded: on timeout the kernel records an error in the status word
//   and leaves.
//
// Baked mode reads the reference layouts with x baked into ax (value half at
// ax[(s/w)*2w + s%w], x half w further), which is what the drop-in entry points receive.
#include <cuda_bf16.h>

#include <type_traits>

#include "gs_bulk.cuh"
#include "gs_internal.cuh"

namespace gs {

namespace {

using namespace bulk;

constexpr int kWarpsPerBlock = 8;
constexpr int kTmaWarps = 4;   // warps per block of the TMA kernel
constexpr int kTmaStages = 4;  // tiles in flight per warp
constexpr unsigned kFull = 0xffffffffu;

// exact product / sum, never contracted into FMA (the reference's CPU loop multiplies and
// adds separately)
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// Segmented inclusive warp scan of S: sstart is the lane of the row start at or before
// this lane (-1: the row began before the window).  Level d adds lane - d into a lane only
// where lane - d >= sstart, i.e. where the lane's run (lane - sstart) is at least d.  SPAN:
// levels above the warp's longest run, which add nothing anywhere, are skipped after one
// max-reduction of the runs; the sums and their order are those of the five-level scan.
template <bool SPAN, class AT> __device__ __forceinline__ void seg_scan(AT &S, int lane, int sstart)
{
    uint32_t span = 32u;
    if constexpr (SPAN) span = __reduce_max_sync(kFull, (uint32_t)(lane - sstart));
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        if (SPAN && (uint32_t)d > span) break;
        AT t = __shfl_up_sync(kFull, S, d);
        if (lane >= d && lane - d >= sstart) S = add_rn(S, t);
    }
}

// ---- streaming loads of 8 consecutive elements from an 8-element-aligned index
template <class T> struct Load8;
template <> struct Load8<double> {
    __device__ __forceinline__ static void run(const double *p, double (&o)[8]) {
        const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            double2 a = __ldcs(q + i);
            o[2 * i] = a.x;
            o[2 * i + 1] = a.y;
        }
    }
};
template <> struct Load8<float> {
    __device__ __forceinline__ static void run(const float *p, float (&o)[8]) {
        const float4 *q = reinterpret_cast<const float4 *>(p);
        float4 a = __ldcs(q), b = __ldcs(q + 1);
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
        o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
    }
};
template <> struct Load8<uint32_t> {
    __device__ __forceinline__ static void run(const uint32_t *p, uint32_t (&o)[8]) {
        const uint4 *q = reinterpret_cast<const uint4 *>(p);
        uint4 a = __ldcs(q), b = __ldcs(q + 1);
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
        o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
    }
};
template <> struct Load8<uint16_t> {
    __device__ __forceinline__ static void run(const uint16_t *p, uint16_t (&o)[8]) {
        uint4 a = __ldcs(reinterpret_cast<const uint4 *>(p));
        uint32_t w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int i = 0; i < 4; i++) { o[2 * i] = w[i] & 0xffff; o[2 * i + 1] = w[i] >> 16; }
    }
};
template <> struct Load8<__nv_bfloat16> {
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

// 32-byte streaming loads (sm_100): a lane's 8 consecutive elements of 4 bytes in one load,
// of 8 bytes in two, so that a warp's load instruction covers 1 KB of the stream in 8 lines
// (16-byte loads at a 32- or 64-byte lane stride ask for each line two or four times).
// The address must be 32-byte aligned.  Two-byte elements keep the 16-byte load, which
// already covers a lane's 8 elements in one piece.
template <class T> struct Load8W {
    __device__ __forceinline__ static void run(const T *p, T (&o)[8]) { Load8<T>::run(p, o); }
};
template <> struct Load8W<double> {
    __device__ __forceinline__ static void run(const double *p, double (&o)[8]) {
        asm("ld.global.cs.v4.f64 {%0, %1, %2, %3}, [%4];"
            : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3]) : "l"(p));
        asm("ld.global.cs.v4.f64 {%0, %1, %2, %3}, [%4];"
            : "=d"(o[4]), "=d"(o[5]), "=d"(o[6]), "=d"(o[7]) : "l"(p + 4));
    }
};
template <> struct Load8W<uint32_t> {
    __device__ __forceinline__ static void run(const uint32_t *p, uint32_t (&o)[8]) {
        asm("ld.global.cs.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=r"(o[0]), "=r"(o[1]), "=r"(o[2]), "=r"(o[3]), "=r"(o[4]), "=r"(o[5]),
              "=r"(o[6]), "=r"(o[7])
            : "l"(p));
    }
};
template <> struct Load8W<float> {
    __device__ __forceinline__ static void run(const float *p, float (&o)[8]) {
        uint32_t r[8];
        Load8W<uint32_t>::run(reinterpret_cast<const uint32_t *>(p), r);
#pragma unroll
        for (int i = 0; i < 8; i++) o[i] = __uint_as_float(r[i]);
    }
};
// a lane's 8 consecutive stream elements: 32-byte loads when both streams allow them
template <class VT, class IT>
__device__ __forceinline__ void load8_streams(bool wide, const VT *val, const IT *col,
                                              VT (&v)[8], IT (&c)[8])
{
    if (wide) {
        Load8W<VT>::run(val, v);
        Load8W<IT>::run(col, c);
    } else {
        Load8<VT>::run(val, v);
        Load8<IT>::run(col, c);
    }
}

// a lane's VM consecutive stream elements from a VM-aligned index: 8 as above; 4 FP64 values
// (32 bytes: one request when wide) with 4 32-bit columns (one 16-byte load)
template <class VT, class IT, int VM>
__device__ __forceinline__ void load_streams(bool wide, const VT *val, const IT *col,
                                             VT (&v)[VM], IT (&c)[VM])
{
    if constexpr (VM == 8) {
        load8_streams<VT, IT>(wide, val, col, v, c);
    } else if constexpr (VM == 4 && sizeof(VT) == 8 && sizeof(IT) == 4) {
        if (wide) {
            asm("ld.global.cs.v4.f64 {%0, %1, %2, %3}, [%4];"
                : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(val));
        } else {
            const double2 a = __ldcs(reinterpret_cast<const double2 *>(val));
            const double2 b = __ldcs(reinterpret_cast<const double2 *>(val) + 1);
            v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
        }
        const uint4 q = __ldcs(reinterpret_cast<const uint4 *>(col));
        c[0] = q.x; c[1] = q.y; c[2] = q.z; c[3] = q.w;
    } else {
#pragma unroll
        for (int k = 0; k < VM; k++) {
            v[k] = __ldcs(val + k);
            c[k] = __ldcs(col + k);
        }
    }
}

template <class T> __device__ __forceinline__ T ld_stream(const T *p) { return __ldcs(p); }
template <> __device__ __forceinline__ __nv_bfloat16 ld_stream(const __nv_bfloat16 *p) {
    return __ushort_as_bfloat16(__ldcs(reinterpret_cast<const unsigned short *>(p)));
}

template <class YT, class AT> __device__ __forceinline__ void store_y(YT *y, AT v) { *y = (YT)v; }

// V bits of a position bitmap starting at position p (V <= 32; the bitmap has two words
// of zero slack past its last window)
__device__ __forceinline__ uint32_t get_bits(const uint32_t *bm, uint32_t p, uint32_t V)
{
    const uint32_t w = p >> 5, sh = p & 31;
    const uint64_t two = (uint64_t)__ldg(bm + w) | ((uint64_t)__ldg(bm + w + 1) << 32);
    return (uint32_t)(two >> sh) & (V >= 32 ? 0xffffffffu : ((1u << V) - 1u));
}

// ---------------------------------------------------------------------------------------
// Window control: which of the lane's V positions belong to this warp.  Before the first
// row start of the warp's range, positions continue an earlier warp's row (skipped); past
// the range ("over"), only the remainder of the warp's last row counts.
struct WinCtl {
    uint32_t vmask;
    unsigned slanes;  // lanes with a row start among their in-bounds positions
    bool skip;        // nothing of this window is ours
};

__device__ __forceinline__ WinCtl window_ctl(int lane, uint32_t W, uint32_t V, uint32_t FULLV,
                                             uint32_t npos, uint32_t sraw, bool seen, bool over)
{
    const uint32_t qb = W + (uint32_t)lane * V;
    WinCtl c;
    const uint32_t inb = (qb >= npos) ? 0u
                         : (qb + V <= npos ? FULLV : ((1u << (npos - qb)) - 1u));
    c.slanes = __ballot_sync(kFull, (sraw & inb) != 0u);
    c.vmask = inb;
    c.skip = false;
    if (!seen || over) {
        if (c.slanes == 0u) {
            if (!seen) c.skip = true;
        } else {
            const int fl = __ffs(c.slanes) - 1;
            const uint32_t fb = __shfl_sync(kFull, sraw & inb, fl);
            const uint32_t fpos = W + (uint32_t)fl * V + (uint32_t)(__ffs(fb) - 1);
            const uint32_t ge = (qb >= fpos) ? FULLV
                                : (qb + V <= fpos ? 0u : ((FULLV << (fpos - qb)) & FULLV));
            c.vmask = seen ? (c.vmask & ~ge) : (c.vmask & ge);
        }
    }
    return c;
}

// Row ranks by ballots, one per bit of the lanes' counts of row starts (BR), or by a shuffle
// scan of those counts: the same ranks.  Ballots ran faster for tiled layouts of 8 positions
// per lane (COM th=8: power-law 394 -> 345 us, 27-point stencil 450 -> 393) and of 2 (COM th=2
// on the power-law 418 -> 404, the stencil 574 -> 577) and for direct layouts of 4 (CSR on the
// power-law 329 -> 324), slower for direct layouts of 8 (CSR on the stencil 321 -> 333) and
// tiled ones of 4 (COM th=4 on the power-law 358 -> 380) and 16 (COM th=16 624 -> 872).
template <int VM, bool TILED>
constexpr bool kBallotRanks = TILED ? (VM == 8 || VM == 2) : VM == 4;
// Span-limited scans (seg_scan) where they measured faster, FP64 with x gathered at run
// time: direct layouts (power-law CSR 323.0 -> 320.9 us, 27-point stencil 313.8 -> 309.4)
// and tiled tileH 8 (COM th=8 345.2 -> 343.3, 394.0 -> 389.8).  Tiled tileH 2 and 4 keep
// the full scan (COM th=2 390 -> 398, th=4 357.5 -> 358.4 with it), and so do tileH 16
// (COM th=16 623.5 -> 626.0) and the baked layouts (drop-in gaxtch1 199 -> 200.6).
template <class VT, int VM, bool TILED, bool BAKED>
constexpr bool kScanSpan = std::is_same<VT, double>::value && !BAKED && (!TILED || VM == 8);

// Row ranks, sequential lane sums, segmented warp scan, y writes and the window carry.
template <class AT, class YT, int VM, bool EMPTY, class PT, bool BR, bool SPAN = false>
__device__ __forceinline__ void window_reduce(const RowsArgs &a, YT *y, int lane, uint32_t W,
                                              uint32_t V, uint32_t sraw, uint32_t vmask,
                                              uint32_t rb, const PT (&prod)[VM], uint32_t &cnt,
                                              AT &carry)
{
    const uint32_t qb = W + (uint32_t)lane * V;
    const uint32_t sb = sraw & vmask;
    const int c0 = __popc(sb);
    // inc: row starts of the window up to and including the lane's; nxt_lane: bit 0 is
    // whether the next lane's first position starts a row
    int inc;
    uint32_t total, nxt_lane;
    if constexpr (BR) {
        constexpr int kCountBits = VM >= 16 ? 5 : (VM >= 8 ? 4 : (VM >= 4 ? 3 : (VM >= 2 ? 2 : 1)));
        const unsigned below = (1u << lane) - 1u;
        inc = c0;
        total = 0;
#pragma unroll
        for (int bit = 0; bit < kCountBits; bit++) {
            const unsigned B = __ballot_sync(kFull, (c0 >> bit) & 1);
            inc += __popc(B & below) << bit;
            total += (uint32_t)__popc(B) << bit;
        }
        nxt_lane = __ballot_sync(kFull, sraw & 1u) >> ((lane + 1) & 31);
    } else {
        inc = c0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int t = __shfl_up_sync(kFull, inc, d);
            if (lane >= d) inc += t;
        }
        total = (uint32_t)__shfl_sync(kFull, inc, 31);
        nxt_lane = __shfl_down_sync(kFull, sraw, 1);
    }
    const uint32_t nxt_win = (lane == 31) ? get_bits(a.sbits, W + 32u * V, 1) : 0u;

    const bool has = vmask != 0u;
    const int kfirst = has ? __ffs(vmask) - 1 : 0;
    const int klast = has ? 31 - __clz(vmask) : 0;
    const bool starts = has && ((sb >> kfirst) & 1u);
    uint32_t rank = cnt + (uint32_t)(inc - c0) - 1u;  // row in progress before the lane
    const uint32_t first_rank = rank + (starts ? 1u : 0u);
    int nb = 0;
    AT head = (AT)0, acc = (AT)0;
    // prod[] is +0 outside the real positions of vmask, and a sum that starts at +0 never
    // changes by adding +0: every position is added without a test
#pragma unroll
    for (int k = 0; k < VM; k++) {
        if (k < (int)V) {
            if ((sb >> k) & 1u) {
                if (k != kfirst) {
                    if (nb == 0) head = acc;
                    else store_y<YT, AT>(y + (EMPTY ? __ldg(a.ne + rank) : rank), acc);
                    nb++;
                }
                rank++;
                acc = (AT)0;
            }
            acc = add_rn(acc, (AT)prod[k]);
        }
    }
    (void)rb;
    const uint32_t last_rank = rank;
    bool next_start;
    if (klast + 1 < (int)V) next_start = (sraw >> (klast + 1)) & 1u;
    else next_start = (lane < 31) ? (nxt_lane & 1u) : (nxt_win & 1u);
    if (qb + (uint32_t)klast + 1 >= a.npos) next_start = true;
    const bool ends = has && next_start;

    const bool rf = has && (nb > 0 || starts);
    const unsigned rmask = __ballot_sync(kFull, rf);
    const unsigned le = rmask & (kFull >> (31 - lane));
    const int sstart = le ? 31 - __clz(le) : -1;
    AT S = acc;
    seg_scan<SPAN>(S, lane, sstart);
    if (sstart < 0) S = add_rn(S, carry);
    AT E = __shfl_up_sync(kFull, S, 1);
    if (lane == 0) E = carry;
    if (has) {
        if (nb > 0)
            store_y<YT, AT>(y + (EMPTY ? __ldg(a.ne + first_rank) : first_rank),
                            starts ? head : add_rn(head, E));
        if (ends) store_y<YT, AT>(y + (EMPTY ? __ldg(a.ne + last_rank) : last_rank), S);
    }
    carry = __shfl_sync(kFull, S, 31);
    cnt += total;
}

// Index in a baked ax ([w values | w x] per tile) of the value of slot s: shifts for the
// power-of-two widths every layout here uses, division otherwise.
__device__ __forceinline__ uint32_t baked_index(uint32_t s, uint32_t w)
{
    if ((w & (w - 1u)) == 0u) {
        const uint32_t lg = (uint32_t)__ffs(w) - 1u;
        return ((s >> lg) << (lg + 1u)) + (s & (w - 1u));
    }
    return (s / w) * 2u * w + s % w;
}

// Products of the lane's real positions, loaded from global memory (vectorised streaming
// loads for direct layouts, one coalesced load per tile row for tiled layouts).
// First slot of a lane's tile column in a tiled layout whose windows hold th positions per
// lane (V = th): the lane's positions qb = 32 V w + V lane are tile column u = 32 w + lane
// counted over all tiles, so the tile is u / thw and the column u % thw -- shifts for the
// power-of-two widths the reference uses, one division otherwise.
__device__ __forceinline__ uint32_t tile_slot0(const RowsArgs &a, uint32_t w, int lane)
{
    const uint32_t u = w * 32u + (uint32_t)lane;
    uint32_t t, c;
    if ((a.thw & (a.thw - 1u)) == 0u) {
        const uint32_t lg = (uint32_t)__ffs(a.thw) - 1u;
        t = u >> lg;
        c = u & (a.thw - 1u);
    } else {
        t = u / a.thw;
        c = u - t * a.thw;
    }
    return t * a.th * a.thw + c;
}

template <class VT, class IT, class XT, class PT, int VM, bool TILED, bool BAKED>
__device__ __forceinline__ void products_ldg(const RowsArgs &a, uint32_t w, uint32_t qb,
                                             uint32_t V, uint32_t rb, PT (&prod)[VM])
{
    const VT *val = static_cast<const VT *>(a.val);
    const IT *col = static_cast<const IT *>(a.col);
    const XT *x = static_cast<const XT *>(a.x);
    const double *ax = static_cast<const double *>(a.val);
#pragma unroll
    for (int k = 0; k < VM; k++) prod[k] = (PT)0;
    if (!rb) return;
    const uint32_t ts0 = TILED ? tile_slot0(a, w, (int)(threadIdx.x & 31u)) : 0u;
    if constexpr (BAKED) {
#pragma unroll
        for (int k = 0; k < VM; k++) {
            if (k < (int)V && ((rb >> k) & 1u)) {
                uint32_t s = qb + k;
                if constexpr (TILED) s = ts0 + (uint32_t)k * a.thw;
                const uint32_t ai = baked_index(s, a.axw);
                prod[k] = (PT)mul_rn(__ldcs(ax + ai), __ldcs(ax + ai + a.axw));
            }
        }
    } else if constexpr (!TILED) {
        VT v[VM];
        IT c[VM];
        if (qb + VM <= a.nslots) {
            load_streams<VT, IT, VM>(a.wide != 0u, val + qb, col + qb, v, c);
        } else {  // stream tail: element loads, never past the last slot
#pragma unroll
            for (int k = 0; k < VM; k++) {
                v[k] = (VT)0;
                c[k] = 0;
                if ((rb >> k) & 1u) {
                    v[k] = ld_stream(val + qb + k);
                    c[k] = ld_stream(col + qb + k);
                }
            }
        }
        const uint32_t cbase = (sizeof(IT) == 2) ? __ldg(a.colbase + w) : 0u;
        XT xv[VM];
#pragma unroll
        for (int k = 0; k < VM; k++)
            xv[k] = ((rb >> k) & 1u) ? __ldg(x + (cbase + (uint32_t)c[k])) : (XT)0;
#pragma unroll
        for (int k = 0; k < VM; k++)
            if ((rb >> k) & 1u) prod[k] = mul_rn((PT)ValTraits<VT>::to_f64(v[k]), (PT)xv[k]);
    } else {
        const uint32_t s0 = ts0;
        VT v[VM];
        IT c[VM];
#pragma unroll
        for (int k = 0; k < VM; k++) {
            v[k] = (VT)0;
            c[k] = 0;
            if (k < (int)V && ((rb >> k) & 1u)) {
                v[k] = ld_stream(val + s0 + (uint32_t)k * a.thw);
                c[k] = ld_stream(col + s0 + (uint32_t)k * a.thw);
            }
        }
        XT xv[VM];
#pragma unroll
        for (int k = 0; k < VM; k++)
            xv[k] = (k < (int)V && ((rb >> k) & 1u)) ? __ldg(x + (uint32_t)c[k]) : (XT)0;
#pragma unroll
        for (int k = 0; k < VM; k++)
            if (k < (int)V && ((rb >> k) & 1u))
                prod[k] = mul_rn((PT)ValTraits<VT>::to_f64(v[k]), (PT)xv[k]);
    }
}

// One window's streams as loaded for a lane: start / real bits and the V value / column
// pairs (baked layouts: value and x halves), requested together.
template <class VT, class IT, int VM, bool BAKED>
struct WinData {
    uint32_t sraw, rraw;
    VT v[VM];
    IT c[VM];
    double xb[BAKED ? VM : 1];
};

template <class VT, class IT, int VM, bool TILED, bool BAKED, bool PADDED>
__device__ __forceinline__ void load_win(const RowsArgs &a, uint32_t w, int lane, uint32_t V,
                                         WinData<VT, IT, VM, BAKED> &d)
{
    const uint32_t qb = w * 32u * V + (uint32_t)lane * V;
    d.sraw = get_bits(a.sbits, qb, V);
    d.rraw = PADDED ? get_bits(a.rbits, qb, V) : 0xffffffffu;
    const VT *val = static_cast<const VT *>(a.val);
    const IT *col = static_cast<const IT *>(a.col);
    const uint32_t ts0 = TILED ? tile_slot0(a, w, lane) : 0u;
    if constexpr (BAKED) {
        const double *ax = static_cast<const double *>(a.val);
        if constexpr (!TILED && VM == 8) {
            // 8 dividing the tile width, a lane's 8 slots lie in one tile: its values and its
            // x are two runs of 8 consecutive doubles (two 32-byte loads each; slots past
            // npos are the last tile's zero fill, masked by the caller)
            if (a.wide && (a.axw & 7u) == 0u && qb < a.npos) {
                const uint32_t ai = baked_index(qb, a.axw);
                Load8W<double>::run(ax + ai, d.v);
                Load8W<double>::run(ax + ai + a.axw, d.xb);
                return;
            }
        }
#pragma unroll
        for (int k = 0; k < VM; k++) {
            d.v[k] = 0.0;
            d.xb[k] = 0.0;
            if (k < (int)V && qb + k < a.npos) {
                uint32_t s = qb + k;
                if constexpr (TILED) s = ts0 + (uint32_t)k * a.thw;
                const uint32_t ai = baked_index(s, a.axw);
                d.v[k] = __ldcs(ax + ai);
                d.xb[k] = __ldcs(ax + ai + a.axw);
            }
        }
    } else if constexpr (!TILED) {
        if (qb + VM <= a.nslots) {
            load_streams<VT, IT, VM>(a.wide != 0u, val + qb, col + qb, d.v, d.c);
        } else {  // stream tail: element loads, never past the last slot
#pragma unroll
            for (int k = 0; k < VM; k++) {
                d.v[k] = (VT)0;
                d.c[k] = 0;
                if (qb + k < a.npos) {
                    d.v[k] = ld_stream(val + qb + k);
                    d.c[k] = ld_stream(col + qb + k);
                }
            }
        }
    } else {
        const uint32_t s0 = ts0;
#pragma unroll
        for (int k = 0; k < VM; k++) {
            d.v[k] = (VT)0;
            d.c[k] = 0;
            if (k < (int)V && qb + k < a.npos) {
                d.v[k] = ld_stream(val + s0 + (uint32_t)k * a.thw);
                d.c[k] = ld_stream(col + s0 + (uint32_t)k * a.thw);
            }
        }
    }
}

// x gathers and products of the real positions rb of a loaded window (0 elsewhere).
template <class VT, class IT, class XT, class PT, int VM, bool BAKED>
__device__ __forceinline__ void win_products(const RowsArgs &a, uint32_t w, uint32_t V,
                                             const WinData<VT, IT, VM, BAKED> &d, uint32_t rb,
                                             PT (&prod)[VM])
{
    if constexpr (BAKED) {
#pragma unroll
        for (int k = 0; k < VM; k++)
            prod[k] = (k < (int)V && ((rb >> k) & 1u)) ? (PT)mul_rn(d.v[k], d.xb[k]) : (PT)0;
    } else {
        const XT *x = static_cast<const XT *>(a.x);
        const uint32_t cbase = (sizeof(IT) == 2) ? __ldg(a.colbase + w) : 0u;
        XT xv[VM];
#pragma unroll
        for (int k = 0; k < VM; k++)
            xv[k] = (k < (int)V && ((rb >> k) & 1u)) ? __ldg(x + (cbase + (uint32_t)d.c[k]))
                                                      : (XT)0;
#pragma unroll
        for (int k = 0; k < VM; k++)
            prod[k] = (k < (int)V && ((rb >> k) & 1u))
                          ? mul_rn((PT)ValTraits<VT>::to_f64(d.v[k]), (PT)xv[k])
                          : (PT)0;
    }
}

// Windows from `w` on, past the warp's range end w1, until its last row ends.
template <class VT, class IT, class XT, class PT, class AT, class YT, int VM, bool TILED,
          bool BAKED, bool PADDED, bool EMPTY>
__device__ __forceinline__ void finish_overhang(const RowsArgs &a, YT *y, int lane, uint32_t w,
                                                uint32_t V, uint32_t FULLV, uint32_t cnt,
                                                AT carry)
{
    for (; w < a.nwin; w++) {
        const uint32_t W = w * 32u * V;
        const uint32_t qb = W + (uint32_t)lane * V;
        const uint32_t sraw = get_bits(a.sbits, qb, V);
        const WinCtl ctl = window_ctl(lane, W, V, FULLV, a.npos, sraw, true, true);
        const uint32_t rb = PADDED ? (get_bits(a.rbits, qb, V) & ctl.vmask) : ctl.vmask;
        PT prod[VM];
        products_ldg<VT, IT, XT, PT, VM, TILED, BAKED>(a, w, qb, V, rb, prod);
        window_reduce<AT, YT, VM, EMPTY, PT, kBallotRanks<VM, TILED>,
                      kScanSpan<VT, VM, TILED, BAKED>>(
            a, y, lane, W, V, sraw, ctl.vmask, rb, prod, cnt, carry);
        if (ctl.slanes != 0u) break;  // the last row ended in this window
    }
}

// ---------------------------------------------------------------------------------------
// LDG-staged kernel (every layout).  VT value storage, IT column storage (u32 or u16
// offsets), XT x type, PT product type, AT accumulation type, YT output type.  VM =
// positions per lane for direct layouts and the upper bound of th for tiled ones.  PADDED:
// the layout has padding positions (real-bit map).  EMPTY: some rows are empty.
template <class VT, class IT, class XT, class PT, class AT, class YT, int VM, bool TILED,
          bool BAKED, bool PADDED, bool EMPTY>
__device__ __forceinline__ void rows_generic(const RowsArgs &a)
{
    const int lane = threadIdx.x & 31;
    YT *y = static_cast<YT *>(a.y);
    const uint32_t V = TILED ? a.th : (uint32_t)VM;
    const uint32_t FULLV = (V >= 32) ? 0xffffffffu : ((1u << V) - 1u);
    const uint32_t WS = 32u * V;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);

    if constexpr (EMPTY) {
        for (uint32_t i = gw * 32 + lane; i < a.n_empty; i += nwarps * 32)
            store_y<YT, AT>(y + __ldg(a.empty + i), (AT)0);
    }
    const uint32_t nranges = (a.nwin + a.wpw - 1) / a.wpw;
    for (uint32_t rg = gw; rg < nranges; rg += nwarps) {
        const uint32_t w0 = rg * a.wpw;
        const uint32_t w1 = min(w0 + a.wpw, a.nwin);
        uint32_t cnt = __ldg(a.wcount + w0);  // row starts before this range
        bool seen = (w0 == 0);                // a row start has been met in the range
        AT carry = (AT)0;
        for (uint32_t w = w0; w < w1; w++) {
            // bits and streams are requested together (the streams do not wait for the
            // bits), then the x gathers
            WinData<VT, IT, VM, BAKED> cur;
            load_win<VT, IT, VM, TILED, BAKED, PADDED>(a, w, lane, V, cur);
            const uint32_t W = w * WS;
            const WinCtl ctl = window_ctl(lane, W, V, FULLV, a.npos, cur.sraw, seen, false);
            if (ctl.skip) continue;  // all of it continues an earlier warp's row
            const uint32_t rb = cur.rraw & ctl.vmask;
            PT prod[VM];
            win_products<VT, IT, XT, PT, VM, BAKED>(a, w, V, cur, rb, prod);
            window_reduce<AT, YT, VM, EMPTY, PT, kBallotRanks<VM, TILED>,
                          kScanSpan<VT, VM, TILED, BAKED>>(
                a, y, lane, W, V, cur.sraw, ctl.vmask, rb, prod, cnt, carry);
            seen = true;
        }
        if (seen)
            finish_overhang<VT, IT, XT, PT, AT, YT, VM, TILED, BAKED, PADDED, EMPTY>(
                a, y, lane, w1, V, FULLV, cnt, carry);
    }
}

template <class VT, class IT, class XT, class PT, class AT, class YT, int VM, bool TILED,
          bool BAKED, bool PADDED, bool EMPTY>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_rows(const RowsArgs a)
{
    rows_generic<VT, IT, XT, PT, AT, YT, VM, TILED, BAKED, PADDED, EMPTY>(a);
}
// The same kernel in blocks of 2 warps, for the FP64 layouts where that measured faster
// (the same bits): direct layouts, i.e. CSR and COM tileH 1 (power-law CSR 324.3 ->
// 323.0 us, 27-point stencil 321.3 -> 313.7; drop-in gaxtch1 205 -> 198.5, 307.5 -> 295.3)
// and tiled tileH 2 (power-law COM th=2 402 -> 389.5, stencil 575 -> 551).  Tiled tileH
// 4 / 8 / 16 stay in blocks of 8 warps, where 2-warp blocks were slower (power-law COM
// th=4 357 -> 394 at 56 registers and 357 -> 366 at the same 48, th=8 345 -> 367, th=16
// 623 -> 675).  The minimum block counts cap the registers at 48 (4 positions per lane) and
// 56 (8 per lane, tileH 2) without spills on the run-time-x forms (32 registers for 4 per
// lane would spill 16-36 bytes).  FP32 / BF16 values keep blocks of 8 and the five-level
// scan: with both, CSR FP32 on the 27-point stencil 213.5 -> 237.0 us, on the power-law
// 310 -> 322; BF16 on the power-law 299 -> 342.
template <class VT, int VM, bool TILED>
constexpr bool kGenericSmallBlocks = std::is_same<VT, double>::value && (!TILED || VM == 2);
template <int VM, bool TILED> constexpr int kGenericMinBlocks2 = (!TILED && VM == 4) ? 21 : 18;
template <class VT, class IT, class XT, class PT, class AT, class YT, int VM, bool TILED,
          bool BAKED, bool PADDED, bool EMPTY>
__global__ void __launch_bounds__(64, kGenericMinBlocks2<VM, TILED>) k_rows2(const RowsArgs a)
{
    rows_generic<VT, IT, XT, PT, AT, YT, VM, TILED, BAKED, PADDED, EMPTY>(a);
}

// ---------------------------------------------------------------------------------------
// NT consecutive 32-wide tiles w .. w+NT-1 (window = tile, lane l owns tile column l, V =
// tileH positions of one row) that a warp owns outright: a row start was met before them
// and all lie inside its range.  The column loads and x gathers of all NT tiles issue
// before any sum and their segmented scans interleave, so a lane keeps NT*V gathers in
// flight where one tile gives V.  The value loads issue after the gathers: they arrive
// while the gathers are in flight, and their registers are not held across the column
// round trip.  Each tile's sums, and their order, are those of the single-tile path.
template <class VT, class IT, class XT, class PT, class AT, class YT, int V, int NT,
          bool PADDED, bool EMPTY>
__device__ __forceinline__ void owned_tiles(const RowsArgs &a, YT *y, int lane, unsigned mine,
                                            uint32_t w, uint32_t &cnt, AT &carry)
{
    constexpr uint32_t WS = 32u * V;
    constexpr uint32_t FULLV = (V >= 32) ? 0xffffffffu : ((1u << V) - 1u);
    const VT *val = static_cast<const VT *>(a.val);
    const IT *col = static_cast<const IT *>(a.col);
    const XT *x = static_cast<const XT *>(a.x);
    IT c[NT][V];
    uint32_t rb[NT];
    unsigned smask[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) {
        const uint32_t s0 = (w + (uint32_t)t) * WS + (uint32_t)lane;
#pragma unroll
        for (int k = 0; k < V; k++) c[t][k] = ld_stream(col + s0 + 32u * (uint32_t)k);
        // V divides 32 and qb is a multiple of V: the lane's bits sit in one word
        const uint32_t qb = (w + (uint32_t)t) * WS + (uint32_t)lane * V;
        const bool inb = qb < a.npos;
        rb[t] = inb ? FULLV : 0u;
        if constexpr (PADDED)
            rb[t] = inb ? ((__ldg(a.rbits + (qb >> 5)) >> (qb & 31)) & FULLV) : 0u;
        smask[t] = __ballot_sync(kFull, inb && ((__ldg(a.sbits + (qb >> 5)) >> (qb & 31)) & 1u));
    }
    XT xv[NT][V];
#pragma unroll
    for (int t = 0; t < NT; t++)
#pragma unroll
        for (int k = 0; k < V; k++)
            xv[t][k] = ((rb[t] >> k) & 1u) ? __ldg(x + (uint32_t)c[t][k]) : (XT)0;
    VT v[NT][V];
#pragma unroll
    for (int t = 0; t < NT; t++)
#pragma unroll
        for (int k = 0; k < V; k++)
            v[t][k] = ld_stream(val + (w + (uint32_t)t) * WS + (uint32_t)lane + 32u * (uint32_t)k);
    AT S[NT];
    int sstart[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) {
        AT acc = (AT)0;
#pragma unroll
        for (int k = 0; k < V; k++)
            acc = add_rn(acc, (AT)(((rb[t] >> k) & 1u)
                                       ? mul_rn((PT)ValTraits<VT>::to_f64(v[t][k]), (PT)xv[t][k])
                                       : (PT)0));
        S[t] = acc;
        const unsigned le = smask[t] & mine;
        sstart[t] = le ? 31 - __clz(le) : -1;
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
        for (int t = 0; t < NT; t++) {
            AT u = __shfl_up_sync(kFull, S[t], d);
            if (lane >= d && lane - d >= sstart[t]) S[t] = add_rn(S[t], u);
        }
    }
#pragma unroll
    for (int t = 0; t < NT; t++) {
        if (sstart[t] < 0) S[t] = add_rn(S[t], carry);
        const uint32_t qb = (w + (uint32_t)t) * WS + (uint32_t)lane * V;
        bool nxt;
        if (lane < 31) nxt = (smask[t] >> (lane + 1)) & 1u;
        else if (t + 1 < NT) nxt = smask[t + 1] & 1u;  // lane 0 of the next tile
        else nxt = (qb + V < a.npos) ? ((__ldg(a.sbits + ((qb + V) >> 5)) >> ((qb + V) & 31)) & 1u)
                                     : true;
        if (qb + V >= a.npos) nxt = true;
        if (qb < a.npos && nxt) {
            const uint32_t rank = cnt + (uint32_t)__popc(smask[t] & mine) - 1u;
            store_y<YT, AT>(y + (EMPTY ? __ldg(a.ne + rank) : rank), S[t]);
        }
        carry = __shfl_sync(kFull, S[t], 31);
        cnt += (uint32_t)__popc(smask[t]);
    }
}

// ---------------------------------------------------------------------------------------
// Aligned kernel.  In the UNC layouts every row starts on a tile column (tileH > 1: a
// multiple of th positions) or a tile (tileH = 1: a multiple of tileHW), and in AXC on a
// brick: with V positions per lane and V dividing that alignment, a lane never holds two
// rows.  Its V products are one partial sum, the window's row starts are one ballot of the
// lanes' first bits, and a row's lanes are joined by one segmented scan -- close to the
// instruction count of a row-per-lane kernel while keeping the AXT tile layout's
// coalesced loads.
//
// T32: tiled layouts with tileHW = 32 and tileH = V, where a window of 32 lanes x V positions
// is exactly one tile and lane l owns its column l: element k of that column is slot
// w * 32V + 32k + l, with no division by the runtime tile size.
//
// NT > 1 (32-wide run-time-x tiles of tileH 2 and 4, x gathers close to random): the
// windows a warp owns outright go NT at a time through owned_tiles.
template <class VT, class IT, class XT, class PT, class AT, class YT, int V, bool TILED,
          bool BAKED, bool PADDED, bool EMPTY, bool T32, bool EARLY, int NT>
__device__ __forceinline__ void rows_aligned(const RowsArgs &a)
{
    const int lane = threadIdx.x & 31;
    YT *y = static_cast<YT *>(a.y);
    const VT *val = static_cast<const VT *>(a.val);
    const IT *col = static_cast<const IT *>(a.col);
    const XT *x = static_cast<const XT *>(a.x);
    const double *ax = static_cast<const double *>(a.val);
    constexpr uint32_t WS = 32u * V;
    constexpr uint32_t FULLV = (V >= 32) ? 0xffffffffu : ((1u << V) - 1u);
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const unsigned mine = 0xffffffffu >> (31 - lane);  // lanes 0..lane

    if constexpr (EMPTY) {
        for (uint32_t i = gw * 32 + lane; i < a.n_empty; i += nwarps * 32)
            store_y<YT, AT>(y + __ldg(a.empty + i), (AT)0);
    }
    const uint32_t nranges = (a.nwin + a.wpw - 1) / a.wpw;
    for (uint32_t rg = gw; rg < nranges; rg += nwarps) {
        const uint32_t w0 = rg * a.wpw;
        const uint32_t w1 = min(w0 + a.wpw, a.nwin);
        uint32_t cnt = __ldg(a.wcount + w0);
        bool seen = (w0 == 0);
        AT carry = (AT)0;
        for (uint32_t w = w0; w < a.nwin; w++) {
            if constexpr (NT > 1) {
                static_assert(EARLY && !BAKED, "tile groups are for 32-wide run-time-x tiles");
                if (seen && w + NT <= w1) {
                    owned_tiles<VT, IT, XT, PT, AT, YT, V, NT, PADDED, EMPTY>(a, y, lane, mine, w,
                                                                           cnt, carry);
                    w += NT - 1;
                    continue;
                }
            }
            const bool over = w >= w1;
            if (over && !seen) break;
            const uint32_t qb = w * WS + (uint32_t)lane * V;
            const bool inb = qb < a.npos;  // rows end on V boundaries: whole lanes only
            // EARLY: the tile's value and column slots (every slot of a tile exists) and the
            // real bits load together with the start bits, not after them
            [[maybe_unused]] VT ev[V];
            [[maybe_unused]] IT ec[V];
            [[maybe_unused]] uint32_t erb = FULLV;
            if constexpr (EARLY) {
                static_assert(TILED && T32, "early loads are for 32-wide tiles");
                const uint32_t s0 = w * WS + (uint32_t)lane;
#pragma unroll
                for (int k = 0; k < V; k++) {
                    ev[k] = ld_stream(val + s0 + 32u * (uint32_t)k);
                    ec[k] = ld_stream(col + s0 + 32u * (uint32_t)k);
                }
                // V divides 32 and qb is a multiple of V: the lane's bits sit in one word
                if constexpr (PADDED)
                    erb = inb ? ((__ldg(a.rbits + (qb >> 5)) >> (qb & 31)) & FULLV) : 0u;
            }
            const bool st = inb && ((__ldg(a.sbits + (qb >> 5)) >> (qb & 31)) & 1u);
            const unsigned smask = __ballot_sync(kFull, st);
            unsigned vl = __ballot_sync(kFull, inb);
            if (!seen || over) {
                if (smask == 0u) {
                    if (!seen) continue;  // all of it continues an earlier warp's row
                } else {
                    const unsigned before = (1u << (__ffs(smask) - 1)) - 1u;
                    vl = seen ? (vl & before) : (vl & ~before);
                }
            }
            const bool valid = (vl >> lane) & 1u;
            uint32_t rb = valid ? FULLV : 0u;
            if constexpr (EARLY) rb &= erb;
            else if constexpr (PADDED) rb &= get_bits(a.rbits, qb, V);
            // ---- the lane's partial sum (loads and gathers of real positions only)
            AT acc = (AT)0;
            if (rb) {
                PT p[V];
                if constexpr (BAKED) {
#pragma unroll
                    for (int k = 0; k < V; k++) {
                        p[k] = (PT)0;
                        if ((rb >> k) & 1u) {
                            uint32_t s = qb + k;
                            if constexpr (TILED && T32) {
                                s = w * WS + 32u * (uint32_t)k + (uint32_t)lane;
                            } else if constexpr (TILED) {
                                s = tile_slot0(a, w, lane) + (uint32_t)k * a.thw;
                            }
                            const uint32_t ai = T32 ? (s >> 5) * 64u + (s & 31u)
                                                    : baked_index(s, a.axw);
                            p[k] = (PT)mul_rn(__ldcs(ax + ai), __ldcs(ax + ai + a.axw));
                        }
                    }
                } else {
                    VT v[V];
                    IT c[V];
                    if constexpr (EARLY) {
#pragma unroll
                        for (int k = 0; k < V; k++) {
                            v[k] = ev[k];
                            c[k] = ec[k];
                        }
                    } else if constexpr (TILED) {
                        uint32_t s0, stride;
                        if constexpr (T32) {
                            s0 = w * WS + (uint32_t)lane;
                            stride = 32u;
                        } else {
                            s0 = tile_slot0(a, w, lane);
                            stride = a.thw;
                        }
#pragma unroll
                        for (int k = 0; k < V; k++) {
                            v[k] = (VT)0;
                            c[k] = 0;
                            if ((rb >> k) & 1u) {
                                v[k] = ld_stream(val + s0 + (uint32_t)k * stride);
                                c[k] = ld_stream(col + s0 + (uint32_t)k * stride);
                            }
                        }
                    } else {
                        bool whole = false;
                        if constexpr (V == 8) {
                            // the lane's whole group (padding slots included, in bounds) in
                            // 32-byte requests; padding products are masked below
                            if (a.wide && qb + 8u <= a.nslots) {
                                load8_streams<VT, IT>(true, val + qb, col + qb, v, c);
                                whole = true;
                            }
                        }
#pragma unroll
                        for (int k = 0; k < V; k++) {
                            if (whole) break;
                            v[k] = (VT)0;
                            c[k] = 0;
                            if ((rb >> k) & 1u) {
                                v[k] = ld_stream(val + qb + k);
                                c[k] = ld_stream(col + qb + k);
                            }
                        }
                    }
                    const uint32_t cbase = (sizeof(IT) == 2) ? __ldg(a.colbase + w) : 0u;
                    XT xv[V];
#pragma unroll
                    for (int k = 0; k < V; k++)
                        xv[k] = ((rb >> k) & 1u) ? __ldg(x + (cbase + (uint32_t)c[k])) : (XT)0;
#pragma unroll
                    for (int k = 0; k < V; k++)
                        p[k] = ((rb >> k) & 1u)
                                   ? mul_rn((PT)ValTraits<VT>::to_f64(v[k]), (PT)xv[k])
                                   : (PT)0;
                }
#pragma unroll
                for (int k = 0; k < V; k++) acc = add_rn(acc, (AT)p[k]);
            }
            // ---- join the lanes of each row, write the rows that end in this window
            const unsigned sm = smask & vl;
            const unsigned le = sm & mine;
            const int sstart = le ? 31 - __clz(le) : -1;
            AT S = acc;
            // span-limited for FP64 with x gathered at run time, one tile per step
            // (power-law UNC th=8 335.0 -> 331.7 us, th=16 365.5 -> 363.9, AXC 433.6 ->
            // 429.5; 27-point stencil UNC th=4 276.0 -> 270.3, th=2 363.0 -> 359.2, AXC
            // 325.2 -> 321.2); the two-tile kernel (power-law UNC th=4 299.0 -> 299.7 with
            // it, th=2 325.6 -> 326.6) and the baked layouts (drop-in gaxtuh th=4 191 ->
            // 192) keep the full scan
            seg_scan<std::is_same<VT, double>::value && !BAKED && NT == 1>(S, lane, sstart);
            if (sstart < 0) S = add_rn(S, carry);
            bool nxt;
            if (lane < 31) nxt = (smask >> (lane + 1)) & 1u;
            else nxt = (qb + V < a.npos) ? ((__ldg(a.sbits + ((qb + V) >> 5)) >> ((qb + V) & 31)) & 1u)
                                         : true;
            if (qb + V >= a.npos) nxt = true;
            if (valid && nxt) {
                const uint32_t rank = cnt + (uint32_t)__popc(le) - 1u;
                store_y<YT, AT>(y + (EMPTY ? __ldg(a.ne + rank) : rank), S);
            }
            carry = __shfl_sync(kFull, S, 31);
            cnt += (uint32_t)__popc(sm);
            seen = true;
            if (over && smask != 0u) break;  // the range's last row ended in this window
        }
    }
}

template <class VT, class IT, class XT, class PT, class AT, class YT, int V, bool TILED,
          bool BAKED, bool PADDED, bool EMPTY, bool T32 = false, bool EARLY = false>
__global__ void __launch_bounds__(256) k_rows_aligned(const RowsArgs a)
{
    rows_aligned<VT, IT, XT, PT, AT, YT, V, TILED, BAKED, PADDED, EMPTY, T32, EARLY, 1>(a);
}
// The same kernel in blocks of 2 warps, for the 32-wide tiles where that measured faster:
// tileH 16 (power-law 458.8 -> 365.2 us, 27-point stencil 385.7 -> 359.2; 80 registers, 12
// blocks per SM) and tileH 8 with x baked in (drop-in gaxtuh th=8 218.2 -> 211.9); slower
// or level elsewhere (run-time-x th=8 on the stencil 321.7 -> 326.6, 320.4 -> 324.5 with the
// span-limited scan, on the power-law 331.6 either way; th=4 275.8 -> 282.6, baked th=4
// 193.6 -> 205.5; the direct AXC / UNC th=1 hw32 layouts at the same 32 / 40 registers:
// power-law 430 -> 433, stencil 321.8 -> 322.7).
template <int V, bool BAKED> constexpr bool kAlignedSmallBlocks = V == 16 || (V == 8 && BAKED);
template <class VT, class IT, class XT, class PT, class AT, class YT, int V, bool TILED,
          bool BAKED, bool PADDED, bool EMPTY, bool T32 = false, bool EARLY = false>
__global__ void __launch_bounds__(64, V == 16 ? 12 : 20) k_rows_aligned2(const RowsArgs a)
{
    rows_aligned<VT, IT, XT, PT, AT, YT, V, TILED, BAKED, PADDED, EMPTY, T32, EARLY, 1>(a);
}

// Two owned tiles per step.  Register caps: 48 for tileH = 4 (40 warps per SM), 40 for
// tileH = 2 (48 warps); uncapped the compiler takes 56-64 and the x gathers in flight per SM
// fall.  TileH 4 at 40 registers (48 warps) spills 32 bytes: power-law 299.9 -> 323.6 us.
constexpr int kGroupTiles = 2;
// Blocks of 2 warps (one warp range each): a block's slot frees as soon as its two ranges
// end, where a block of 8 waits for the slowest of 8 (power-law th=4 303.1 -> 298.6 us, 4
// warps 299.4; th=2 unchanged).  The same registers: 20 / 24 blocks per SM.
constexpr int kGroupedWarps = 2;
template <class VT, class IT, class XT, class PT, class AT, class YT, int V, bool PADDED,
          bool EMPTY>
__global__ void __launch_bounds__(32 * kGroupedWarps, (V == 2 ? 48 : 40) / kGroupedWarps)
    k_rows_grouped(const RowsArgs a)
{
    rows_aligned<VT, IT, XT, PT, AT, YT, V, true, false, PADDED, EMPTY, true, true,
                 kGroupTiles>(a);
}

// ---------------------------------------------------------------------------------------
// Striped kernel for the direct (tileH = 1) layouts: lane L takes position 32c + L of each
// 32-position chunk c, so every load instruction of the warp is one contiguous 256 B
// (values) / 128 B (columns) access and the chunk's row structure is a single broadcast
// word of the start bitmap.  Each step handles SU chunks: all their stream loads, then all
// their x gathers, then the per-chunk segmented scans -- many independent requests per
// warp, few registers, full occupancy.  Ranges are whole windows of the plan (32*V
// positions) so the plan's per-window start counts give each range its first row rank.
constexpr int kStripeU = 4;

// One chunk after its loads and gathers: ownership masks, segmented scan of the lanes'
// products, y writes of the rows that end in the chunk, carry.  Returns false once the
// warp's last row has ended past its range ("over").
template <class AT, class YT, class PT, bool EMPTY>
__device__ __forceinline__ bool stripe_chunk(const RowsArgs &a, YT *y, int lane, unsigned lt,
                                             uint32_t ch, uint32_t nchunk, bool over,
                                             uint32_t word, uint32_t vm, PT prod, uint32_t &cnt,
                                             bool &seen, AT &carry)
{
    uint32_t vmw = vm;
    const uint32_t sw0 = word & vmw;
    if (!seen || over) {
        if (sw0 == 0u) {
            if (!seen) return !over;  // all of it continues an earlier warp's row
        } else {
            const uint32_t below = (1u << (__ffs(sw0) - 1)) - 1u;
            vmw = seen ? (vmw & below) : (vmw & ~below);
        }
    }
    const uint32_t sw = word & vmw;
    const unsigned mine = lt | (1u << lane);
    const bool valid = (vmw >> lane) & 1u;
    const unsigned le = sw & mine;
    const int sstart = le ? 31 - __clz(le) : -1;
    AT S = valid ? (AT)prod : (AT)0;
    seg_scan<false>(S, lane, sstart);
    if (sstart < 0) S = add_rn(S, carry);
    // does the row in progress at this lane end here?
    bool nxt;
    if (lane < 31) nxt = (word >> (lane + 1)) & 1u;
    else nxt = (ch + 1 < nchunk) ? (__ldg(a.sbits + ch + 1) & 1u) : true;
    if (ch * 32u + (uint32_t)lane + 1u >= a.npos) nxt = true;
    if (valid && nxt) {
        const uint32_t rank = cnt + (uint32_t)__popc(sw & mine) - 1u;
        store_y<YT, AT>(y + (EMPTY ? __ldg(a.ne + rank) : rank), S);
    }
    carry = __shfl_sync(kFull, S, 31);
    cnt += (uint32_t)__popc(sw);
    seen = true;
    return !(over && sw0 != 0u);
}

template <class VT, class IT, class XT, class PT, class AT, class YT, bool BAKED, bool PADDED,
          bool EMPTY>
__global__ void __launch_bounds__(256) k_rows_striped(const RowsArgs a)
{
    const int lane = threadIdx.x & 31;
    YT *y = static_cast<YT *>(a.y);
    const VT *val = static_cast<const VT *>(a.val);
    const IT *col = static_cast<const IT *>(a.col);
    const XT *x = static_cast<const XT *>(a.x);
    const double *ax = static_cast<const double *>(a.val);
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t cpwin = a.V;  // chunks per plan window
    const unsigned lt = (1u << lane) - 1u;  // lanes below this one

    if constexpr (EMPTY) {
        for (uint32_t i = gw * 32 + lane; i < a.n_empty; i += nwarps * 32)
            store_y<YT, AT>(y + __ldg(a.empty + i), (AT)0);
    }
    const uint32_t nchunk = (a.npos + 31) / 32;
    // stream loads of chunk ch for this lane: start-bit word, in-bounds mask, real mask
    auto load_chunk = [&](uint32_t ch, uint32_t lim, uint32_t &word, uint32_t &vm,
                          uint32_t &rm, VT &v, IT &c, double &xb) {
        const uint32_t q = ch * 32u + (uint32_t)lane;
        const bool in = ch < lim;
        word = in ? __ldg(a.sbits + ch) : 0u;
        vm = !in ? 0u
             : (ch * 32u + 32u <= a.npos ? 0xffffffffu : ((1u << (a.npos - ch * 32u)) - 1u));
        rm = (PADDED ? (in ? __ldg(a.rbits + ch) : 0u) : 0xffffffffu) & vm;
        v = (VT)0;
        c = 0;
        xb = 0.0;
        if ((rm >> lane) & 1u) {
            if constexpr (BAKED) {
                const uint32_t ai = baked_index(q, a.axw);
                v = __ldcs(ax + ai);
                xb = __ldcs(ax + ai + a.axw);
            } else {
                v = ld_stream(val + q);
                c = ld_stream(col + q);
            }
        }
    };
    // x gather and product of the lane's position (0 when not real)
    auto product = [&](uint32_t ch, uint32_t rm, VT v, IT c, double xb) -> PT {
        if (!((rm >> lane) & 1u)) return (PT)0;
        if constexpr (BAKED) {
            return (PT)mul_rn(v, xb);
        } else {
            const uint32_t cbase = (sizeof(IT) == 2) ? __ldg(a.colbase + ch / cpwin) : 0u;
            return mul_rn((PT)ValTraits<VT>::to_f64(v), (PT)__ldg(x + (cbase + (uint32_t)c)));
        }
    };
    const uint32_t nranges = (a.nwin + a.wpw - 1) / a.wpw;
    for (uint32_t rg = gw; rg < nranges; rg += nwarps) {
        const uint32_t c0 = rg * a.wpw * cpwin;
        const uint32_t c1 = min(c0 + a.wpw * cpwin, nchunk);
        uint32_t cnt = __ldg(a.wcount + rg * a.wpw);  // row starts before the range
        bool seen = (c0 == 0);
        AT carry = (AT)0;
        // the range's own chunks, kStripeU at a time: all loads, then all gathers, then the
        // per-chunk scans
        for (uint32_t cb = c0; cb < c1; cb += kStripeU) {
            uint32_t word[kStripeU], vm[kStripeU], rm[kStripeU];
            VT v[kStripeU];
            IT c[kStripeU];
            double xb[kStripeU];
            PT prod[kStripeU];
#pragma unroll
            for (int u = 0; u < kStripeU; u++)
                load_chunk(cb + u, c1, word[u], vm[u], rm[u], v[u], c[u], xb[u]);
#pragma unroll
            for (int u = 0; u < kStripeU; u++) prod[u] = product(cb + u, rm[u], v[u], c[u], xb[u]);
#pragma unroll
            for (int u = 0; u < kStripeU; u++)
                if (cb + u < c1)
                    stripe_chunk<AT, YT, PT, EMPTY>(a, y, lane, lt, cb + u, nchunk, false,
                                                    word[u], vm[u], prod[u], cnt, seen, carry);
        }
        // past the range: one chunk at a time until the range's last row ends
        if (seen) {
            for (uint32_t ch = c1; ch < nchunk; ch++) {
                uint32_t word, vm, rm;
                VT v;
                IT c;
                double xb;
                load_chunk(ch, nchunk, word, vm, rm, v, c, xb);
                const PT p = product(ch, rm, v, c, xb);
                if (!stripe_chunk<AT, YT, PT, EMPTY>(a, y, lane, lt, ch, nchunk, true, word, vm,
                                                     p, cnt, seen, carry))
                    break;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// TMA-staged kernel for tiled layouts with 32-wide tiles (tileHW = 32, tileH = TH): a window
// is exactly one tile.  Each warp owns a contiguous range of tiles and keeps kTmaStages of
// them in flight in its shared-memory ring; stage layout: [val tile | col tile | start
// bits | real bits] (baked: [ax tile | start bits | real bits]).
template <class VT, class IT, int TH, bool BAKED, bool PADDED>
struct TmaStage {
    static constexpr uint32_t WS = 32u * TH;
    static constexpr uint32_t VAL = BAKED ? 2u * WS * 8u : WS * (uint32_t)sizeof(VT);
    static constexpr uint32_t COL = BAKED ? 0u : WS * (uint32_t)sizeof(IT);
    static constexpr uint32_t BITS = (uint32_t)TH * 4u;
    static constexpr uint32_t COPY = VAL + COL + BITS * (PADDED ? 2u : 1u);
    static constexpr uint32_t BYTES = (COPY + 127u) & ~127u;
    static constexpr uint32_t PER_WARP = BYTES * kTmaStages;
    static constexpr uint32_t SMEM = PER_WARP * kTmaWarps + kTmaWarps * kTmaStages * 8u;
};

template <class VT, class IT, class XT, class PT, class AT, class YT, int TH, bool BAKED,
          bool PADDED, bool EMPTY>
__global__ void __launch_bounds__(kTmaWarps * 32) k_rows_tma(const RowsArgs a)
{
    using ST = TmaStage<VT, IT, TH, BAKED, PADDED>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned char *ring = smem + wib * ST::PER_WARP;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kTmaWarps * ST::PER_WARP) +
                     wib * kTmaStages;
    YT *y = static_cast<YT *>(a.y);
    const XT *x = static_cast<const XT *>(a.x);
    constexpr uint32_t V = TH;
    constexpr uint32_t FULLV = (V >= 32) ? 0xffffffffu : ((1u << V) - 1u);
    constexpr uint32_t WS = ST::WS;
    const uint32_t nwarps = gridDim.x * kTmaWarps;
    const uint32_t gw = blockIdx.x * kTmaWarps + wib;

    if constexpr (EMPTY) {
        for (uint32_t i = gw * 32 + lane; i < a.n_empty; i += nwarps * 32)
            store_y<YT, AT>(y + __ldg(a.empty + i), (AT)0);
    }
    // contiguous, equal ranges of tiles (positions) per warp
    const uint32_t per = (a.nwin + nwarps - 1) / nwarps;
    const uint32_t w0 = gw * per;
    const uint32_t w1 = min(w0 + per, a.nwin);
    if (w0 >= w1) return;

    if (lane == 0) {
        for (int s = 0; s < kTmaStages; s++) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncwarp();
    auto issue = [&](uint32_t w, int s) {
        if (lane == 0) {
            unsigned char *st = ring + s * ST::BYTES;
            mbar_expect_tx(&bars[s], ST::COPY);
            if constexpr (BAKED) {
                bulk_g2s(st, static_cast<const double *>(a.val) + (size_t)w * 2u * WS, ST::VAL,
                         &bars[s]);
            } else {
                bulk_g2s(st, static_cast<const VT *>(a.val) + (size_t)w * WS, ST::VAL, &bars[s]);
                bulk_g2s(st + ST::VAL, static_cast<const IT *>(a.col) + (size_t)w * WS, ST::COL,
                         &bars[s]);
            }
            bulk_g2s(st + ST::VAL + ST::COL, a.sbits + (size_t)w * TH, ST::BITS, &bars[s]);
            if constexpr (PADDED)
                bulk_g2s(st + ST::VAL + ST::COL + ST::BITS, a.rbits + (size_t)w * TH, ST::BITS,
                         &bars[s]);
        }
    };
    const uint32_t npre = min((uint32_t)kTmaStages, w1 - w0);
    for (uint32_t i = 0; i < npre; i++) issue(w0 + i, (int)i);

    uint32_t cnt = __ldg(a.wcount + w0);
    bool seen = (w0 == 0);
    AT carry = (AT)0;
    uint32_t parity = 0;  // bit s: phase parity expected next at stage s
    for (uint32_t w = w0; w < w1; w++) {
        const int s = (int)((w - w0) % kTmaStages);
        if (!mbar_wait_bounded(&bars[s], (parity >> s) & 1u)) {
            // the copy never completed: report, drain what is in flight (bounded), leave
            if (lane == 0) atomicOr(a.status, 1u);
            for (uint32_t v = w; v < min(w + (uint32_t)kTmaStages, w1); v++) {
                const int t = (int)((v - w0) % kTmaStages);
                mbar_wait_bounded(&bars[t], (parity >> t) & 1u);
            }
            return;
        }
        parity ^= 1u << s;
        const unsigned char *st = ring + s * ST::BYTES;
        const uint32_t *sbw = reinterpret_cast<const uint32_t *>(st + ST::VAL + ST::COL);
        const uint32_t W = w * WS;
        const uint32_t lb = (uint32_t)lane * V;
        const uint32_t sraw = (sbw[lb >> 5] >> (lb & 31)) & FULLV;
        const WinCtl ctl = window_ctl(lane, W, V, FULLV, a.npos, sraw, seen, false);
        if (!ctl.skip) {
            uint32_t rb = ctl.vmask;
            if constexpr (PADDED) rb &= (sbw[TH + (lb >> 5)] >> (lb & 31));
            PT prod[TH];
            if constexpr (BAKED) {
                const double *sax = reinterpret_cast<const double *>(st);
#pragma unroll
                for (int k = 0; k < TH; k++)
                    prod[k] = ((rb >> k) & 1u)
                                  ? (PT)mul_rn(sax[2 * 32 * k + lane], sax[2 * 32 * k + 32 + lane])
                                  : (PT)0;
            } else {
                const VT *sv = reinterpret_cast<const VT *>(st);
                const IT *sc = reinterpret_cast<const IT *>(st + ST::VAL);
                XT xv[TH];
#pragma unroll
                for (int k = 0; k < TH; k++)
                    xv[k] = ((rb >> k) & 1u) ? __ldg(x + (uint32_t)sc[32 * k + lane]) : (XT)0;
#pragma unroll
                for (int k = 0; k < TH; k++)
                    prod[k] = ((rb >> k) & 1u)
                                  ? mul_rn((PT)ValTraits<VT>::to_f64(sv[32 * k + lane]), (PT)xv[k])
                                  : (PT)0;
            }
            window_reduce<AT, YT, TH, EMPTY, PT, kBallotRanks<TH, true>>(
                a, y, lane, W, V, sraw, ctl.vmask, rb, prod, cnt, carry);
            seen = true;
        }
        __syncwarp();
        if (w + kTmaStages < w1) {
            fence_proxy_async();  // our reads of this stage precede the next bulk write to it
            issue(w + kTmaStages, s);
        }
    }
    if (seen)
        finish_overhang<VT, IT, XT, PT, AT, YT, TH, true, BAKED, PADDED, EMPTY>(
            a, y, lane, w1, V, FULLV, cnt, carry);
}

// ---------------------------------------------------------------------------------------
template <class VT, class IT, class XT, class PT, class AT, class YT, int VM, bool TILED,
          bool BAKED>
gs_status launch_k(const RowsArgs &a, bool padded, cudaStream_t s)
{
    const uint32_t nranges = (a.nwin + a.wpw - 1) / a.wpw;
    uint32_t warps = nranges;
    if (a.n_empty) warps = max(warps, min((a.n_empty + 31) / 32, 148u * 64u));
    if (warps == 0) return GS_OK;
    uint32_t blocks = (warps + kWarpsPerBlock - 1) / kWarpsPerBlock;
    blocks = min(blocks, 148u * 256u);
    const bool empty = a.n_empty != 0;
    // Loading a window's streams a window ahead paid for tileH 2..4 while the tiled slots
    // were found by dividing by the tile size (COM th=4 on the power-law 423 -> 399 us); with
    // the division gone the 64 registers it needs cost more than it hides (power-law COM
    // th=4 380 -> 364 us without it, th=2 500 -> 476; drop-in gaxtch th=4 326 -> 295;
    // 27-point stencil th=4 478 -> 454), so every window loads just before its use.
    if constexpr (kGenericSmallBlocks<VT, VM, TILED>) {
#define GS_D(P, E)                                                                          \
    k_rows2<VT, IT, XT, PT, AT, YT, VM, TILED, BAKED, P, E><<<(warps + 1) / 2, 64, 0, s>>>(a)
        if (padded) {
            if (empty) GS_D(true, true); else GS_D(true, false);
        } else {
            if (empty) GS_D(false, true); else GS_D(false, false);
        }
#undef GS_D
        GS_CHECK_LAUNCH();
        return GS_OK;
    }
#define GS_L(P, E)                                                                          \
    k_rows<VT, IT, XT, PT, AT, YT, VM, TILED, BAKED, P, E><<<blocks, kWarpsPerBlock * 32, 0, s>>>(a)
    if (padded) {
        if (empty) GS_L(true, true); else GS_L(true, false);
    } else {
        if (empty) GS_L(false, true); else GS_L(false, false);
    }
#undef GS_L
    GS_CHECK_LAUNCH();
    return GS_OK;
}

template <class VT, class IT, class XT, class PT, class AT, class YT, int V, bool TILED,
          bool BAKED>
gs_status launch_aligned(const RowsArgs &a, bool padded, cudaStream_t s)
{
    const uint32_t nranges = (a.nwin + a.wpw - 1) / a.wpw;
    uint32_t warps = nranges;
    if (a.n_empty) warps = max(warps, min((a.n_empty + 31) / 32, 148u * 64u));
    if (warps == 0) return GS_OK;
    uint32_t blocks = min((warps + 7) / 8, 148u * 256u);
    const bool empty = a.n_empty != 0;
    const bool t32 = TILED && a.thw == 32 && a.th == (uint32_t)V;
    // 32-wide tiles with x gathered at run time load a tile's streams with its start bits,
    // not after them (power-law UNC th=4 324 -> 320 us, th=8 348 -> 337; 27-point stencil
    // th=4 334 -> 289, th=8 412 -> 322; the same bits).  The direct layouts keep the
    // dependent loads: there the early loads cost 8 registers (48 for 8 positions per
    // lane) and AXC on the power-law went 461 -> 558 us.
    // random x gathers on 32-wide tiles of tileH 2 or 4: two owned tiles per step
    // (power-law UNC th=4 318 -> 303 us, th=2 352 -> 326, the same bits; on the 27-point
    // stencil, whose gathers mostly hit lines already in L1, one tile per step stays faster:
    // th=4 276 against 301 us)
    if constexpr (TILED && !BAKED && (V == 2 || V == 4)) {
        if (t32 && a.grouped) {
            const uint32_t gblocks = (warps + kGroupedWarps - 1) / kGroupedWarps;
#define GS_G(P, E)                                                                          \
    k_rows_grouped<VT, IT, XT, PT, AT, YT, V, P, E><<<gblocks, 32 * kGroupedWarps, 0, s>>>(a)
            if (padded) {
                if (empty) GS_G(true, true); else GS_G(true, false);
            } else {
                if (empty) GS_G(false, true); else GS_G(false, false);
            }
#undef GS_G
            GS_CHECK_LAUNCH();
            return GS_OK;
        }
    }
#define GS_T32_LAUNCH(P, E)                                                                 \
    do {                                                                                    \
        if constexpr (TILED && kAlignedSmallBlocks<V, BAKED>)                               \
            k_rows_aligned2<VT, IT, XT, PT, AT, YT, V, TILED, BAKED, P, E, TILED,           \
                            TILED && !BAKED><<<(warps + 1) / 2, 64, 0, s>>>(a);             \
        else                                                                                \
            k_rows_aligned<VT, IT, XT, PT, AT, YT, V, TILED, BAKED, P, E, TILED,            \
                           TILED && !BAKED><<<blocks, 256, 0, s>>>(a);                      \
    } while (0)
#define GS_L(P, E)                                                                          \
    do {                                                                                    \
        if (t32)                                                                            \
            GS_T32_LAUNCH(P, E);                                                            \
        else                                                                                \
            k_rows_aligned<VT, IT, XT, PT, AT, YT, V, TILED, BAKED, P, E, false>            \
                <<<blocks, 256, 0, s>>>(a);                                                 \
    } while (0)
    if (padded) {
        if (empty) GS_L(true, true); else GS_L(true, false);
    } else {
        if (empty) GS_L(false, true); else GS_L(false, false);
    }
#undef GS_L
#undef GS_T32_LAUNCH
    GS_CHECK_LAUNCH();
    return GS_OK;
}

template <class VT, class IT, class XT, class PT, class AT, class YT, bool BAKED>
gs_status launch_striped(const RowsArgs &a, bool padded, cudaStream_t s)
{
    const uint32_t nranges = (a.nwin + a.wpw - 1) / a.wpw;
    uint32_t warps = nranges;
    if (a.n_empty) warps = max(warps, min((a.n_empty + 31) / 32, 148u * 64u));
    if (warps == 0) return GS_OK;
    uint32_t blocks = min((warps + 7) / 8, 148u * 256u);
    const bool empty = a.n_empty != 0;
#define GS_L(P, E) k_rows_striped<VT, IT, XT, PT, AT, YT, BAKED, P, E><<<blocks, 256, 0, s>>>(a)
    if (padded) {
        if (empty) GS_L(true, true); else GS_L(true, false);
    } else {
        if (empty) GS_L(false, true); else GS_L(false, false);
    }
#undef GS_L
    GS_CHECK_LAUNCH();
    return GS_OK;
}

template <class VT, class IT, class XT, class PT, class AT, class YT, int TH, bool BAKED,
          bool PADDED, bool EMPTY>
gs_status launch_tma_one(const RowsArgs &a, cudaStream_t s)
{
    using ST = TmaStage<VT, IT, TH, BAKED, PADDED>;
    auto kern = k_rows_tma<VT, IT, XT, PT, AT, YT, TH, BAKED, PADDED, EMPTY>;
    static int blocks_per_sm = -1;  // per instantiation, resolved on first launch
    static int sms = 0;
    if (blocks_per_sm < 0) {
        GS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ST::SMEM));
        int dev = 0;
        GS_CUDA(cudaGetDevice(&dev));
        GS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        int bps = 0;
        GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, kTmaWarps * 32,
                                                              ST::SMEM));
        blocks_per_sm = bps > 0 ? bps : 1;
    }
    uint32_t blocks = (uint32_t)(blocks_per_sm * sms);
    const uint32_t need = (a.nwin + kTmaWarps - 1) / kTmaWarps;
    if (need < blocks) blocks = max(need, 1u);
    kern<<<blocks, kTmaWarps * 32, ST::SMEM, s>>>(a);
    GS_CHECK_LAUNCH();
    return GS_OK;
}

template <class VT, class IT, class XT, class PT, class AT, class YT, int TH, bool BAKED>
gs_status launch_tma(const RowsArgs &a, bool padded, cudaStream_t s)
{
    const bool empty = a.n_empty != 0;
    if (padded) {
        if (empty) return launch_tma_one<VT, IT, XT, PT, AT, YT, TH, BAKED, true, true>(a, s);
        return launch_tma_one<VT, IT, XT, PT, AT, YT, TH, BAKED, true, false>(a, s);
    }
    if (empty) return launch_tma_one<VT, IT, XT, PT, AT, YT, TH, BAKED, false, true>(a, s);
    return launch_tma_one<VT, IT, XT, PT, AT, YT, TH, BAKED, false, false>(a, s);
}

template <class VT, class IT, class XT, class PT, class AT, class YT, bool BAKED>
gs_status launch_shape(const RowsArgs &a, bool tiled, bool padded, uint32_t flags,
                       cudaStream_t s)
{
    const bool tma = (flags & GS_FLAG_TMA) != 0;
    const bool striped = (flags & GS_FLAG_STRIPED) != 0;
    if constexpr (!std::is_same<VT, double>::value) {
        if (tiled) return fail(GS_ERR_UNSUPPORTED, "FP32/BF16 storage needs a tileH=1 layout");
        if (a.aligned && a.V == 8)
            return launch_aligned<VT, IT, XT, PT, AT, YT, 8, false, BAKED>(a, padded, s);
        if (a.V != kDirectV) return fail(GS_ERR_INVALID, "plan built for another shape");
        if (striped) return launch_striped<VT, IT, XT, PT, AT, YT, BAKED>(a, padded, s);
        return launch_k<VT, IT, XT, PT, AT, YT, 8, false, BAKED>(a, padded, s);
    } else {
        if (tiled) {
            if (tma && a.thw == 32 && a.status) {
                if (a.th == 4) return launch_tma<VT, IT, XT, PT, AT, YT, 4, BAKED>(a, padded, s);
                if (a.th == 8) return launch_tma<VT, IT, XT, PT, AT, YT, 8, BAKED>(a, padded, s);
                if (a.th == 16)
                    return launch_tma<VT, IT, XT, PT, AT, YT, 16, BAKED>(a, padded, s);
            }
            if (a.aligned) {
                switch (a.th) {
                case 2: return launch_aligned<VT, IT, XT, PT, AT, YT, 2, true, BAKED>(a, padded, s);
                case 4: return launch_aligned<VT, IT, XT, PT, AT, YT, 4, true, BAKED>(a, padded, s);
                case 8: return launch_aligned<VT, IT, XT, PT, AT, YT, 8, true, BAKED>(a, padded, s);
                case 16:
                    return launch_aligned<VT, IT, XT, PT, AT, YT, 16, true, BAKED>(a, padded, s);
                default: break;
                }
            }
            // tileH 2 on a kernel of 2 positions per lane, not 4 with half of them idle (COM
            // th=2: 46 registers and no spill against 48 and a spill; on the power-law 464 ->
            // 416 us, on the 27-point stencil 702 -> 572; drop-in gaxtch th=2 427 -> 386 and
            // 646 -> 579; same bits)
            if (a.th <= 2) return launch_k<VT, IT, XT, PT, AT, YT, 2, true, BAKED>(a, padded, s);
            if (a.th <= 4) return launch_k<VT, IT, XT, PT, AT, YT, 4, true, BAKED>(a, padded, s);
            if (a.th <= 8) return launch_k<VT, IT, XT, PT, AT, YT, 8, true, BAKED>(a, padded, s);
            if (a.th <= 16)
                return launch_k<VT, IT, XT, PT, AT, YT, 16, true, BAKED>(a, padded, s);
            return fail(GS_ERR_UNSUPPORTED, "tileH %u > 16 not supported by the kernels", a.th);
        }
        if (a.aligned) {
            switch (a.V) {
            case 4: return launch_aligned<VT, IT, XT, PT, AT, YT, 4, false, BAKED>(a, padded, s);
            case 8: return launch_aligned<VT, IT, XT, PT, AT, YT, 8, false, BAKED>(a, padded, s);
            case 16: return launch_aligned<VT, IT, XT, PT, AT, YT, 16, false, BAKED>(a, padded, s);
            default: break;
            }
        }
        // FP64 direct layouts with run-time x: 4 or 8 positions per lane
        // (direct_lane_positions); the striped kernel takes either plan
        if (a.V != kDirectV && (BAKED || a.V != 4))
            return fail(GS_ERR_INVALID, "plan built for another shape");
        if (striped) return launch_striped<VT, IT, XT, PT, AT, YT, BAKED>(a, padded, s);
        if constexpr (!BAKED) {
            if (a.V == 4) return launch_k<VT, IT, XT, PT, AT, YT, 4, false, BAKED>(a, padded, s);
        }
        return launch_k<VT, IT, XT, PT, AT, YT, 8, false, BAKED>(a, padded, s);
    }
}

// ------------------------------------------------------------------ plan construction
__global__ void k_set_starts(uint32_t n, const uint32_t *rpos, uint32_t *sbits)
{
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n && rpos[r + 1] > rpos[r]) atomicOr(sbits + (rpos[r] >> 5), 1u << (rpos[r] & 31));
}

__global__ void k_set_real(uint32_t n, const uint32_t *rpos, const uint32_t *rlen,
                           uint32_t *rbits)
{
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    uint32_t p = rpos[r];
    const uint32_t e = p + rlen[r];
    while (p < e) {
        const uint32_t w = p >> 5, b = p & 31;
        const uint32_t cnt = min(32u - b, e - p);
        const uint32_t m = (cnt == 32 ? 0xffffffffu : ((1u << cnt) - 1u)) << b;
        atomicOr(rbits + w, m);
        p += cnt;
    }
}

// Column locality of a CSR matrix, sampled: rows r = t * stride (t < samples), the first
// 33 elements of each; cnt[0] += in-row steps, cnt[1] += steps |col[e] - col[e-1]| < 16 (the
// next column within one 128-byte line of FP64 x).
__global__ void k_col_steps(const uint32_t *row, const uint32_t *col, uint32_t stride,
                            uint32_t samples, unsigned long long *cnt)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t steps = 0, near = 0;
    if (t < samples) {
        const uint32_t r = t * stride;
        const uint32_t b = row[r], e = min(row[r + 1], b + 33u);
        for (uint32_t i = b + 1; i < e; i++) {
            const uint32_t c0 = col[i - 1], c1 = col[i];
            steps++;
            near += (c1 > c0 ? c1 - c0 : c0 - c1) < 16u ? 1u : 0u;
        }
    }
    steps = __reduce_add_sync(0xffffffffu, steps);
    near = __reduce_add_sync(0xffffffffu, near);
    if ((threadIdx.x & 31) == 0 && steps) {
        atomicAdd(cnt, (unsigned long long)steps);
        atomicAdd(cnt + 1, (unsigned long long)near);
    }
}

__global__ void k_narrow_u32(uint32_t n1, const uint64_t *a, uint32_t *b)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n1) b[i] = (uint32_t)a[i];
}

__global__ void k_split_rows(uint32_t n, const uint32_t *rpos, const uint64_t *pre,
                             uint32_t *ne, uint32_t *empty)
{
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t k = (uint32_t)pre[r];
    if (rpos[r + 1] > rpos[r]) ne[k] = r;
    else empty[r - k] = r;
}

// per window: min column over real positions -> base; flag if the spread exceeds 16 bits;
// then col16 = col32 - base (padding slots keep 0)
// nreal: slots at or past it hold no element (the tail of a compact layout's last tile)
__global__ void k_u16_cols(uint32_t nwin, uint32_t WS, uint32_t nslots, uint32_t nreal,
                           const uint32_t *col32, const uint32_t *rbits, uint32_t *colbase,
                           uint16_t *col16, uint32_t *flag)
{
    const int lane = threadIdx.x & 31;
    for (uint32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < nwin;
         w += gridDim.x * (blockDim.x >> 5)) {
        const uint32_t b = w * WS, e = min(b + WS, nslots);
        uint32_t mn = 0xffffffffu, mx = 0;
        for (uint32_t s = b + lane; s < e; s += 32) {
            const bool real = s < nreal && (!rbits || ((rbits[s >> 5] >> (s & 31)) & 1u));
            if (real) { mn = min(mn, col32[s]); mx = max(mx, col32[s]); }
        }
        for (int o = 16; o > 0; o >>= 1) {
            mn = min(mn, __shfl_xor_sync(kFull, mn, o));
            mx = max(mx, __shfl_xor_sync(kFull, mx, o));
        }
        const uint32_t base = (mn == 0xffffffffu) ? 0u : mn;
        if (lane == 0) {
            colbase[w] = base;
            if (mn != 0xffffffffu && mx - mn > 65535u) atomicOr(flag, 1u);
        }
        for (uint32_t s = b + lane; s < e; s += 32) {
            const bool real = s < nreal && (!rbits || ((rbits[s >> 5] >> (s & 31)) & 1u));
            col16[s] = real ? (uint16_t)(col32[s] - base) : (uint16_t)0;
        }
    }
}

// ---------------------------------------------------------------------------------------
// Layouts made of whole tiles per row: UNC tileH = 1 (tiles of THW slots) and AXC (bricks of
// the same shape); baked (the reference's ax: tiles of [THW values | THW x]) or with value /
// column streams and x gathered at run time (real slots only: the slot-level bitmap a.rbits,
// when the layout pads).  The plan is built over tiles (a.npos = tiles, a.sbits = first tile
// of each non-empty row), so one lane of a 32-tile chunk stands for one tile and the striped
// segmented scan (stripe_chunk) adds tile sums into rows.  The tiles' data are loaded
// cooperatively: in each of THW/2 load steps, groups of G = THW/2 lanes read 16 bytes of one
// tile's values and the matching 16 bytes of its x half (baked) or 8 bytes of its columns
// (coalesced across the warp), form two products, and sum them over the group (shuffle tree);
// a shuffle transpose then hands tile k's sum to lane k.  Per tile: products in pairs, pairs
// summed over a binary tree, fixed order.
template <int THW, bool BAKED, bool EMPTY>
__global__ void __launch_bounds__(256) k_tiles(const RowsArgs a)
{
    constexpr int G = THW / 2;      // lanes per tile in a load step
    constexpr int TPI = 32 / G;     // tiles per load step
    constexpr int NI = G;           // load steps per 32-tile chunk
    const int lane = threadIdx.x & 31;
    double *y = static_cast<double *>(a.y);
    const double *val = static_cast<const double *>(a.val);
    const uint32_t *col = static_cast<const uint32_t *>(a.col);
    const double *x = static_cast<const double *>(a.x);
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t cpwin = a.V;  // chunks per plan window
    const unsigned lt = (1u << lane) - 1u;
    if constexpr (EMPTY) {
        for (uint32_t i = gw * 32 + lane; i < a.n_empty; i += nwarps * 32)
            y[__ldg(a.empty + i)] = 0.0;
    }
    const uint32_t ntiles = a.npos;
    const uint32_t nchunk = (ntiles + 31) / 32;
    const int gl = lane % G, gt = lane / G;
    // the sum of tile ch*32 + lane, in this lane (0 past the last tile)
    auto chunk_sums = [&](uint32_t ch) -> double {
        double part[NI];
#pragma unroll
        for (int i = 0; i < NI; i++) {
            const uint32_t t = ch * 32u + (uint32_t)(i * TPI + gt);
            part[i] = 0.0;
            if (t < ntiles) {
                if constexpr (BAKED) {
                    const double *tp = val + (size_t)t * (2 * THW) + 2 * gl;
                    const double2 v = __ldcs(reinterpret_cast<const double2 *>(tp));
                    const double2 xv = __ldcs(reinterpret_cast<const double2 *>(tp + THW));
                    part[i] = __dadd_rn(__dmul_rn(v.x, xv.x), __dmul_rn(v.y, xv.y));
                } else {
                    const uint32_t s0 = t * THW + 2u * (uint32_t)gl;  // even: one bitmap word
                    const double2 v = __ldcs(reinterpret_cast<const double2 *>(val + s0));
                    const uint2 c = __ldcs(reinterpret_cast<const uint2 *>(col + s0));
                    const uint32_t rb =
                        a.rbits ? (__ldg(a.rbits + (s0 >> 5)) >> (s0 & 31)) & 3u : 3u;
                    const double p0 = (rb & 1u) ? __dmul_rn(v.x, __ldg(x + c.x)) : 0.0;
                    const double p1 = (rb & 2u) ? __dmul_rn(v.y, __ldg(x + c.y)) : 0.0;
                    part[i] = __dadd_rn(p0, p1);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < NI; i++) {
#pragma unroll
            for (int d = G / 2; d >= 1; d >>= 1)
                part[i] = __dadd_rn(part[i], __shfl_down_sync(kFull, part[i], d, G));
        }
        double sum = 0.0;
#pragma unroll
        for (int i = 0; i < NI; i++) {
            const double v = __shfl_sync(kFull, part[i], (lane % TPI) * G);
            if (lane / TPI == i) sum = v;
        }
        return sum;
    };
    const uint32_t nranges = (a.nwin + a.wpw - 1) / a.wpw;
    for (uint32_t rg = gw; rg < nranges; rg += nwarps) {
        const uint32_t c0 = rg * a.wpw * cpwin;
        const uint32_t c1 = min(c0 + a.wpw * cpwin, nchunk);
        uint32_t cnt = __ldg(a.wcount + rg * a.wpw);  // row starts before the range
        bool seen = (c0 == 0);
        double carry = 0.0;
        for (uint32_t ch = c0; ch < c1; ch++) {
            const uint32_t word = __ldg(a.sbits + ch);
            const uint32_t vm =
                ch * 32u + 32u <= ntiles ? 0xffffffffu : ((1u << (ntiles - ch * 32u)) - 1u);
            const double prod = chunk_sums(ch);
            stripe_chunk<double, double, double, EMPTY>(a, y, lane, lt, ch, nchunk, false, word,
                                                        vm, prod, cnt, seen, carry);
        }
        // past the range: until the range's last row ends
        if (seen) {
            for (uint32_t ch = c1; ch < nchunk; ch++) {
                const uint32_t word = __ldg(a.sbits + ch);
                const uint32_t vm =
                    ch * 32u + 32u <= ntiles ? 0xffffffffu : ((1u << (ntiles - ch * 32u)) - 1u);
                const double prod = chunk_sums(ch);
                if (!stripe_chunk<double, double, double, EMPTY>(a, y, lane, lt, ch, nchunk, true,
                                                                 word, vm, prod, cnt, seen, carry))
                    break;
            }
        }
    }
}

template <int THW, bool BAKED>
gs_status launch_tiles_t(const RowsArgs &a, cudaStream_t s)
{
    const uint32_t nranges = (a.nwin + a.wpw - 1) / a.wpw;
    uint32_t warps = nranges;
    if (a.n_empty) warps = max(warps, min((a.n_empty + 31) / 32, 148u * 64u));
    if (warps == 0) return GS_OK;
    const uint32_t blocks = min((warps + 7) / 8, 148u * 256u);
    if (a.n_empty) k_tiles<THW, BAKED, true><<<blocks, 256, 0, s>>>(a);
    else k_tiles<THW, BAKED, false><<<blocks, 256, 0, s>>>(a);
    GS_CHECK_LAUNCH();
    return GS_OK;
}

}  // namespace

gs_status random_columns(const uint32_t *d_row, const uint32_t *d_col, uint32_t n,
                         bool *random, cudaStream_t s)
{
    *random = false;
    if (n == 0) return GS_OK;
    const uint32_t samples = n < 65536u ? n : 65536u;
    const uint32_t stride = n / samples;
    DevBuf cnt;
    GS_TRY(cnt.alloc_zero(16, s));
    k_col_steps<<<(samples + 255) / 256, 256, 0, s>>>(d_row, d_col, stride, samples,
                                                      cnt.as<unsigned long long>());
    GS_CHECK_LAUNCH();
    unsigned long long h[2] = {0, 0};
    GS_CUDA(cudaMemcpyAsync(h, cnt.p, 16, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    *random = h[1] * 4 < h[0];
    return GS_OK;
}

gs_status direct_lane_positions(const uint32_t *d_row, const uint32_t *d_col, uint32_t n,
                                uint64_t nnz, uint32_t *V, cudaStream_t s)
{
    *V = kDirectV;
    if (n == 0 || nnz == 0) return GS_OK;
    if ((double)nnz / (double)n < 8.0) {  // short rows: more warps beat longer lanes
        *V = 4;
        return GS_OK;
    }
    // random x gathers set the pace: 4 positions per lane
    bool rnd = false;
    GS_TRY(random_columns(d_row, d_col, n, &rnd, s));
    if (rnd) *V = 4;
    return GS_OK;
}

gs_status build_rows_plan(const uint32_t *d_rpos, const uint32_t *d_rlen, uint32_t n,
                          uint32_t V, RowsPlan &P, cudaStream_t s, bool tiled)
{
    P.V = V;
    P.padded = d_rlen != nullptr;
    uint32_t npos = 0;
    GS_CUDA(cudaMemcpyAsync(&npos, d_rpos + n, 4, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    P.npos = npos;
    const uint64_t WS = 32ull * V;
    P.nwin = (uint32_t)(((uint64_t)npos + WS - 1) / WS);
    // windows per warp range of the LDG kernels: ~2048 positions at 8 per lane (27-point
    // stencil against ~1024: CSR 330 -> 318 us, COM th=8 547 -> 471, UNC th=8 448 -> 408;
    // power-law: COM th=8 437 -> 409, UNC th=8 364 -> 343) and for tiled layouts of tileH
    // 2-4 (27-point stencil: COM th=4 452 -> 420 us, UNC th=4 288 -> 276; drop-in gaxtch
    // th=4 on the power-law 295 -> 281), ~1024 otherwise (CSR at 4 per lane on the
    // power-law: 329 against 334 us); fewer when the matrix is too small to give every SM
    // enough warps
    const uint32_t range = (V == 8 || (tiled && V <= 4)) ? 2048u : 1024u;
    uint32_t wpw = (uint32_t)((range + WS - 1) / WS);
    while (wpw > 1 && (uint64_t)P.nwin / wpw < 148ull * 48ull) wpw >>= 1;
    P.wpw = wpw;
    const size_t words = (size_t)P.nwin * V + 2;
    GS_TRY(P.sbits.alloc_zero(words * 4, s));
    const unsigned g = (n + 255) / 256;
    k_set_starts<<<g, 256, 0, s>>>(n, d_rpos, P.sbits.as<uint32_t>());
    GS_CHECK_LAUNCH();
    if (P.padded) {
        GS_TRY(P.rbits.alloc_zero(words * 4, s));
        k_set_real<<<g, 256, 0, s>>>(n, d_rpos, d_rlen, P.rbits.as<uint32_t>());
        GS_CHECK_LAUNCH();
    }
    DevBuf pre;
    GS_TRY(pre.alloc(((size_t)P.nwin + 1) * 8));
    CountSpec cw{CountKind::WindowPopc};
    cw.arr = P.sbits.as<uint32_t>();
    cw.a = V;
    GS_TRY(exclusive_scan(cw, P.nwin, pre.as<uint64_t>(), nullptr, s));
    GS_TRY(P.wcount.alloc(((size_t)P.nwin + 1) * 4));
    k_narrow_u32<<<(P.nwin + 256) / 256, 256, 0, s>>>(P.nwin + 1, pre.as<uint64_t>(),
                                                       P.wcount.as<uint32_t>());
    GS_CHECK_LAUNCH();
    // empty rows: rank -> row map and the list of rows to zero
    DevBuf pe;
    GS_TRY(pe.alloc(((size_t)n + 1) * 8));
    CountSpec ce{CountKind::NonEmpty};
    ce.row = d_rpos;
    uint64_t nonempty = 0;
    GS_TRY(exclusive_scan(ce, n, pe.as<uint64_t>(), &nonempty, s));
    P.n_empty = (uint32_t)(n - nonempty);
    if (P.n_empty) {
        GS_TRY(P.ne.alloc((size_t)nonempty * 4 + 4));
        GS_TRY(P.empty.alloc((size_t)P.n_empty * 4));
        k_split_rows<<<g, 256, 0, s>>>(n, d_rpos, pe.as<uint64_t>(), P.ne.as<uint32_t>(),
                                       P.empty.as<uint32_t>());
        GS_CHECK_LAUNCH();
    }
    GS_TRY(P.status.alloc_zero(4, s));
    GS_CUDA(cudaStreamSynchronize(s));
    return GS_OK;
}

gs_status build_u16_columns(const uint32_t *d_col32, uint32_t nslots, RowsPlan &P,
                            uint16_t *d_col16, cudaStream_t s)
{
    GS_TRY(P.colbase.alloc((size_t)P.nwin * 4 + 4));
    DevBuf flag;
    GS_TRY(flag.alloc_zero(4, s));
    const uint32_t blocks = min((P.nwin + 7) / 8, 148u * 64u);
    if (blocks)
        k_u16_cols<<<blocks, 256, 0, s>>>(P.nwin, 32u * P.V, nslots,
                                          P.padded ? nslots : min(P.npos, nslots), d_col32,
                                          P.padded ? P.rbits.as<uint32_t>() : nullptr,
                                          P.colbase.as<uint32_t>(), d_col16, flag.as<uint32_t>());
    GS_CHECK_LAUNCH();
    uint32_t hf = 0;
    GS_CUDA(cudaMemcpyAsync(&hf, flag.p, 4, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    if (hf)
        return fail(GS_ERR_UNSUPPORTED,
                    "a window of %u positions spans more than 65536 columns: 16-bit column "
                    "offsets do not fit this matrix", 32u * P.V);
    return GS_OK;
}

uint32_t aligned_lane_positions(uint32_t align, bool *aligned)
{
    *aligned = false;
    if (align == 0) return kDirectV;
    for (uint32_t v : {16u, 8u, 4u, 2u}) {
        if (v > align || align % v) continue;
        if (v == 16 && align != 16) continue;  // 16 only for 16-high tiles
        *aligned = true;
        return v;
    }
    return kDirectV;
}

RowsArgs rows_args(const RowsPlan &P)
{
    RowsArgs a{};
    a.aligned = P.aligned ? 1u : 0u;
    a.grouped = P.grouped ? 1u : 0u;
    a.npos = P.npos;
    a.nwin = P.nwin;
    a.wpw = P.wpw;
    a.V = P.V;
    a.n_empty = P.n_empty;
    a.sbits = P.sbits.as<uint32_t>();
    a.rbits = P.rbits.as<uint32_t>();
    a.wcount = P.wcount.as<uint32_t>();
    a.ne = P.ne.as<uint32_t>();
    a.empty = P.empty.as<uint32_t>();
    a.colbase = P.colbase.as<uint32_t>();
    a.status = P.status.as<uint32_t>();
    a.thw = 1;
    a.th = 1;
    return a;
}

gs_status launch_rows(const RowsArgs &a0, gs_dtype vtype, gs_itype itype, gs_dtype ytype,
                      uint32_t flags, bool tiled, bool baked, bool padded, cudaStream_t s)
{
    RowsArgs a = a0;
    a.wide = ((reinterpret_cast<uintptr_t>(a.val) | reinterpret_cast<uintptr_t>(a.col)) & 31u)
                 ? 0u
                 : 1u;
    if (tiled && (a.thw == 0 || 32 % a.thw != 0))
        return fail(GS_ERR_UNSUPPORTED, "tileH>1 kernels need tileHW dividing 32 (got %u)",
                    a.thw);
    if (tiled && a.V != a.th) return fail(GS_ERR_INVALID, "tiled plan built for another tileH");
    if (baked) {
        if (vtype != GS_F64 || ytype != GS_F64)
            return fail(GS_ERR_UNSUPPORTED, "baked layouts are FP64 only");
        return launch_shape<double, uint32_t, double, double, double, double, true>(
            a, tiled, padded, flags, s);
    }
    const bool acc64 = (flags & GS_FLAG_ACC_F64) != 0;
    if (vtype == GS_F64) {
        if (ytype != GS_F64 || itype != GS_IDX_U32)
            return fail(GS_ERR_UNSUPPORTED, "FP64 matrices take FP64 y and 32-bit columns");
        return launch_shape<double, uint32_t, double, double, double, double, false>(
            a, tiled, padded, flags, s);
    }
#define GS_MIXED(VT_, IT_)                                                                   \
    do {                                                                                     \
        if (acc64 && ytype == GS_F64)                                                        \
            return launch_shape<VT_, IT_, float, float, double, double, false>(a, tiled,     \
                                                                               padded, flags, s); \
        if (acc64)                                                                           \
            return launch_shape<VT_, IT_, float, float, double, float, false>(a, tiled,      \
                                                                              padded, flags, s); \
        if (ytype == GS_F64)                                                                 \
            return launch_shape<VT_, IT_, float, float, float, double, false>(a, tiled,      \
                                                                              padded, flags, s); \
        return launch_shape<VT_, IT_, float, float, float, float, false>(a, tiled, padded,   \
                                                                         flags, s);          \
    } while (0)
    if (vtype == GS_F32 && itype == GS_IDX_U32) GS_MIXED(float, uint32_t);
    if (vtype == GS_F32 && itype == GS_IDX_U16) GS_MIXED(float, uint16_t);
    if (vtype == GS_BF16 && itype == GS_IDX_U32) GS_MIXED(__nv_bfloat16, uint32_t);
    if (vtype == GS_BF16 && itype == GS_IDX_U16) GS_MIXED(__nv_bfloat16, uint16_t);
#undef GS_MIXED
    return fail(GS_ERR_UNSUPPORTED, "value type %d / index type %d not supported", (int)vtype,
                (int)itype);
}

gs_status launch_tiles(const RowsArgs &a, uint32_t thw, bool baked, cudaStream_t s)
{
    switch (thw) {
    case 4: return baked ? launch_tiles_t<4, true>(a, s) : launch_tiles_t<4, false>(a, s);
    case 8: return baked ? launch_tiles_t<8, true>(a, s) : launch_tiles_t<8, false>(a, s);
    case 16: return baked ? launch_tiles_t<16, true>(a, s) : launch_tiles_t<16, false>(a, s);
    case 32: return baked ? launch_tiles_t<32, true>(a, s) : launch_tiles_t<32, false>(a, s);
    default: return fail(GS_ERR_UNSUPPORTED, "tile width %u (4, 8, 16 or 32)", thw);
    }
}

}  // namespace gs
