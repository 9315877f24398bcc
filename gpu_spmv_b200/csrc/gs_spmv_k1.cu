// gs_spmv_k1.cu -- K1 SpMV (sorted, 32-row chunked ELL) and its work plan.
//
// Reference: gk1 (cudaSpmv.cu:851-867) gives one thread per sorted row; lane l of chunk c
// reads slot chp[c] + 32*j + l for j < nmc[c] (so a warp's loads are coalesced) and
// scatters y[permi[32c + l]].  Because the chunks are sorted by decreasing length, the
// first chunks of a power-law matrix are thousands of steps long and a single warp would
// walk them serially.  Here a chunk longer than kK1Split steps is cut into pieces that
// separate warps process; each piece writes its 32 partial sums to a scratch array and
// the last piece to finish (an arrival counter per chunk) adds the pieces in piece order
// and writes y -- deterministic, no atomics on y, no waiting.  Unsplit chunks sum each row
// sequentially in column order, exactly like the reference's CPU loop.
//
// Rows shorter than their chunk's nmc are padded with zeros in the layout
// (cudaSpmv.cu:818-819 calloc); the engine stops at the row's own length when it is known
// (native matrices keep the sorted lengths) and, like gk1, reads the padding otherwise.
// A chunk whose rows are all empty reads nothing (gk1 reads one slot past it,
// cudaSpmv.cu:861).
//
// Reduced-precision storage (an extension; the reference is FP64 only): values in FP32 or
// BF16 with FP32 x, products in FP32 and sums in FP32 or FP64; columns either 32-bit or as
// 16-bit steps from the row's previous column, re-anchored at the first slot of every
// work unit by a 32-bit checkpoint (ck[unit * 32 + lane]), so each unit decodes its
// columns with a running sum and no unit depends on another.
#include "gs_internal.cuh"

namespace gs {

namespace {

template <class T> __device__ __forceinline__ float k1_val_f32(T v);
template <> __device__ __forceinline__ float k1_val_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ float k1_val_f32<__nv_bfloat16>(__nv_bfloat16 v)
{
    return __bfloat162float(v);
}

// products: FP64 matrices multiply and add in FP64 (non-fused, like the CPU loop); reduced
// matrices multiply in FP32 and add in AT
template <class VT, class XT, class AT>
__device__ __forceinline__ AT k1_fma(AT acc, VT v, XT x)
{
    if constexpr (std::is_same<VT, double>::value) {
        return __dadd_rn(acc, __dmul_rn(v, x));
    } else {
        const float p = __fmul_rn(k1_val_f32(v), x);
        if constexpr (std::is_same<AT, double>::value) return __dadd_rn(acc, (double)p);
        else return __fadd_rn(acc, p);
    }
}

// 8 consecutive values of a lane-blocked group as floats (16- or 32-byte streaming loads)
__device__ __forceinline__ void ld8_vals(const float *p, float (&v)[8])
{
    const float4 a = __ldcs(reinterpret_cast<const float4 *>(p));
    const float4 b = __ldcs(reinterpret_cast<const float4 *>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void ld8_vals(const __nv_bfloat16 *p, float (&v)[8])
{
    const uint4 w = __ldcs(reinterpret_cast<const uint4 *>(p));
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&ws[i]));
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}
template <class T> __device__ __forceinline__ void ld8_vals(const T *, float (&)[8]) {}
// 8 consecutive 16-bit column steps (one 16-byte streaming load)
__device__ __forceinline__ void ld8_steps(const uint16_t *p, uint32_t (&c)[8])
{
    const uint4 w = __ldcs(reinterpret_cast<const uint4 *>(p));
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        c[2 * i] = ws[i] & 0xffffu;
        c[2 * i + 1] = ws[i] >> 16;
    }
}

// Blocks of 256 per SM: 8 (32 registers) for FP64 and for 16-bit steps, whose units carry
// few bytes each, so that more of them are in flight (16-bit steps on the 27-point stencil:
// 150 -> 136 us over 6 blocks); 6 (40 registers) for FP32 / BF16 values with 32-bit columns.
template <class VT, class IT, class AT, class YT>
__global__ void __launch_bounds__(256, std::is_same<VT, double>::value
                                           ? 8
                                           : (std::is_same<IT, uint16_t>::value ? 8 : 6))
    k_k1(const K1Args a)
{
    using XT = typename std::conditional<std::is_same<VT, double>::value, double, float>::type;
    constexpr bool kDelta = std::is_same<IT, uint16_t>::value;
    const VT *__restrict__ val = static_cast<const VT *>(a.val);
    const IT *__restrict__ col = static_cast<const IT *>(a.col);
    const XT *__restrict__ x = static_cast<const XT *>(a.x);
    YT *__restrict__ y = static_cast<YT *>(a.y);
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    // no chunk cut into pieces: unit u is chunk u (one dependent load less per unit)
    const bool whole = a.units == a.chunkNum;
    for (uint32_t u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < a.units;
         u += warps) {
        const uint32_t c = whole ? u : __ldg(a.unit_chunk + u);
        const uint32_t ub = whole ? u : __ldg(a.unit_base + c);
        const uint32_t np = whole ? 1u : __ldg(a.unit_base + c + 1) - ub;
        const uint32_t piece = u - ub;
        const uint32_t nmc = __ldg(a.nmc + c);
        const uint32_t g = 32u * c + (uint32_t)lane;
        const bool valid = g < a.nrows;
        const uint32_t len = valid ? (a.klen ? __ldg(a.klen + g) : nmc) : 0u;
        const uint32_t j0 = piece * kK1Split;
        const uint32_t j1 = min(len, j0 + kK1Split);
        const uint32_t base = __ldg(a.chp + c) + (uint32_t)lane;
        uint32_t run = 0;  // decoded column of the previous slot (16-bit steps)
        if constexpr (kDelta) run = j0 < j1 ? __ldg(a.ck + (size_t)u * 32 + lane) : 0u;
        AT acc = AT(0);
        uint32_t j = j0;
        if constexpr (kDelta) {
            // lane-blocked groups of 8 steps: one 16-byte load of 8 column steps and one
            // or two of 8 values (k1_slot); steps past this lane's row are padding
            const uint32_t jg = min(j1, nmc & ~7u), cb = __ldg(a.chp + c);
            for (; j < jg; j += 8) {
                const uint32_t gp = cb + (j >> 3) * 256u + (uint32_t)lane * 8u;
                float v[8];
                uint32_t cc[8];
                ld8_vals(val + gp, v);
                ld8_steps(reinterpret_cast<const uint16_t *>(col) + gp, cc);
                XT xv[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    run += cc[k];
                    xv[k] = j + k < j1 ? __ldg(x + run) : XT(0);
                }
#pragma unroll
                for (int k = 0; k < 8; k++)
                    if (j + k < j1) acc = k1_fma<float, XT, AT>(acc, v[k], xv[k]);
            }
        }
        // 8 slots in flight per lane: loads first, then gathers, then the ordered sum
        // (16-bit steps: fewer than 8 steps remain after the groups)
        for (; !kDelta && j + 8 <= j1; j += 8) {
            VT v[8];
            XT xv[8];
            uint32_t cc[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t pos = base + 32u * (j + k);
                v[k] = __ldcs(val + pos);
                cc[k] = (uint32_t)__ldcs(col + pos);
            }
            if constexpr (kDelta) {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    run += cc[k];
                    cc[k] = run;
                }
            }
#pragma unroll
            for (int k = 0; k < 8; k++) xv[k] = __ldg(x + cc[k]);
#pragma unroll
            for (int k = 0; k < 8; k++) acc = k1_fma<VT, XT, AT>(acc, v[k], xv[k]);
        }
        // the last 1-7 slots of this lane.  FP32 / BF16 values with 32-bit columns: loads
        // first, as one batch (5 % faster on the 27-point stencil); FP64 the same when the
        // whole chunk is shorter than 8 steps (its rows are all tail), else the plain loop,
        // as for 16-bit steps, which measured faster for them (27-point stencil FP32 values
        // with 16-bit steps: 132.0 us plain, 133.7 / 135.7 batched 4 / 8 at a time)
        constexpr bool kF64 = std::is_same<VT, double>::value;
        const bool batch_tail = !kDelta && (!kF64 || nmc < 8u);
        for (; !batch_tail && j < j1; j++) {
            const uint32_t pos = base + 32u * j;
            uint32_t cj = (uint32_t)__ldcs(col + pos);
            if constexpr (kDelta) {
                run += cj;
                cj = run;
            }
            acc = k1_fma<VT, XT, AT>(acc, __ldcs(val + pos), __ldg(x + cj));
        }
        constexpr int kTail = kF64 ? 4 : 7;  // FP64: 4 slots in its 32 registers
        for (; batch_tail && j < j1; j += kTail) {
            const uint32_t rem = j1 - j;
            VT v[kTail];
            XT xv[kTail];
            uint32_t cc[kTail];
#pragma unroll
            for (int k = 0; k < kTail; k++) {
                const uint32_t pos = base + 32u * (j + k);
                v[k] = (uint32_t)k < rem ? __ldcs(val + pos) : VT(0);
                cc[k] = (uint32_t)k < rem ? (uint32_t)__ldcs(col + pos) : 0u;
            }
#pragma unroll
            for (int k = 0; k < kTail; k++) xv[k] = (uint32_t)k < rem ? __ldg(x + cc[k]) : XT(0);
#pragma unroll
            for (int k = 0; k < kTail; k++)
                if ((uint32_t)k < rem) acc = k1_fma<VT, XT, AT>(acc, v[k], xv[k]);
        }
        if (np == 1) {
            if (valid) y[__ldg(a.permi + g)] = (YT)acc;
            continue;
        }
        a.partial[(size_t)u * 32 + lane] = (double)acc;
        __threadfence();
        __syncwarp();
        uint32_t ticket = 0;
        if (lane == 0) ticket = atomicAdd(a.count + c, 1u);
        ticket = __shfl_sync(0xffffffffu, ticket, 0);
        if (ticket == np - 1) {
            __threadfence();
            AT s = AT(0);
            for (uint32_t k = 0; k < np; k++) {
                const AT pk = (AT)__ldcg(a.partial + (size_t)(ub + k) * 32 + lane);
                if constexpr (std::is_same<AT, double>::value) s = __dadd_rn(s, pk);
                else s = __fadd_rn(s, pk);
            }
            if (valid) y[__ldg(a.permi + g)] = (YT)s;
            if (lane == 0) a.count[c] = 0;  // ready for the next launch
        }
    }
}

// 16-bit column steps: for unit u and lane l, ck = column of the unit's first slot,
// col16 = column - previous column inside the unit (0 at the first slot); flag bit 0 when
// a step is negative or above 65535.
__global__ void __launch_bounds__(256) k_k1_deltas(const K1Args a, const uint32_t *col32,
                                                   uint16_t *col16, uint32_t *ck,
                                                   uint32_t *flag)
{
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < a.units;
         u += warps) {
        const uint32_t c = a.unit_chunk[u];
        const uint32_t piece = u - a.unit_base[c];
        const uint32_t g = 32u * c + (uint32_t)lane;
        const uint32_t len = g < a.nrows ? a.klen[g] : 0u;
        const uint32_t j0 = piece * kK1Split;
        const uint32_t j1 = min(len, j0 + kK1Split);
        const uint32_t cb = a.chp[c], m = a.nmc[c];
        uint32_t prev = j0 < j1 ? col32[k1_slot(cb, m, j0, lane, true)] : 0u;
        ck[(size_t)u * 32 + lane] = prev;
        bool bad = false;
        for (uint32_t j = j0; j < j1; j++) {
            const uint32_t pos = k1_slot(cb, m, j, lane, true);
            const uint32_t cj = col32[pos];
            const uint32_t d = cj - prev;  // wraps when the row's columns decrease
            bad |= d > 0xffffu;
            col16[pos] = (uint16_t)d;
            prev = cj;
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flag, 1u);
    }
}

__global__ void k_k1_units(const uint64_t *ubase64, const uint32_t *nmc, uint32_t chunkNum,
                           uint32_t *unit_chunk, uint32_t *unit_base)
{
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= chunkNum) unit_base[c] = (uint32_t)ubase64[c];
    if (c < chunkNum) {
        uint32_t b = (uint32_t)ubase64[c], e = (uint32_t)ubase64[c + 1];
        for (uint32_t u = b; u < e; u++) unit_chunk[u] = c;
    }
}

}  // namespace

gs_status build_k1_plan(const uint32_t *d_nmc, uint32_t chunkNum, DevBuf &unit_chunk,
                        DevBuf &unit_base, DevBuf &partial, DevBuf &count, uint32_t *units,
                        cudaStream_t s)
{
    DevBuf pre;
    GS_TRY(pre.alloc(((size_t)chunkNum + 1) * 8));
    CountSpec spec{CountKind::PiecesMin1};
    spec.arr = d_nmc;
    spec.a = kK1Split;
    uint64_t total = 0;
    GS_TRY(exclusive_scan(spec, chunkNum, pre.as<uint64_t>(), &total, s));
    if (total >= 0xffffffffull) return fail(GS_ERR_OVERFLOW, "K1 plan too large");
    *units = (uint32_t)total;
    GS_TRY(unit_chunk.alloc((size_t)total * 4));
    GS_TRY(unit_base.alloc(((size_t)chunkNum + 1) * 4));
    GS_TRY(partial.alloc((size_t)total * 32 * 8));
    GS_TRY(count.alloc_zero((size_t)chunkNum * 4, s));
    k_k1_units<<<(chunkNum + 256) / 256, 256, 0, s>>>(pre.as<uint64_t>(), d_nmc, chunkNum,
                                                     unit_chunk.as<uint32_t>(),
                                                     unit_base.as<uint32_t>());
    GS_CHECK_LAUNCH();
    GS_CUDA(cudaStreamSynchronize(s));
    return GS_OK;
}

namespace {
uint32_t k1_blocks(uint32_t units) { return min((units + 7) / 8, 148u * 64u); }

template <class VT, class IT, class AT, class YT>
gs_status launch_k1_t(const K1Args &a, cudaStream_t s)
{
    k_k1<VT, IT, AT, YT><<<k1_blocks(a.units), 256, 0, s>>>(a);
    GS_CHECK_LAUNCH();
    return GS_OK;
}

template <class VT, class IT>
gs_status launch_k1_acc(const K1Args &a, bool acc64, gs_dtype ytype, cudaStream_t s)
{
    if (acc64) {
        if (ytype == GS_F64) return launch_k1_t<VT, IT, double, double>(a, s);
        return launch_k1_t<VT, IT, double, float>(a, s);
    }
    if (ytype == GS_F64) return launch_k1_t<VT, IT, float, double>(a, s);
    return launch_k1_t<VT, IT, float, float>(a, s);
}
}  // namespace

gs_status launch_k1(const K1Args &a, gs_dtype vtype, gs_itype itype, gs_dtype ytype, bool acc64,
                    cudaStream_t s)
{
    if (a.units == 0) return GS_OK;
    if (itype == GS_IDX_U16 && !a.ck) return fail(GS_ERR_INVALID, "16-bit K1 without checkpoints");
    if (vtype == GS_F64) {
        if (itype != GS_IDX_U32 || ytype != GS_F64)
            return fail(GS_ERR_UNSUPPORTED, "FP64 K1 takes 32-bit columns and FP64 y");
        return launch_k1_t<double, uint32_t, double, double>(a, s);
    }
    if (vtype == GS_F32) {
        if (itype == GS_IDX_U16) return launch_k1_acc<float, uint16_t>(a, acc64, ytype, s);
        return launch_k1_acc<float, uint32_t>(a, acc64, ytype, s);
    }
    if (vtype == GS_BF16) {
        if (itype == GS_IDX_U16) return launch_k1_acc<__nv_bfloat16, uint16_t>(a, acc64, ytype, s);
        return launch_k1_acc<__nv_bfloat16, uint32_t>(a, acc64, ytype, s);
    }
    return fail(GS_ERR_UNSUPPORTED, "value type %d", (int)vtype);
}

gs_status build_k1_deltas(const K1Args &a, const uint32_t *d_col32, uint16_t *d_col16,
                          uint32_t *d_ck, cudaStream_t s)
{
    if (a.units == 0) return GS_OK;
    DevBuf flag;
    GS_TRY(flag.alloc_zero(4, s));
    k_k1_deltas<<<k1_blocks(a.units), 256, 0, s>>>(a, d_col32, d_col16, d_ck,
                                                     flag.as<uint32_t>());
    GS_CHECK_LAUNCH();
    uint32_t hf = 0;
    GS_CUDA(cudaMemcpyAsync(&hf, flag.p, 4, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    if (hf)
        return fail(GS_ERR_UNSUPPORTED,
                    "a row's consecutive columns are more than 65535 apart (or decrease): "
                    "16-bit K1 column steps do not fit this matrix");
    return GS_OK;
}

}  // namespace gs
