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
#include "gs_internal.cuh"

namespace gs {

namespace {

__global__ void __launch_bounds__(256) k_k1(const K1Args a)
{
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < a.units;
         u += warps) {
        const uint32_t c = __ldg(a.unit_chunk + u);
        const uint32_t ub = __ldg(a.unit_base + c);
        const uint32_t np = __ldg(a.unit_base + c + 1) - ub;
        const uint32_t piece = u - ub;
        const uint32_t nmc = __ldg(a.nmc + c);
        const uint32_t g = 32u * c + (uint32_t)lane;
        const bool valid = g < a.nrows;
        const uint32_t len = valid ? (a.klen ? __ldg(a.klen + g) : nmc) : 0u;
        const uint32_t j0 = piece * kK1Split;
        const uint32_t j1 = min(len, j0 + kK1Split);
        const uint32_t base = __ldg(a.chp + c) + (uint32_t)lane;
        double acc = 0.0;
        uint32_t j = j0;
        // 8 slots in flight per lane: loads first, then gathers, then the ordered sum
        for (; j + 8 <= j1; j += 8) {
            double v[8], xv[8];
            uint32_t c[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const uint32_t pos = base + 32u * (j + u);
                v[u] = __ldcs(a.val + pos);
                c[u] = __ldcs(a.col + pos);
            }
#pragma unroll
            for (int u = 0; u < 8; u++) xv[u] = __ldg(a.x + c[u]);
#pragma unroll
            for (int u = 0; u < 8; u++) acc = __dadd_rn(acc, __dmul_rn(v[u], xv[u]));
        }
        for (; j < j1; j++) {
            const uint32_t pos = base + 32u * j;
            const double v = __ldcs(a.val + pos);
            const double xv = __ldg(a.x + __ldcs(a.col + pos));
            acc = __dadd_rn(acc, __dmul_rn(v, xv));
        }
        if (np == 1) {
            if (valid) a.y[__ldg(a.permi + g)] = acc;
            continue;
        }
        a.partial[(size_t)u * 32 + lane] = acc;
        __threadfence();
        __syncwarp();
        uint32_t ticket = 0;
        if (lane == 0) ticket = atomicAdd(a.count + c, 1u);
        ticket = __shfl_sync(0xffffffffu, ticket, 0);
        if (ticket == np - 1) {
            __threadfence();
            double s = 0.0;
            for (uint32_t k = 0; k < np; k++)
                s = __dadd_rn(s, __ldcg(a.partial + (size_t)(ub + k) * 32 + lane));
            if (valid) a.y[__ldg(a.permi + g)] = s;
            if (lane == 0) a.count[c] = 0;  // ready for the next launch
        }
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

gs_status launch_k1(const K1Args &a, cudaStream_t s)
{
    if (a.units == 0) return GS_OK;
    uint32_t blocks = (a.units + 7) / 8;
    blocks = min(blocks, 148u * 64u);
    k_k1<<<blocks, 256, 0, s>>>(a);
    GS_CHECK_LAUNCH();
    return GS_OK;
}

}  // namespace gs
