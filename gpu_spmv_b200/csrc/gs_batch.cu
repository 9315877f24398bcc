// gs_batch.cu -- many K1 matrices of uneven size, each with its own right-hand sides, in one
// persistent launch.
//
// Work list: one item per (matrix, K1 unit, right-hand-side block), ordered by decreasing
// work (steps of the unit's piece times block width, longest first), so the persistent
// warps, which take items four at a time from an atomic counter, finish together.  Each
// matrix keeps its own right-hand-side block width kb (a divisor of its padded count kpad;
// chosen by the autotuner), and its descriptor (layout arrays, operands, scratch) lives in
// device memory, so new operands need no new launch configuration: a CUDA graph captured
// once (counter reset + kernel) is replayed as is.
//
// No counterpart in the reference, which runs one matrix and one right-hand side per call.
#include <algorithm>
#include <numeric>
#include <vector>

#include "gs_mm.cuh"

using gs::DevBuf;
using gs::fail;

struct gs_batch {
    gs_dtype vtype = GS_F64;
    std::vector<gs_matrix *> mats;
    std::vector<uint32_t> k, kpad, kb;
    std::vector<gs::mm::MMArgs> desc;  // host copy of the device descriptors
    std::vector<std::vector<uint32_t>> nmc, unit_base, unit_chunk;
    std::vector<size_t> count_off;
    DevBuf d_desc, d_items, d_next, d_counts;
    uint32_t nitems = 0;
    int blocks = 0;
    double flops = 0;
    bool operands = false;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    void drop_graph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~gs_batch()
    {
        drop_graph();
        if (cap) cudaStreamDestroy(cap);
    }
};

namespace gs {
namespace {

constexpr uint32_t kGrab = 4;  // items a warp takes per atomic

// MAXK: the widest block in the batch (8, 16 or 32); narrower instantiations need fewer
// registers and keep more warps resident
template <class T, int MAXK>
__global__ void __launch_bounds__(256) k_batch(const mm::MMArgs *__restrict__ desc,
                                               const uint2 *__restrict__ items, uint32_t nitems,
                                               uint32_t *next)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        uint32_t first = 0;
        if (lane == 0) first = atomicAdd(next, kGrab);
        first = __shfl_sync(0xffffffffu, first, 0);
        if (first >= nitems) return;
        const uint32_t last = min(nitems, first + kGrab);
        for (uint32_t it = first; it < last; it++) {
            const uint2 w = items[it];
            const uint32_t mi = w.x >> 5, rb = w.x & 31u;
            const mm::MMArgs &a = desc[mi];
            const uint32_t kb = a.ld / a.nrb;
            if (kb == 1) mm::mm_unit<T, 1, false>(a, w.y, rb);
            else if (kb == 2) mm::mm_unit<T, 2, false>(a, w.y, rb);
            else if (kb == 4) mm::mm_unit<T, 4, false>(a, w.y, rb);
            else if (kb == 8) mm::mm_unit<T, 8, false>(a, w.y, rb);
            else if constexpr (MAXK >= 16) {
                if (kb == 16) mm::mm_unit<T, 16, false>(a, w.y, rb);
                else if constexpr (MAXK >= 32) mm::mm_unit<T, 32, false>(a, w.y, rb);
            }
        }
    }
}

uint32_t pow2_at_least(uint32_t k)
{
    uint32_t p = 1;
    while (p < k) p <<= 1;
    return p;
}

// (re)build the work list and the device descriptors for the current block widths
gs_status build_items(gs_batch *B, cudaStream_t s)
{
    struct Item {
        uint64_t cost;
        uint32_t x, y;
    };
    std::vector<Item> items;
    for (size_t i = 0; i < B->mats.size(); i++) {
        const gs_matrix *A = B->mats[i];
        const uint32_t nrb = B->kpad[i] / B->kb[i];
        for (uint32_t u = 0; u < A->k1units; u++) {
            const uint32_t c = B->unit_chunk[i][u];
            const uint32_t piece = u - B->unit_base[i][c];
            const uint32_t nmc = B->nmc[i][c];
            const uint32_t steps = nmc > piece * kK1Split ? std::min(nmc - piece * kK1Split, kK1Split) : 0u;
            for (uint32_t rb = 0; rb < nrb; rb++)
                items.push_back({(uint64_t)(steps + 1) * (B->kb[i] + 4), ((uint32_t)i << 5) | rb, u});
        }
        B->desc[i].ld = B->kpad[i];
        B->desc[i].nrb = nrb;
    }
    std::stable_sort(items.begin(), items.end(),
                     [](const Item &a, const Item &b) { return a.cost > b.cost; });
    std::vector<uint2> packed(items.size());
    for (size_t t = 0; t < items.size(); t++) packed[t] = make_uint2(items[t].x, items[t].y);
    B->nitems = (uint32_t)items.size();
    GS_TRY(B->d_items.alloc(packed.size() * sizeof(uint2) + 16));
    if (!packed.empty())
        GS_CUDA(cudaMemcpyAsync(B->d_items.p, packed.data(), packed.size() * sizeof(uint2),
                                cudaMemcpyHostToDevice, s));
    GS_CUDA(cudaMemcpyAsync(B->d_desc.p, B->desc.data(), B->desc.size() * sizeof(mm::MMArgs),
                            cudaMemcpyHostToDevice, s));
    GS_CUDA(cudaStreamSynchronize(s));
    B->drop_graph();
    return GS_OK;
}

template <class T, int MAXK>
gs_status launch_batch(gs_batch *B, cudaStream_t s)
{
    int per_sm = 0, dev = 0, sms = 148;
    GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<T, MAXK>, 256, 0));
    GS_CUDA(cudaGetDevice(&dev));
    GS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    B->blocks = std::max(1, per_sm) * sms;  // persistent: every resident block, once
    GS_CUDA(cudaMemsetAsync(B->d_next.p, 0, 4, s));
    if (B->nitems)
        k_batch<T, MAXK><<<B->blocks, 256, 0, s>>>(B->d_desc.as<mm::MMArgs>(),
                                                   B->d_items.as<uint2>(), B->nitems,
                                                   B->d_next.as<uint32_t>());
    GS_CHECK_LAUNCH();
    return GS_OK;
}

template <class T>
gs_status launch_t(gs_batch *B, cudaStream_t s)
{
    const uint32_t w = B->kb.empty() ? 1u : *std::max_element(B->kb.begin(), B->kb.end());
    if (w <= 8) return launch_batch<T, 8>(B, s);
    if (w <= 16) return launch_batch<T, 16>(B, s);
    return launch_batch<T, 32>(B, s);
}

gs_status launch(gs_batch *B, cudaStream_t s)
{
    return B->vtype == GS_F64 ? launch_t<double>(B, s) : launch_t<float>(B, s);
}

}  // namespace
}  // namespace gs

using namespace gs;

extern "C" {

gs_status gs_batch_create(gs_batch **out, UIN count, gs_matrix *const *mats, const UIN *k,
                          gs_stream stream)
{
    if (!out || (count && (!mats || !k))) return fail(GS_ERR_INVALID, "NULL argument");
    *out = nullptr;
    if (count >= (1u << 27)) return fail(GS_ERR_UNSUPPORTED, "batch of %u matrices", count);
    cudaStream_t s = cs(stream);
    auto *B = new gs_batch();
    auto bail = [&](gs_status st) { delete B; return st; };
    for (UIN i = 0; i < count; i++) {
        gs_matrix *A = mats[i];
        if (!A) return bail(fail(GS_ERR_INVALID, "matrix %u is NULL", i));
        if (A->p.format != GS_FMT_K1 || A->p.itype != GS_IDX_U32 ||
            (A->p.vtype != GS_F64 && A->p.vtype != GS_F32))
            return bail(fail(GS_ERR_UNSUPPORTED,
                             "matrix %u: batches take K1 matrices with FP64 or FP32 values and "
                             "32-bit columns", i));
        if (i && A->p.vtype != mats[0]->p.vtype)
            return bail(fail(GS_ERR_UNSUPPORTED, "matrix %u: all matrices share one value type", i));
        if (k[i] < 1 || k[i] > 32)
            return bail(fail(GS_ERR_UNSUPPORTED, "matrix %u: %u right-hand sides (1..32)", i, k[i]));
        gs_status st = prepare_mm_scratch(A, s);
        if (st) return bail(st);
    }
    B->vtype = count ? mats[0]->p.vtype : GS_F64;
    B->mats.assign(mats, mats + count);
    B->k.assign(k, k + count);
    B->kpad.resize(count);
    B->kb.resize(count);
    B->desc.resize(count);
    B->nmc.resize(count);
    B->unit_base.resize(count);
    B->unit_chunk.resize(count);
    B->count_off.resize(count + 1, 0);
    for (UIN i = 0; i < count; i++) {
        const gs_matrix *A = mats[i];
        B->kpad[i] = pow2_at_least(k[i]);
        B->kb[i] = B->kpad[i];
        B->count_off[i + 1] = B->count_off[i] + (size_t)A->chunkNum * B->kpad[i];
        B->flops += 2.0 * (double)A->nnz * (double)k[i];
        B->nmc[i].resize(A->chunkNum);
        B->unit_base[i].resize((size_t)A->chunkNum + 1);
        B->unit_chunk[i].resize(A->k1units);
        if (A->chunkNum) {
            cudaError_t e = cudaMemcpy(B->nmc[i].data(), A->nmc.p, (size_t)A->chunkNum * 4,
                                       cudaMemcpyDeviceToHost);
            if (e == cudaSuccess)
                e = cudaMemcpy(B->unit_base[i].data(), A->k1unit_base.p,
                               ((size_t)A->chunkNum + 1) * 4, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess && A->k1units)
                e = cudaMemcpy(B->unit_chunk[i].data(), A->k1unit_chunk.p, (size_t)A->k1units * 4,
                               cudaMemcpyDeviceToHost);
            if (e != cudaSuccess)
                return bail(fail(GS_ERR_CUDA, "batch plan copy: %s", cudaGetErrorString(e)));
        }
    }
    gs_status st;
    if ((st = B->d_counts.alloc_zero(B->count_off[count] * 4 + 4, s)) ||
        (st = B->d_next.alloc_zero(4, s)) ||
        (st = B->d_desc.alloc(std::max<size_t>(1, count) * sizeof(mm::MMArgs))))
        return bail(st);
    for (UIN i = 0; i < count; i++) {
        gs_matrix *A = mats[i];
        mm::MMArgs &a = B->desc[i];
        a = mm::MMArgs{};
        a.nrows = A->nrows;
        a.permi = A->permi.as<uint32_t>();
        a.nmc = A->nmc.as<uint32_t>();
        a.chp = A->chp.as<uint32_t>();
        a.klen = A->k1len.as<uint32_t>();
        a.val = A->val.p;
        a.col = A->col.as<uint32_t>();
        a.unit_chunk = A->k1unit_chunk.as<uint32_t>();
        a.unit_base = A->k1unit_base.as<uint32_t>();
        a.units = A->k1units;
        a.split_units = A->k1split_units;
        a.partial = A->mmpartial.p;
        a.count = B->d_counts.as<uint32_t>() + B->count_off[i];
    }
    if ((st = build_items(B, s))) return bail(st);
    *out = B;
    return GS_OK;
}

gs_status gs_batch_destroy(gs_batch *B)
{
    if (!B) return GS_OK;
    cudaDeviceSynchronize();
    delete B;
    return GS_OK;
}

gs_status gs_batch_info(const gs_batch *B, UIN *nitems, UIN *kpad, double *flops)
{
    if (!B) return fail(GS_ERR_INVALID, "NULL argument");
    if (nitems) *nitems = B->nitems;
    if (kpad)
        for (size_t i = 0; i < B->kpad.size(); i++) kpad[i] = B->kpad[i];
    if (flops) *flops = B->flops;
    return GS_OK;
}

gs_status gs_batch_set_operands(gs_batch *B, void *const *d_X, void *const *d_Y, gs_stream stream)
{
    if (!B || (!B->mats.empty() && (!d_X || !d_Y))) return fail(GS_ERR_INVALID, "NULL argument");
    for (size_t i = 0; i < B->mats.size(); i++) {
        if (!d_X[i] || !d_Y[i]) return fail(GS_ERR_INVALID, "operand %zu is NULL", i);
        if ((reinterpret_cast<uintptr_t>(d_X[i]) | reinterpret_cast<uintptr_t>(d_Y[i])) & 31u)
            return fail(GS_ERR_INVALID, "operands of matrix %zu must be 32-byte aligned", i);
        B->desc[i].xin = d_X[i];
        B->desc[i].yout = d_Y[i];
    }
    cudaStream_t s = cs(stream);
    if (!B->mats.empty())
        GS_CUDA(cudaMemcpyAsync(B->d_desc.p, B->desc.data(), B->desc.size() * sizeof(mm::MMArgs),
                                cudaMemcpyHostToDevice, s));
    GS_CUDA(cudaStreamSynchronize(s));  // the host table is reused by later calls
    B->operands = true;
    return GS_OK;
}

gs_status gs_batch_set_blocking(gs_batch *B, const UIN *kb, gs_stream stream)
{
    if (!B || (!B->mats.empty() && !kb)) return fail(GS_ERR_INVALID, "NULL argument");
    for (size_t i = 0; i < B->mats.size(); i++) {
        const UIN w = kb[i];
        if (w == 0 || (w & (w - 1)) || w > B->kpad[i])
            return fail(GS_ERR_INVALID, "matrix %zu: block width %u must be a power of two "
                                        "<= %u", i, w, B->kpad[i]);
    }
    std::copy(kb, kb + B->mats.size(), B->kb.begin());
    return build_items(B, cs(stream));
}

gs_status gs_batch_run(gs_batch *B, gs_stream stream)
{
    if (!B) return fail(GS_ERR_INVALID, "NULL argument");
    if (!B->operands) return fail(GS_ERR_INVALID, "gs_batch_set_operands must run first");
    return launch(B, cs(stream));
}

gs_status gs_batch_run_graph(gs_batch *B, gs_stream stream)
{
    if (!B) return fail(GS_ERR_INVALID, "NULL argument");
    if (!B->operands) return fail(GS_ERR_INVALID, "gs_batch_set_operands must run first");
    if (!B->exec) {
        if (!B->cap) GS_CUDA(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking));
        GS_CUDA(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
        const gs_status st = launch(B, B->cap);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(B->cap, &g);
        if (st) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return fail(GS_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
        B->graph = g;
        GS_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
    }
    GS_CUDA(cudaGraphLaunch(B->exec, cs(stream)));
    return GS_OK;
}

}  // extern "C"
