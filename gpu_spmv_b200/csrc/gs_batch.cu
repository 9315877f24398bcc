// gs_batch.cu -- many K1 matrices of uneven size, each with its own right-hand sides, in one
// persistent launch.
//
// Two kinds of work.  K1 units: one warp per (matrix, K1 unit, right-hand-side block), the
// multi-RHS K1 product of gs_mm.cuh, gathering X rows through L1 / L2.  Row blocks: one
// thread block per (matrix, block of consecutive rows, right-hand-side block) for matrices
// whose rows touch a narrow band of columns.  The block's CSR value and column segments and
// the rows lo..hi-1 of X its columns reach are staged into shared memory (1-D TMA bulk
// copies completing on an mbarrier; X by plain loads when its block is strided), and every
// X access of the product is then a shared-memory load: for banded matrices whose X rows
// all sit in L2 the K1 gathers are bound by the L1TEX line rate, which the staged loads do
// not touch.  A row block's rows are cut at the same kK1Split-element pieces as K1 and
// summed in the same order, so either kind gives the same bits as the single-matrix K1
// product.  Each matrix takes row blocks where its blocks fit the shared-memory budget
// (GS_BATCH_AUTO), or the kind the caller sets.
//
// Work list: ordered by decreasing work (longest first), so the persistent blocks (warps
// for a K1-only batch), which take items from an atomic counter, finish together.  Each
// matrix keeps its own right-hand-side block width kb (a divisor of its padded count kpad;
// chosen by the autotuner), and its descriptors (layout arrays, operands, scratch) live in
// device memory, so new operands need no new launch configuration: a CUDA graph captured
// once (counter reset + kernel) is replayed as is.
//
// No counterpart in the reference, which runs one matrix and one right-hand side per call.
#include <algorithm>
#include <numeric>
#include <vector>

#include "gs_bulk.cuh"
#include "gs_mm.cuh"

using gs::DevBuf;
using gs::fail;

namespace gs {
// One row block: rows row0..row1-1 of the matrix, which read X rows lo..hi-1; its elements
// are e0..e1-1 of the block-ordered arrays.
struct BandBlock {
    uint32_t row0, row1, lo, hi, e0, e1, pad0, pad1;
};
// Row-block form of one matrix, planned once at its padded width kpad (a narrower block of
// right-hand sides only shrinks a block's X rows): consecutive rows while their X rows and
// elements fit a thread block's shared memory.  Inside a block the rows are ordered by
// decreasing length (ties by row), each row's elements in CSR order padded with zeros to a
// multiple of 4; info[p] of the row at position p of this order: x = its element offset in
// the block | (row - row0) << 16, y = its length.
struct BandMat {
    bool tried = false, fits = false;
    uint32_t rows_max = 0;  // rows per block at most (the height of the row blocks)
    DevBuf info, col, val, blocks;
    std::vector<BandBlock> hblocks;
};
// Device descriptor of a matrix in row-block form.
struct BandArgs {
    const uint2 *info;
    const uint32_t *col;
    const void *val;
    const BandBlock *blocks;
    const void *xin;
    void *yout;
    uint32_t ld, nrb;
    uint32_t xbulk;  // 1: a block's X rows are contiguous (kb = ld, kb values >= 16 bytes)
};
}  // namespace gs

struct gs_batch {
    gs_dtype vtype = GS_F64;
    std::vector<gs_matrix *> mats;
    std::vector<uint32_t> k, kpad, kb;
    std::vector<uint32_t> path_req, path;  // requested (GS_BATCH_*), effective (K1 / BAND)
    std::vector<gs::mm::MMArgs> desc;  // host copy of the device descriptors
    std::vector<gs::BandArgs> bdesc;
    std::vector<gs::BandMat> band;
    std::vector<std::vector<uint32_t>> nmc, unit_base, unit_chunk;
    std::vector<size_t> count_off;
    DevBuf d_desc, d_bdesc, d_items, d_bitems, d_next, d_counts, d_status;
    uint32_t nitems = 0;   // K1 items (warp kernel)
    uint32_t nbitems = 0;  // row-block items (thread-block kernel)
    uint32_t maxk1 = 0;    // widest block of the matrices that run as K1 units
    int bblocks = 0;
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

// ---------------------------------------------------------------------------------------
// Row blocks with the X band in shared memory.
constexpr int kBandConsumers = 736;                   // 23 warps multiply
constexpr int kBandThreads = kBandConsumers + 32;     // + 1 warp stages the blocks
constexpr uint32_t kBandSmem = 110u * 1024u;          // shared memory per stage
constexpr int kBandStages = 2;                        // one block per SM: 220 KB
constexpr uint32_t kBandRowsMax = 4096;        // rows per block (< 2^16: packed in info)
constexpr uint32_t kBandPad = 4;               // row segments start on multiples of 4 elements

__host__ __device__ __forceinline__ size_t round16(size_t b) { return (b + 15) & ~size_t(15); }

// Shared-memory bytes of a row block: X rows lo..hi-1 (row_bytes each), the value and
// column segments of its elements e0..e1-1 (multiples of 4: 16-byte multiples), and its
// row infos (widened to 16-byte boundaries of the array), in that order.
struct BandBytes {
    size_t x, v, c, i;
};
__host__ __device__ __forceinline__ BandBytes band_bytes(uint32_t lo, uint32_t hi, uint32_t e0,
                                                         uint32_t e1, uint32_t row0,
                                                         uint32_t row1, size_t row_bytes,
                                                         size_t vsize)
{
    BandBytes b;
    b.x = hi > lo ? round16((size_t)(hi - lo) * row_bytes) : 0;
    b.v = (size_t)(e1 - e0) * vsize;
    b.c = (size_t)(e1 - e0) * 4;
    b.i = row1 > row0 ? round16((size_t)row1 * 8) - (((size_t)row0 * 8) & ~size_t(15)) : 0;
    return b;
}

// V consecutive values from shared memory (16, 8 or 4 bytes, aligned to that)
template <class T, int V>
__device__ __forceinline__ void lds_vec(const T *p, T (&v)[V])
{
    if constexpr (V * sizeof(T) == 16 && sizeof(T) == 4) {
        const float4 w = *reinterpret_cast<const float4 *>(p);
        v[0] = w.x, v[1] = w.y, v[2] = w.z, v[3] = w.w;
    } else if constexpr (V * sizeof(T) == 16) {
        const double2 w = *reinterpret_cast<const double2 *>(p);
        v[0] = w.x, v[1] = w.y;
    } else if constexpr (V * sizeof(T) == 8 && sizeof(T) == 4) {
        const float2 w = *reinterpret_cast<const float2 *>(p);
        v[0] = w.x, v[1] = w.y;
    } else {
#pragma unroll
        for (int k = 0; k < V; k++) v[k] = p[k];
    }
}
template <class T, int V>
__device__ __forceinline__ void stg_vec(T *p, const T (&v)[V])
{
    if constexpr (V * sizeof(T) == 16 && sizeof(T) == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (V * sizeof(T) == 16) {
        *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
    } else if constexpr (V * sizeof(T) == 8 && sizeof(T) == 4) {
        *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
    } else {
#pragma unroll
        for (int k = 0; k < V; k++) p[k] = v[k];
    }
}
// 4 values of a row segment (16-byte aligned in shared memory)
__device__ __forceinline__ void lds4(const float *p, float (&v)[4])
{
    const float4 w = *reinterpret_cast<const float4 *>(p);
    v[0] = w.x, v[1] = w.y, v[2] = w.z, v[3] = w.w;
}
__device__ __forceinline__ void lds4(const double *p, double (&v)[4])
{
    const double2 a = *reinterpret_cast<const double2 *>(p);
    const double2 b = *reinterpret_cast<const double2 *>(p + 2);
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}

// Two FP32 sums at once (sm_100 packed f32x2 add): each half rounds exactly as the scalar
// add.rn.  The products stay scalar mul.rn: ptxas contracts a packed multiply feeding a
// packed add into a fused multiply-add, which would change the bits.
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b)
{
    float2 d;
    asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
        " add.rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
// acc[k] = acc[k] + v x[k] for k < V, multiply and add rounded separately
template <class T, int V>
__device__ __forceinline__ void madd_row(T (&acc)[V], T v, const T (&x)[V])
{
    if constexpr (std::is_same<T, float>::value && V % 2 == 0) {
#pragma unroll
        for (int k = 0; k < V; k += 2) {
            const float2 p = make_float2(__fmul_rn(v, x[k]), __fmul_rn(v, x[k + 1]));
            const float2 r = add2_rn(make_float2(acc[k], acc[k + 1]), p);
            acc[k] = r.x;
            acc[k + 1] = r.y;
        }
    } else {
        using A = mm::Arith<T>;
#pragma unroll
        for (int k = 0; k < V; k++) acc[k] = A::add(acc[k], A::mul(v, x[k]));
    }
}

// The dynamic shared memory of the row-block kernel (named here so that every access in the
// non-inlined block function is known to be a shared-memory one)
extern __shared__ __align__(128) unsigned char g_band_smem[];

// The rows of a staged block, K right-hand sides: P lanes per row (16 bytes of the row's K
// values each, or one lane for rows under 16 bytes), rows taken in the block's order (longest
// first) round-robin by the lane groups, so the rows of a warp have similar lengths.  Each
// row sums its products in element order, restarting every kK1Split elements and adding the
// pieces in order, as the K1 kernels do.  sxo, svo, sco, sio: byte offsets in shared memory
// of X row lo, the value and column segments and the row infos.  Consumer threads only.
template <class T, int K>
__device__ __forceinline__ void band_rows(const BandArgs &m, uint32_t row0, uint32_t nr,
                                          uint32_t lo, uint32_t sxo, uint32_t svo,
                                          uint32_t sco, uint32_t sio, uint32_t off)
{
    using A = mm::Arith<T>;
    constexpr int P = (K * (int)sizeof(T) >= 16) ? K * (int)sizeof(T) / 16 : 1;
    constexpr int V = K / P;
    constexpr int G = kBandConsumers / P;
    constexpr uint32_t rowb = K * sizeof(T);
    const int grp = (int)threadIdx.x / P, pl = (int)threadIdx.x % P;
    T *__restrict__ y = static_cast<T *>(m.yout) + off + pl * V;
    // X row c at byte xo + c * rowb (modulo 2^32: xo wraps below zero for lo > 0)
    const uint32_t xo = sxo + (uint32_t)(pl * V * (int)sizeof(T)) - lo * rowb;
    const uint2 *sinfo = reinterpret_cast<const uint2 *>(g_band_smem + sio);
#pragma unroll 1
    for (uint32_t i = (uint32_t)grp; i < nr; i += G) {
        const uint2 inf = sinfo[i];
        const uint32_t st = inf.x & 0xffffu, len = inf.y;
        const T *rv = reinterpret_cast<const T *>(g_band_smem + svo) + st;
        const uint32_t *rc = reinterpret_cast<const uint32_t *>(g_band_smem + sco) + st;
        T tot[V];
#pragma unroll 1
        for (uint32_t p0 = 0;; p0 += kK1Split) {
            T acc[V];
#pragma unroll
            for (int k = 0; k < V; k++) acc[k] = T(0);
            const uint32_t pe = min(len, p0 + kK1Split);
            uint32_t j = p0;
#pragma unroll 1
            for (; j + kBandPad <= pe; j += kBandPad) {
                T v[4], xv[4][V];
                lds4(rv + j, v);
                const uint4 c4 = *reinterpret_cast<const uint4 *>(rc + j);
                const uint32_t c[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
                for (int b = 0; b < 4; b++)
                    lds_vec<T, V>(reinterpret_cast<const T *>(g_band_smem + (xo + c[b] * rowb)), xv[b]);
#pragma unroll
                for (int b = 0; b < 4; b++) madd_row<T, V>(acc, v[b], xv[b]);
            }
            if (j < pe) {  // the last 1-3 elements
                T v[4], xv[4][V];
                lds4(rv + j, v);
                const uint4 c4 = *reinterpret_cast<const uint4 *>(rc + j);
                const uint32_t c[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
                for (int b = 0; b < 3; b++) {
                    if (j + b < pe) {
                        lds_vec<T, V>(reinterpret_cast<const T *>(g_band_smem + (xo + c[b] * rowb)), xv[b]);
                        madd_row<T, V>(acc, v[b], xv[b]);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < V; k++) tot[k] = p0 == 0 ? acc[k] : A::add(tot[k], acc[k]);
            if (pe >= len) break;
        }
        stg_vec<T, V>(y + (size_t)(row0 + (inf.x >> 16)) * m.ld, tot);
    }
}

// Plan of one staged item, written by the producer before it arrives on the stage's full
// barrier (whose completion makes it visible to the consumers).
struct BandStage {
    uint32_t valid, mi, rb, row0, nr, lo, hi;
    uint32_t svo, sco, sio;  // byte offsets in the stage buffer
};

// Producer, before its stage is free: item w's descriptors and copy sizes.
struct BandPlan {
    BandStage st;
    const void *val, *col, *info, *x;
    uint32_t e0, nv, nc, ni, nx;  // nx: bytes of X by bulk copy (0: none or plain loads)
    size_t i0;
};
template <class T>
__device__ __forceinline__ BandPlan band_plan(const BandArgs *__restrict__ bdesc, uint2 w)
{
    BandPlan p;
    const uint32_t mi = w.x >> 5, rb = w.x & 31u;
    const BandArgs &m = bdesc[mi];
    const uint32_t K = m.ld / m.nrb;
    const uint4 q0 = __ldg(reinterpret_cast<const uint4 *>(m.blocks + w.y));
    const uint4 q1 = __ldg(reinterpret_cast<const uint4 *>(m.blocks + w.y) + 1);
    const uint32_t row0 = q0.x, row1 = q0.y, lo = q0.z, hi = q0.w, e0 = q1.x, e1 = q1.y;
    const BandBytes nb = band_bytes(lo, hi, e0, e1, row0, row1, (size_t)K * sizeof(T), sizeof(T));
    p.i0 = ((size_t)row0 * 8) & ~size_t(15);
    p.st.valid = 1;
    p.st.mi = mi;
    p.st.rb = rb;
    p.st.row0 = row0;
    p.st.nr = row1 - row0;
    p.st.lo = lo;
    p.st.hi = hi;
    p.st.svo = (uint32_t)nb.x;
    p.st.sco = p.st.svo + (uint32_t)nb.v;
    p.st.sio = p.st.sco + (uint32_t)nb.c;
    p.val = static_cast<const T *>(m.val) + e0;
    p.col = m.col + e0;
    p.info = reinterpret_cast<const unsigned char *>(m.info) + p.i0;
    p.x = static_cast<const T *>(m.xin) + (size_t)lo * K;
    p.e0 = e0;
    p.nv = (uint32_t)nb.v;
    p.nc = (uint32_t)nb.c;
    p.ni = (uint32_t)nb.i;
    p.nx = m.xbulk ? (uint32_t)nb.x : 0u;
    return p;
}
// Producer, once the stage is free: the plan -> st, the bulk copies into stage buffer `buf`
// (values, columns, row infos, and X rows lo..hi-1 when contiguous), completing on `full`.
__device__ __forceinline__ void band_arm(const BandPlan &p, BandStage &st, uint32_t buf,
                                         uint64_t *full)
{
    st = p.st;
    st.sio = p.st.sio + (uint32_t)((size_t)p.st.row0 * 8 - p.i0);
    unsigned char *b = g_band_smem + buf;
    bulk::mbar_expect_tx(full, p.nv + p.nc + p.ni + p.nx);  // the producer's arrival too
    if (p.nv) bulk::bulk_g2s(b + p.st.svo, p.val, p.nv, full);
    if (p.nc) bulk::bulk_g2s(b + p.st.sco, p.col, p.nc, full);
    if (p.ni) bulk::bulk_g2s(b + p.st.sio, p.info, p.ni, full);
    if (p.nx) bulk::bulk_g2s(b, p.x, p.nx, full);
}

// Consumers: one staged item (its copies complete), K right-hand sides.
template <class T, int K>
__device__ __noinline__ void band_item(const BandArgs &m, const BandStage &st, uint32_t buf)
{
    const uint32_t off = st.rb * K;
    constexpr size_t rowb = K * sizeof(T);
    if (m.xbulk == 0 && st.hi > st.lo) {
        // strided or narrow X block: plain loads, 16 bytes (or the whole row) per thread
        constexpr uint32_t u = rowb >= 16 ? 16 : (uint32_t)rowb;
        constexpr uint32_t upr = (uint32_t)rowb / u;
        const uint32_t total = (st.hi - st.lo) * upr;
        const unsigned char *xg = static_cast<const unsigned char *>(m.xin) +
                                  ((size_t)st.lo * m.ld + off) * sizeof(T);
        const size_t gstride = (size_t)m.ld * sizeof(T);
        unsigned char *sb = g_band_smem + buf;
#pragma unroll 4
        for (uint32_t q = threadIdx.x; q < total; q += kBandConsumers) {
            const uint32_t row = q / upr, part = q % upr;
            const unsigned char *src = xg + (size_t)row * gstride + part * u;
            unsigned char *dst = sb + row * (uint32_t)rowb + part * u;
            if constexpr (u == 16) *reinterpret_cast<uint4 *>(dst) = __ldg(reinterpret_cast<const uint4 *>(src));
            else if constexpr (u == 8) *reinterpret_cast<uint2 *>(dst) = __ldg(reinterpret_cast<const uint2 *>(src));
            else *reinterpret_cast<uint32_t *>(dst) = __ldg(reinterpret_cast<const uint32_t *>(src));
        }
        asm volatile("bar.sync 1, %0;" ::"n"(kBandConsumers) : "memory");  // consumers only
    }
    band_rows<T, K>(m, st.row0, st.nr, st.lo, buf, buf + st.svo, buf + st.sco, buf + st.sio, off);
}

// Persistent, one block per SM over a work list of row blocks (x = matrix << 5 | right-hand-
// side block, y = row block), warp-specialised: the last warp takes items from the atomic
// counter and stages each into one of two shared-memory buffers with TMA bulk copies (full
// barrier: copies and plan landed); the other 15 warps multiply the staged block and release
// the buffer (empty barrier), so the next block's copies overlap this block's products.
// Every wait is bounded (about 2 s): a timeout sets bit 0 of the status word, and the
// producer waits (bounded) for the copies it issued before it leaves.
template <class T>
__global__ void __launch_bounds__(kBandThreads, 1) k_batch_band(
    const BandArgs *__restrict__ bdesc, const uint2 *__restrict__ items, uint32_t nitems,
    uint32_t *next, uint32_t *status)
{
    __shared__ uint64_t full[kBandStages], empty[kBandStages];
    __shared__ BandStage st[kBandStages];
    if (threadIdx.x == 0) {
        for (int i = 0; i < kBandStages; i++) {
            bulk::mbar_init(&full[i], 1);
            bulk::mbar_init(&empty[i], kBandConsumers / 32);
        }
        bulk::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x >= kBandConsumers) {
        // producer: one lane
        if (threadIdx.x != kBandConsumers) return;
        uint32_t eph = 0;     // bit s: parity of stage s's empty barrier awaited next
        uint32_t issued = 0;  // bit s: stage s has been armed (its copies may be in flight)
        for (uint32_t k = 0;; k++) {
            const int sidx = (int)(k & 1u);
            // the next item's descriptors load while the consumers still use the stage
            const uint32_t it = atomicAdd(next, 1u);
            BandPlan p;
            if (it < nitems) p = band_plan<T>(bdesc, items[it]);
            if ((issued >> sidx) & 1u) {
                if (!bulk::mbar_wait_bounded(&empty[sidx], (eph >> sidx) & 1u)) {
                    atomicOr(status, 1u);
                    // leave only once the copies issued earlier have landed (bounded): the
                    // full barrier of stage t was armed last for phase (k - 2 + t') / 2
                    for (int t = 0; t < kBandStages; t++) {
                        const uint32_t last = (k - 1u - (uint32_t)((sidx + 1 + t) & 1)) >> 1;
                        if ((issued >> t) & 1u) bulk::mbar_wait_bounded(&full[t], last & 1u);
                    }
                    return;
                }
                eph ^= 1u << sidx;
            }
            if (it >= nitems) {
                st[sidx].valid = 0;
                bulk::mbar_expect_tx(&full[sidx], 0);
                return;
            }
            band_arm(p, st[sidx], (uint32_t)sidx * kBandSmem, &full[sidx]);
            issued |= 1u << sidx;
        }
    }
    // consumers
    uint32_t fph = 0;  // bit s: parity of stage s's full barrier awaited next
    for (uint32_t k = 0;; k++) {
        const int sidx = (int)(k & 1u);
        if (!bulk::mbar_wait_bounded(&full[sidx], (fph >> sidx) & 1u)) {
            if ((threadIdx.x & 31) == 0) atomicOr(status, 1u);
            return;
        }
        fph ^= 1u << sidx;
        const BandStage &sp = st[sidx];
        if (!sp.valid) return;
        const BandArgs &m = bdesc[sp.mi];
        const uint32_t kb = m.ld / m.nrb;
        const uint32_t buf = (uint32_t)sidx * kBandSmem;
        if (kb == 1) band_item<T, 1>(m, sp, buf);
        else if (kb == 2) band_item<T, 2>(m, sp, buf);
        else if (kb == 4) band_item<T, 4>(m, sp, buf);
        else if (kb == 8) band_item<T, 8>(m, sp, buf);
        else if (kb == 16) band_item<T, 16>(m, sp, buf);
        else band_item<T, 32>(m, sp, buf);
        // this warp's reads (and plain writes) of the buffer precede its next bulk copies
        bulk::fence_proxy_async();
        __syncwarp();
        if ((threadIdx.x & 31) == 0) bulk::mbar_arrive(&empty[sidx]);
    }
}

// Column range of each row, from the K1 layout (warp per 32-row chunk, lane = sorted row):
// lo = min column, hi = max column + 1 (lo > hi for an empty row), at the original row.
__global__ void k_k1_row_range(uint32_t nrows, uint32_t chunks,
                               const uint32_t *__restrict__ permi, const uint32_t *__restrict__ chp,
                               const uint32_t *__restrict__ klen, const uint32_t *__restrict__ col,
                               uint32_t *__restrict__ lo, uint32_t *__restrict__ hi)
{
    const uint32_t c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31u;
    if (c >= chunks) return;
    const uint32_t g = 32u * c + lane;
    if (g >= nrows) return;
    const uint32_t len = __ldg(klen + g), s0 = __ldg(chp + c) + lane;
    uint32_t a = 0xffffffffu, b = 0;
    for (uint32_t j = 0; j < len; j++) {
        const uint32_t v = __ldcs(col + s0 + 32u * j);
        a = min(a, v);
        b = max(b, v + 1u);
    }
    const uint32_t r = __ldg(permi + g);
    lo[r] = a;
    hi[r] = b;
}

// K1 layout -> row-block arrays: each row's elements (CSR order) from dst[row] on.
template <class T>
__global__ void k_k1_to_band(uint32_t nrows, uint32_t chunks, const uint32_t *__restrict__ permi,
                             const uint32_t *__restrict__ chp, const uint32_t *__restrict__ klen,
                             const T *__restrict__ val, const uint32_t *__restrict__ col,
                             const uint32_t *__restrict__ dst, T *__restrict__ oval,
                             uint32_t *__restrict__ ocol)
{
    const uint32_t c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31u;
    if (c >= chunks) return;
    const uint32_t g = 32u * c + lane;
    if (g >= nrows) return;
    const uint32_t len = __ldg(klen + g), base = __ldg(dst + __ldg(permi + g));
    const uint32_t s0 = __ldg(chp + c) + lane;
    for (uint32_t j = 0; j < len; j++) {
        oval[base + j] = __ldcs(val + s0 + 32u * j);
        ocol[base + j] = __ldcs(col + s0 + 32u * j);
    }
}

uint32_t pow2_at_least(uint32_t k)
{
    uint32_t p = 1;
    while (p < k) p <<= 1;
    return p;
}

// Row-block form of matrix i (allocates, synchronises): column range of every row, blocks
// planned at kpad, the order and offsets inside each block, then the arrays filled on the
// device from the K1 layout.  bm.fits stays false if some single row does not fit.
template <class T>
gs_status build_band_t(gs_batch *B, size_t i, cudaStream_t s)
{
    gs_matrix *A = B->mats[i];
    BandMat &bm = B->band[i];
    bm.tried = true;
    bm.fits = false;
    const uint32_t n = A->nrows;
    const size_t vsize = sizeof(T), rowb = (size_t)B->kpad[i] * vsize;
    std::vector<uint32_t> permi(n), klen(n), lo(n), hi(n);
    DevBuf dlo, dhi;
    GS_TRY(dlo.alloc((size_t)n * 4));
    GS_TRY(dhi.alloc((size_t)n * 4));
    if (n) {
        k_k1_row_range<<<(A->chunkNum + 7) / 8, 256, 0, s>>>(
            n, A->chunkNum, A->permi.as<uint32_t>(), A->chp.as<uint32_t>(),
            A->k1len.as<uint32_t>(), A->col.as<uint32_t>(), dlo.as<uint32_t>(), dhi.as<uint32_t>());
        GS_CHECK_LAUNCH();
        GS_CUDA(cudaMemcpyAsync(permi.data(), A->permi.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
        GS_CUDA(cudaMemcpyAsync(klen.data(), A->k1len.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
        GS_CUDA(cudaMemcpyAsync(lo.data(), dlo.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
        GS_CUDA(cudaMemcpyAsync(hi.data(), dhi.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
        GS_CUDA(cudaStreamSynchronize(s));
    }
    std::vector<uint32_t> rl(n, 0);
    for (uint32_t g = 0; g < n; g++) rl[permi[g]] = klen[g];
    auto padded = [](uint32_t len) { return (len + kBandPad - 1) / kBandPad * kBandPad; };
    // blocks: consecutive rows while everything fits (one X width: kpad)
    std::vector<BandBlock> blocks;
    {
        auto fits = [&](uint32_t l, uint32_t h, uint64_t e, uint32_t r0, uint32_t r1) {
            if (e > 0xffffu) return false;  // element offsets are packed in 16 bits
            const BandBytes b = band_bytes(l, h, 0, (uint32_t)e, r0, r1, rowb, vsize);
            return b.x + b.v + b.c + b.i <= kBandSmem;
        };
        uint32_t r0 = 0, l = 0xffffffffu, h = 0;
        uint64_t e = 0, etot = 0;
        for (uint32_t r = 0; r < n; r++) {
            const bool empty = lo[r] >= hi[r];
            uint32_t nl = empty ? l : std::min(l, lo[r]), nh = empty ? h : std::max(h, hi[r]);
            uint64_t ne = e + padded(rl[r]);
            if (r > r0 && (r - r0 >= bm.rows_max || !fits(nl, nh, ne, r0, r + 1))) {
                blocks.push_back({r0, r, l < h ? l : 0u, l < h ? h : 0u, (uint32_t)etot,
                                  (uint32_t)(etot + e), 0u, 0u});
                etot += e;
                r0 = r;
                nl = empty ? 0xffffffffu : lo[r];
                nh = empty ? 0u : hi[r];
                ne = padded(rl[r]);
            }
            if (!fits(nl, nh, ne, r0, r + 1)) return GS_OK;  // this row alone does not fit
            l = nl;
            h = nh;
            e = ne;
        }
        if (r0 < n)
            blocks.push_back({r0, n, l < h ? l : 0u, l < h ? h : 0u, (uint32_t)etot,
                              (uint32_t)(etot + e), 0u, 0u});
        if (etot + e >= (1ull << 32))
            return fail(GS_ERR_OVERFLOW, "matrix %zu: padded row blocks exceed 2^32 elements", i);
    }
    // order inside each block: decreasing length, ties by row
    std::vector<uint32_t> dst(n);
    std::vector<uint2> info(n);
    std::vector<uint32_t> ord;
    for (const BandBlock &bk : blocks) {
        ord.resize(bk.row1 - bk.row0);
        std::iota(ord.begin(), ord.end(), bk.row0);
        std::stable_sort(ord.begin(), ord.end(),
                         [&](uint32_t a, uint32_t b) { return rl[a] > rl[b]; });
        uint32_t at = 0;
        for (uint32_t p = 0; p < (uint32_t)ord.size(); p++) {
            const uint32_t r = ord[p];
            dst[r] = bk.e0 + at;
            info[bk.row0 + p] = make_uint2(at | ((r - bk.row0) << 16), rl[r]);
            at += padded(rl[r]);
        }
    }
    const size_t etot = blocks.empty() ? 0 : blocks.back().e1;
    DevBuf ddst;
    GS_TRY(ddst.alloc((size_t)n * 4));
    GS_TRY(bm.info.alloc((size_t)n * 8));
    GS_TRY(bm.col.alloc_zero(etot * 4, s));
    GS_TRY(bm.val.alloc_zero(etot * vsize, s));
    GS_TRY(bm.blocks.alloc(std::max<size_t>(1, blocks.size()) * sizeof(BandBlock)));
    if (n) {
        GS_CUDA(cudaMemcpyAsync(ddst.p, dst.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
        GS_CUDA(cudaMemcpyAsync(bm.info.p, info.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
        GS_CUDA(cudaMemcpyAsync(bm.blocks.p, blocks.data(), blocks.size() * sizeof(BandBlock),
                                cudaMemcpyHostToDevice, s));
        k_k1_to_band<T><<<(A->chunkNum + 7) / 8, 256, 0, s>>>(
            n, A->chunkNum, A->permi.as<uint32_t>(), A->chp.as<uint32_t>(), A->k1len.as<uint32_t>(),
            A->val.as<T>(), A->col.as<uint32_t>(), ddst.as<uint32_t>(), bm.val.as<T>(),
            bm.col.as<uint32_t>());
        GS_CHECK_LAUNCH();
    }
    GS_CUDA(cudaStreamSynchronize(s));
    bm.hblocks = std::move(blocks);
    bm.fits = true;
    return GS_OK;
}

gs_status build_band(gs_batch *B, size_t i, cudaStream_t s)
{
    if (B->band[i].tried) return GS_OK;
    return B->vtype == GS_F64 ? build_band_t<double>(B, i, s) : build_band_t<float>(B, i, s);
}

// (re)build the work list and the device descriptors for the current block widths and paths
gs_status build_items(gs_batch *B, cudaStream_t s)
{
    struct Item {
        uint64_t cost;
        uint32_t x, y;
    };
    const size_t vsize = dtype_size(B->vtype);
    std::vector<Item> items, bitems;
    B->maxk1 = 0;
    for (size_t i = 0; i < B->mats.size(); i++) {
        const gs_matrix *A = B->mats[i];
        const uint32_t nrb = B->kpad[i] / B->kb[i];
        B->desc[i].ld = B->kpad[i];
        B->desc[i].nrb = nrb;
        B->path[i] = GS_BATCH_K1;
        if (B->path_req[i] != GS_BATCH_K1) {
            GS_TRY(build_band(B, i, s));
            if (B->band[i].fits) {
                B->path[i] = GS_BATCH_BAND;
            } else if (B->path_req[i] == GS_BATCH_BAND) {
                return fail(GS_ERR_UNSUPPORTED, "matrix %zu: a row and its X band at %u "
                            "right-hand sides exceed the %u bytes of shared memory of a block",
                            i, B->kpad[i], kBandSmem);
            }
        }
        if (B->path[i] == GS_BATCH_BAND) {
            const BandMat &bm = B->band[i];
            BandArgs &ba = B->bdesc[i];
            ba.info = bm.info.as<uint2>();
            ba.col = bm.col.as<uint32_t>();
            ba.val = bm.val.p;
            ba.blocks = bm.blocks.as<BandBlock>();
            ba.xin = B->desc[i].xin;
            ba.yout = B->desc[i].yout;
            ba.ld = B->kpad[i];
            ba.nrb = nrb;
            ba.xbulk = (nrb == 1 && (size_t)B->kb[i] * vsize >= 16) ? 1u : 0u;
            const uint32_t kb = B->kb[i];
            const uint32_t P = std::max<uint32_t>(1, (uint32_t)(kb * vsize / 16));
            const uint32_t V = kb / P;
            for (uint32_t b = 0; b < (uint32_t)bm.hblocks.size(); b++) {
                const BandBlock &blk = bm.hblocks[b];
                const uint64_t e = blk.e1 - blk.e0;
                const uint64_t cost = (e * P / kBandConsumers + 1) * (V + 4) + (blk.row1 - blk.row0) / 8 +
                                      (uint64_t)(blk.hi - blk.lo) * kb * vsize / 1024;
                for (uint32_t rb = 0; rb < nrb; rb++)
                    bitems.push_back({cost, ((uint32_t)i << 5) | rb, b});
            }
            continue;
        }
        B->maxk1 = std::max(B->maxk1, B->kb[i]);
        for (uint32_t u = 0; u < A->k1units; u++) {
            const uint32_t c = B->unit_chunk[i][u];
            const uint32_t piece = u - B->unit_base[i][c];
            const uint32_t nmc = B->nmc[i][c];
            const uint32_t steps = nmc > piece * kK1Split ? std::min(nmc - piece * kK1Split, kK1Split) : 0u;
            for (uint32_t rb = 0; rb < nrb; rb++)
                items.push_back({(uint64_t)(steps + 1) * (B->kb[i] + 4), ((uint32_t)i << 5) | rb, u});
        }
    }
    auto longest_first = [](const Item &a, const Item &b) { return a.cost > b.cost; };
    auto upload = [&](std::vector<Item> &v, DevBuf &d, uint32_t &n) -> gs_status {
        std::stable_sort(v.begin(), v.end(), longest_first);
        std::vector<uint2> packed(v.size());
        for (size_t t = 0; t < v.size(); t++) packed[t] = make_uint2(v[t].x, v[t].y);
        n = (uint32_t)packed.size();
        GS_TRY(d.alloc(packed.size() * sizeof(uint2) + 16));
        if (!packed.empty())
            GS_CUDA(cudaMemcpyAsync(d.p, packed.data(), packed.size() * sizeof(uint2),
                                    cudaMemcpyHostToDevice, s));
        return GS_OK;
    };
    GS_TRY(upload(items, B->d_items, B->nitems));
    GS_TRY(upload(bitems, B->d_bitems, B->nbitems));
    GS_CUDA(cudaMemcpyAsync(B->d_desc.p, B->desc.data(), B->desc.size() * sizeof(mm::MMArgs),
                            cudaMemcpyHostToDevice, s));
    GS_CUDA(cudaMemcpyAsync(B->d_bdesc.p, B->bdesc.data(), B->bdesc.size() * sizeof(BandArgs),
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
gs_status launch_band(gs_batch *B, cudaStream_t s)
{
    const uint32_t smem = kBandStages * kBandSmem;
    GS_CUDA(cudaFuncSetAttribute(k_batch_band<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    int per_sm = 0, dev = 0, sms = 148;
    GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_band<T>, kBandThreads,
                                                          smem));
    GS_CUDA(cudaGetDevice(&dev));
    GS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    B->bblocks = std::max(1, per_sm) * sms;
    GS_CUDA(cudaMemsetAsync(B->d_next.as<uint32_t>() + 1, 0, 4, s));
    k_batch_band<T><<<B->bblocks, kBandThreads, smem, s>>>(
        B->d_bdesc.as<BandArgs>(), B->d_bitems.as<uint2>(), B->nbitems,
        B->d_next.as<uint32_t>() + 1, B->d_status.as<uint32_t>());
    GS_CHECK_LAUNCH();
    return GS_OK;
}

// The row-block items, then the K1 items: one persistent launch each (a batch whose
// matrices all take one path is one launch)
template <class T>
gs_status launch_t(gs_batch *B, cudaStream_t s)
{
    if (B->nbitems) GS_TRY(launch_band<T>(B, s));
    if (B->nitems || !B->nbitems) {
        if (B->maxk1 <= 8) return launch_batch<T, 8>(B, s);
        if (B->maxk1 <= 16) return launch_batch<T, 16>(B, s);
        return launch_batch<T, 32>(B, s);
    }
    return GS_OK;
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
    if (count >= (1u << 26)) return fail(GS_ERR_UNSUPPORTED, "batch of %u matrices", count);
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
    B->bdesc.resize(count);
    B->band.resize(count);
    for (UIN i = 0; i < count; i++) B->band[i].rows_max = kBandRowsMax;
    B->path_req.assign(count, GS_BATCH_AUTO);
    B->path.assign(count, GS_BATCH_K1);
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
        (st = B->d_next.alloc_zero(8, s)) || (st = B->d_status.alloc_zero(4, s)) ||
        (st = B->d_desc.alloc(std::max<size_t>(1, count) * sizeof(mm::MMArgs))) ||
        (st = B->d_bdesc.alloc(std::max<size_t>(1, count) * sizeof(BandArgs))))
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
    if (nitems) *nitems = B->nitems + B->nbitems;
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
        B->bdesc[i].xin = d_X[i];
        B->bdesc[i].yout = d_Y[i];
    }
    cudaStream_t s = cs(stream);
    if (!B->mats.empty()) {
        GS_CUDA(cudaMemcpyAsync(B->d_desc.p, B->desc.data(), B->desc.size() * sizeof(mm::MMArgs),
                                cudaMemcpyHostToDevice, s));
        GS_CUDA(cudaMemcpyAsync(B->d_bdesc.p, B->bdesc.data(), B->bdesc.size() * sizeof(BandArgs),
                                cudaMemcpyHostToDevice, s));
    }
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
    const std::vector<uint32_t> old = B->kb;
    std::copy(kb, kb + B->mats.size(), B->kb.begin());
    const gs_status st = build_items(B, cs(stream));
    if (st != GS_OK) {  // a matrix held to row blocks does not fit at the new width
        B->kb = old;
        build_items(B, cs(stream));
    }
    return st;
}

gs_status gs_batch_set_row_blocks(gs_batch *B, const UIN *rows_max, gs_stream stream)
{
    if (!B || (!B->mats.empty() && !rows_max)) return fail(GS_ERR_INVALID, "NULL argument");
    for (size_t i = 0; i < B->mats.size(); i++)
        if (rows_max[i] < 32 || rows_max[i] > kBandRowsMax)
            return fail(GS_ERR_INVALID, "matrix %zu: %u rows per block (32..%u)", i, rows_max[i],
                        kBandRowsMax);
    B->drop_graph();  // it may name the row-block arrays replaced below
    std::vector<uint32_t> old(B->mats.size());
    for (size_t i = 0; i < B->mats.size(); i++) {
        BandMat &bm = B->band[i];
        old[i] = bm.rows_max;
        if (bm.rows_max != rows_max[i]) {  // planned again on its next use
            bm = BandMat();
            bm.rows_max = rows_max[i];
        }
    }
    const gs_status st = build_items(B, cs(stream));
    if (st != GS_OK) {
        for (size_t i = 0; i < B->mats.size(); i++) {
            if (B->band[i].rows_max != old[i]) {
                B->band[i] = BandMat();
                B->band[i].rows_max = old[i];
            }
        }
        build_items(B, cs(stream));
    }
    return st;
}

gs_status gs_batch_row_blocks(const gs_batch *B, UIN *rows_max, UIN *blocks)
{
    if (!B) return fail(GS_ERR_INVALID, "NULL argument");
    for (size_t i = 0; i < B->mats.size(); i++) {
        if (rows_max) rows_max[i] = B->band[i].rows_max;
        if (blocks) blocks[i] = B->path[i] == GS_BATCH_BAND ? (UIN)B->band[i].hblocks.size() : 0u;
    }
    return GS_OK;
}

gs_status gs_batch_set_paths(gs_batch *B, const UIN *path, gs_stream stream)
{
    if (!B || (!B->mats.empty() && !path)) return fail(GS_ERR_INVALID, "NULL argument");
    for (size_t i = 0; i < B->mats.size(); i++)
        if (path[i] != GS_BATCH_AUTO && path[i] != GS_BATCH_K1 && path[i] != GS_BATCH_BAND)
            return fail(GS_ERR_INVALID, "matrix %zu: path %u (GS_BATCH_AUTO, _K1 or _BAND)", i,
                        path[i]);
    const std::vector<uint32_t> old = B->path_req;
    std::copy(path, path + B->mats.size(), B->path_req.begin());
    const gs_status st = build_items(B, cs(stream));
    if (st != GS_OK) {
        B->path_req = old;
        build_items(B, cs(stream));
    }
    return st;
}

gs_status gs_batch_paths(const gs_batch *B, UIN *path)
{
    if (!B || (!B->mats.empty() && !path)) return fail(GS_ERR_INVALID, "NULL argument");
    std::copy(B->path.begin(), B->path.end(), path);
    return GS_OK;
}

gs_status gs_batch_status(gs_batch *B, UIN *flags, gs_stream stream)
{
    if (!B || !flags) return fail(GS_ERR_INVALID, "NULL argument");
    cudaStream_t s = cs(stream);
    GS_CUDA(cudaMemcpyAsync(flags, B->d_status.p, 4, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    GS_CUDA(cudaMemsetAsync(B->d_status.p, 0, 4, s));
    GS_CUDA(cudaStreamSynchronize(s));
    return GS_OK;
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
