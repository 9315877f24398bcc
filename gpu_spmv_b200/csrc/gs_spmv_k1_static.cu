// gs_spmv_k1_static.cu -- K1 SpMV over caller-owned device arrays, allocating nothing.
//
// The K1 kernel of gs_spmv_k1.cu cuts long chunks into pieces whose
// partial sums meet in scratch memory (32 doubles per piece, one arrival counter per
// chunk); gs_spmv keeps that scratch, and the piece plan, in the gs_matrix.  This variant
// takes the arrays the reference's gk1 kernel takes (cudaSpmv.cu:851: val, col, nmc, chp,
// permi, x, y, all on the device) and keeps the piece plan and the scratch in the
// file-scope array gs_k1_static_scratch below, so a call makes no allocation of any kind.
//
// Layout of the scratch (one copy per device, 8.25 MiB):
//   partial   kStaticUnits x 32 doubles   partial sums of the pieces of split chunks
//   count     kStaticChunks words         arrival counter of each split chunk
//   unit_base kStaticChunks + 1 words     first piece of each split chunk
//   hdr       2 words                     split chunks S and their pieces, for the launch
//
// K1 chunks come in order of decreasing nmc (rows sorted by decreasing length,
// cudaSpmv.cu:723-737; nmc of a chunk is its first row's length, cudaSpmv.cu:744-749), so
// the chunks that are split form a prefix 0..S-1.  A one-block
// kernel finds S by bisection and writes the piece offsets of that prefix; the SpMV kernel
// then runs split pieces first and every other chunk as one unit.  With nmc out of order
// the bisection still stops at some S: chunks before it are cut into pieces where they are
// longer than one piece, and every chunk from S on runs whole in one warp, whatever its
// length.  When the prefix does not fit the scratch (more than kStaticChunks chunks or
// kStaticUnits pieces) nothing is split and every chunk runs whole.  Every case sums each
// row correctly, but a row summed whole rounds differently from the same row summed in
// pieces, so such results can differ in the last bits (within the FP64 error bound).
// Pieces here are 256 steps long, where gs_spmv on a K1 matrix cuts at 128 steps: on rows
// longer than 128 elements the two entry points also differ in the last bits.  The host
// refuses layouts above GS_K1_STATIC_MAX_SLOTS slots, for which a sorted nmc could need
// more pieces than the scratch holds.
//
// What must start at zero: the arrival counters.  The first call on a device zeroes them
// (with the symbol lookup, before any launch); each launch's last-arriving piece resets
// its chunk's counter, so they are zero again whenever no launch is running.  unit_base
// and hdr are rewritten by every call and partial is written before it is read.
//
// Calls on one device share the scratch: two calls that can run at the same time (two
// streams without an ordering event between them, or two host threads) race on it and
// must be serialised by the caller.
#include <mutex>

#include "gs_internal.cuh"

namespace gs {

namespace {

constexpr uint32_t kStaticSplit = 256;     // steps per piece (the bound below assumes 256)
constexpr uint32_t kStaticUnits = 32768;   // pieces of split chunks
constexpr uint32_t kStaticChunks = 32768;  // split chunks
constexpr size_t kPartialBytes = (size_t)kStaticUnits * 32 * sizeof(double);
constexpr size_t kCountOff = kPartialBytes;
constexpr size_t kCountBytes = (size_t)kStaticChunks * 4;
constexpr size_t kBaseOff = kCountOff + kCountBytes;
constexpr size_t kBaseBytes = ((size_t)(kStaticChunks + 1) * 4 + 255) / 256 * 256;
constexpr size_t kHdrOff = kBaseOff + kBaseBytes;
constexpr size_t kScratchBytes = kHdrOff + 256;
static_assert(GS_K1_STATIC_MAX_SLOTS == 4096ull * kStaticUnits,
              "a sorted layout of at most GS_K1_STATIC_MAX_SLOTS slots needs at most "
              "slots/8192 + slots/8224 < kStaticUnits pieces");

__device__ __align__(256) unsigned char gs_k1_static_scratch[kScratchBytes];

struct K1StaticArgs {
    uint32_t nrows, chunkNum;
    const double *val;
    const uint32_t *col, *nmc, *chp, *permi;
    const double *x;
    double *y;
    double *partial;
    uint32_t *count, *unit_base, *hdr;
};

// One block: S = number of leading chunks longer than kStaticSplit (bisection on the sorted
// nmc), unit_base[c] = first piece of chunk c < S, hdr = {S, pieces}; {0, 0} when the
// prefix does not fit the scratch.
__global__ void __launch_bounds__(1024) k_k1s_prefix(const K1StaticArgs a)
{
    __shared__ uint32_t s_split, s_carry, s_warp[32];
    const uint32_t t = threadIdx.x, lane = t & 31u, wid = t >> 5;
    if (t == 0) {
        uint32_t lo = 0, hi = a.chunkNum;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (__ldg(a.nmc + mid) > kStaticSplit) lo = mid + 1;
            else hi = mid;
        }
        s_split = lo <= kStaticChunks ? lo : 0u;
        s_carry = 0;
    }
    __syncthreads();
    const uint32_t S = s_split;
    for (uint32_t b = 0; b < S; b += 1024) {
        const uint32_t c = b + t;
        uint32_t p = 0;
        if (c < S) {
            p = (__ldg(a.nmc + c) + kStaticSplit - 1) / kStaticSplit;
            p = max(1u, min(p, kStaticUnits + 1));  // bounded: the sum cannot wrap
        }
        uint32_t v = p;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
            if ((int)lane >= o) v += n;
        }
        if (lane == 31) s_warp[wid] = v;
        __syncthreads();
        if (wid == 0) {
            uint32_t w = s_warp[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t n = __shfl_up_sync(0xffffffffu, w, o);
                if ((int)lane >= o) w += n;
            }
            s_warp[lane] = w;
        }
        __syncthreads();
        const uint32_t incl = v + (wid ? s_warp[wid - 1] : 0u);
        const uint32_t carry = s_carry;
        if (c < S) a.unit_base[c] = carry + incl - p;
        __syncthreads();
        if (t == 1023) s_carry = carry + incl;
        __syncthreads();
    }
    if (t == 0) {
        const uint32_t total = s_carry;
        const bool fits = total <= kStaticUnits;
        if (fits) a.unit_base[S] = total;
        a.hdr[0] = fits ? S : 0u;
        a.hdr[1] = fits ? total : 0u;
    }
}

// Work units: pieces of the split prefix first (chunk found by bisection on unit_base),
// then one unit per remaining chunk.  Per lane the sum runs over the chunk's nmc padded
// steps in slot order, like gk1 (cudaSpmv.cu:859-864); pieces of a split chunk are added
// in piece order by whichever warp arrives last.
__global__ void __launch_bounds__(256) k_k1s(const K1StaticArgs a)
{
    const int lane = threadIdx.x & 31;
    const uint32_t S = a.hdr[0], su = a.hdr[1];
    const uint32_t units = su + (a.chunkNum - S);
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < units;
         u += warps) {
        uint32_t c, ub = 0, np = 1, piece = 0;
        if (u < su) {
            uint32_t lo = 0, hi = S - 1;  // last chunk whose first piece is <= u
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) / 2;
                if (__ldg(a.unit_base + mid) <= u) lo = mid;
                else hi = mid - 1;
            }
            c = lo;
            ub = __ldg(a.unit_base + c);
            np = __ldg(a.unit_base + c + 1) - ub;
            piece = u - ub;
        } else {
            c = S + (u - su);
        }
        const uint32_t g = 32u * c + (uint32_t)lane;
        const bool valid = g < a.nrows;
        const uint32_t len = valid ? __ldg(a.nmc + c) : 0u;
        const uint32_t j0 = piece * kStaticSplit;
        const uint32_t j1 = np == 1 ? len : min(len, j0 + kStaticSplit);
        const uint32_t base = __ldg(a.chp + c) + (uint32_t)lane;
        double acc = 0.0;
        uint32_t j = j0;
        for (; j + 8 <= j1; j += 8) {
            double v[8], xv[8];
            uint32_t cc[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t pos = base + 32u * (j + k);
                v[k] = __ldcs(a.val + pos);
                cc[k] = __ldcs(a.col + pos);
            }
#pragma unroll
            for (int k = 0; k < 8; k++) xv[k] = __ldg(a.x + cc[k]);
#pragma unroll
            for (int k = 0; k < 8; k++) acc = __dadd_rn(acc, __dmul_rn(v[k], xv[k]));
        }
        for (; j < j1; j++) {
            const uint32_t pos = base + 32u * j;
            acc = __dadd_rn(acc, __dmul_rn(__ldcs(a.val + pos), __ldg(a.x + __ldcs(a.col + pos))));
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
            if (lane == 0) a.count[c] = 0;  // zero again for the next launch
        }
    }
}

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch[kMaxDevices];

// Address of this device's copy of gs_k1_static_scratch.  The first call per device looks
// the symbol up and zeroes the arrival counters; it synchronises the device, so it belongs
// before any stream capture or timed loop.
gs_status device_scratch(unsigned char **out)
{
    int dev = 0;
    GS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(GS_ERR_UNSUPPORTED, "device ordinal %d is above %d", dev, kMaxDevices - 1);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, gs_k1_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(GS_ERR_CUDA, "cudaGetSymbolAddress(gs_k1_static_scratch) on device %d: %s",
                        dev, cudaGetErrorString(e));
        unsigned char *base = static_cast<unsigned char *>(p);
        GS_CUDA(cudaMemset(base + kCountOff, 0, kCountBytes));
        GS_CUDA(cudaDeviceSynchronize());
        g_scratch[dev] = base;
    }
    *out = g_scratch[dev];
    return GS_OK;
}

}  // namespace

}  // namespace gs

extern "C" gs_status gs_k1_spmv_f64_static(UIN nrows, UIN chunkNum, UIN lenVC,
                                           const double *d_val, const UIN *d_col,
                                           const UIN *d_nmc, const UIN *d_chp,
                                           const UIN *d_permi, const double *d_x,
                                           double *d_y, gs_stream stream)
{
    using namespace gs;
    if (nrows == 0) return GS_OK;
    if (!d_val || !d_col || !d_nmc || !d_chp || !d_permi || !d_x || !d_y)
        return fail(GS_ERR_INVALID, "NULL argument");
    const uint64_t chunks = ((uint64_t)nrows + 31) / 32;
    if (chunkNum != chunks)
        return fail(GS_ERR_INVALID, "chunkNum is %u; a K1 layout of %u rows has %llu chunks",
                    chunkNum, nrows, (unsigned long long)chunks);
    if ((uint64_t)lenVC > GS_K1_STATIC_MAX_SLOTS)
        return fail(GS_ERR_UNSUPPORTED,
                    "K1 layout of %u slots is above the %llu slots the static scratch "
                    "(%u split pieces) is sized for; use gs_matrix_create(GS_FMT_K1) and gs_spmv",
                    lenVC, (unsigned long long)GS_K1_STATIC_MAX_SLOTS, kStaticUnits);
    unsigned char *base = nullptr;
    GS_TRY(device_scratch(&base));
    K1StaticArgs a{};
    a.nrows = nrows;
    a.chunkNum = chunkNum;
    a.val = d_val;
    a.col = d_col;
    a.nmc = d_nmc;
    a.chp = d_chp;
    a.permi = d_permi;
    a.x = d_x;
    a.y = d_y;
    a.partial = reinterpret_cast<double *>(base);
    a.count = reinterpret_cast<uint32_t *>(base + kCountOff);
    a.unit_base = reinterpret_cast<uint32_t *>(base + kBaseOff);
    a.hdr = reinterpret_cast<uint32_t *>(base + kHdrOff);
    cudaStream_t s = cs(stream);
    k_k1s_prefix<<<1, 1024, 0, s>>>(a);
    GS_CHECK_LAUNCH();
    // at most chunkNum + lenVC / 4096 units (sorted layouts); the grid strides over the rest
    const uint64_t units = chunks + lenVC / 4096u;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((units + 7) / 8, 148ull * 64ull);
    k_k1s<<<blocks, 256, 0, s>>>(a);
    GS_CHECK_LAUNCH();
    return GS_OK;
}
