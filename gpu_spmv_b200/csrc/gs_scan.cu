// gs_scan.cu -- error state, device buffers and the device scan / sort primitives used by
// the format converters.
//
// The reference builds every format on the CPU with serial prefix loops (row pointers of
// AXC cudaSpmv.cu:937-948, AXT con cudaSpmv.cu:1158-1201, K1 chunk pointers 741-754) and a
// qsort for the K1 permutation (716-737); its block-local scan micro-benchmark (scan.cu)
// has no carry between blocks.  Here those become one device-wide exclusive scan
// (reduce / scan-of-block-sums / down-sweep, 64-bit offsets so 32-bit overflow is
// detected, no inter-block waiting) and a stable LSD radix sort built on it.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "gs_internal.cuh"

namespace gs {

// ------------------------------------------------------------------ errors
static thread_local char g_err[512] = "";

gs_status fail(gs_status st, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return st;
}
void clear_error() { g_err[0] = 0; }
const char *last_error_text() { return g_err; }

// ------------------------------------------------------------------ DevBuf
gs_status DevBuf::alloc(size_t nbytes)
{
    reset();
    size_t n = ((nbytes + 255) / 256) * 256 + 256;  // slack: vector loads may touch the tail
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        return fail(GS_ERR_ALLOC, "cudaMalloc(%zu) failed: %s", n, cudaGetErrorString(e));
    }
    bytes = nbytes;
    return GS_OK;
}

gs_status DevBuf::alloc_zero(size_t nbytes, cudaStream_t s)
{
    GS_TRY(alloc(nbytes));
    GS_CUDA(cudaMemsetAsync(p, 0, ((nbytes + 255) / 256) * 256 + 256, s));
    return GS_OK;
}

// ------------------------------------------------------------------ scan
// kind follows CountKind's order.
struct CountDev {
    int kind;
    const uint32_t *row;
    const uint32_t *arr;
    uint32_t a;
    __device__ __forceinline__ uint64_t operator()(size_t i) const
    {
        switch (kind) {
        case 0: return (uint64_t)(row[i + 1] - row[i]);
        case 1: {
            uint32_t l = row[i + 1] - row[i];
            return (uint64_t)((l + a - 1) / a);
        }
        case 2: return (uint64_t)arr[i];
        case 3: return (uint64_t)arr[i] * (uint64_t)a;
        case 4: return (uint64_t)(((arr[i] >> a) & 1u) == 0u);
        case 5: {
            uint32_t t = (arr[i] + a - 1) / a;
            return (uint64_t)(t ? t : 1u);
        }
        case 6: {
            uint64_t c = 0;
            for (uint32_t j = 0; j < a; j++) c += __popc(arr[i * a + j]);
            return c;
        }
        default: return (uint64_t)(row[i + 1] > row[i]);
        }
    }
};

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint64_t warp_incl_scan_u64(uint64_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint64_t u = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += u;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive prefix and the
// block total through *total.
__device__ __forceinline__ uint64_t block_excl_scan_u64(uint64_t v, uint64_t *total)
{
    __shared__ uint64_t wsum[kScanThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t inc = warp_incl_scan_u64(v);
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        constexpr int NW = kScanThreads / 32;
        uint64_t s = (lane < NW) ? wsum[lane] : 0;
        uint64_t si = warp_incl_scan_u64(s);
        if (lane < NW) wsum[lane] = si - s;  // exclusive offset of each warp
        if (lane == NW - 1) *total = si;
    }
    __syncthreads();
    uint64_t r = inc - v + wsum[w];
    __syncthreads();
    return r;
}

__global__ void k_scan_reduce(CountDev f, size_t n, uint64_t *bsum)
{
    size_t base = (size_t)blockIdx.x * kScanTile;
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        size_t i = base + (size_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += f(i);
    }
    __shared__ uint64_t tot;
    uint64_t t;
    (void)block_excl_scan_u64(s, &tot);
    __syncthreads();
    t = tot;
    if (threadIdx.x == 0) bsum[blockIdx.x] = t;
}

// Exclusive scan of nb block sums in place, one block of 1024 threads; bsum[nb] = total.
__global__ void k_scan_blocks(uint64_t *bsum, size_t nb)
{
    __shared__ uint64_t wsum[32];
    __shared__ uint64_t carry;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (size_t base = 0; base < nb; base += blockDim.x) {
        size_t i = base + threadIdx.x;
        uint64_t v = (i < nb) ? bsum[i] : 0;
        uint64_t inc = warp_incl_scan_u64(v);
        if (lane == 31) wsum[w] = inc;
        __syncthreads();
        if (w == 0) {
            uint64_t s = wsum[lane];
            uint64_t si = warp_incl_scan_u64(s);
            wsum[lane] = si - s;
        }
        __syncthreads();
        uint64_t ex = inc - v + wsum[w] + carry;
        __syncthreads();
        if (i < nb) bsum[i] = ex;
        if (threadIdx.x == blockDim.x - 1) carry = ex + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) bsum[nb] = carry;
}

__global__ void k_scan_down(CountDev f, size_t n, const uint64_t *bsum, uint64_t *out)
{
    size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint64_t v[kScanItems];
    uint64_t s = 0;
    // blocked arrangement: thread t owns items base + 0..7 (contiguous)
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        size_t i = base + k;
        v[k] = (i < n) ? f(i) : 0;
        s += v[k];
    }
    __shared__ uint64_t tot;
    uint64_t ex = block_excl_scan_u64(s, &tot) + bsum[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        size_t i = base + k;
        if (i < n) out[i] = ex;
        ex += v[k];
    }
}

__global__ void k_write_total(const uint64_t *bsum, size_t nb, uint64_t *out, size_t n)
{
    out[n] = bsum[nb];
}

static gs_status scan_impl(const CountDev &f, size_t n, uint64_t *out, uint64_t *total,
                           cudaStream_t s)
{
    size_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 0) nb = 1;
    uint64_t *bsum = nullptr;
    GS_CUDA(cudaMallocAsync(&bsum, (nb + 1) * sizeof(uint64_t), s));
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(f, n, bsum);
    k_scan_blocks<<<1, 1024, 0, s>>>(bsum, nb);
    k_scan_down<<<(unsigned)nb, kScanThreads, 0, s>>>(f, n, bsum, out);
    k_write_total<<<1, 1, 0, s>>>(bsum, nb, out, n);
    cudaError_t le = cudaGetLastError();
    cudaFreeAsync(bsum, s);
    if (le != cudaSuccess)
        return fail(GS_ERR_CUDA, "scan launch failed: %s", cudaGetErrorString(le));
    if (total) {
        GS_CUDA(cudaMemcpyAsync(total, out + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        GS_CUDA(cudaStreamSynchronize(s));
    }
    return GS_OK;
}

gs_status exclusive_scan(const CountSpec &spec, size_t n, uint64_t *out, uint64_t *total,
                         cudaStream_t s)
{
    CountDev f{(int)spec.kind, spec.row, spec.arr, spec.a};
    return scan_impl(f, n, out, total, s);
}

// ------------------------------------------------------------------ stable radix sort
__global__ void k_sort_init(const uint32_t *key, uint32_t n, uint32_t max_key, uint32_t *k,
                            uint32_t *idx)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        k[i] = max_key - key[i];  // ascending in k == descending in key
        idx[i] = i;
    }
}

__global__ void k_sort_scatter(const uint32_t *kin, const uint32_t *iin, uint32_t n,
                               uint32_t bit, const uint64_t *zpre, uint32_t *kout,
                               uint32_t *iout)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        uint64_t z = zpre[i], Z = zpre[n];
        uint32_t kv = kin[i];
        uint64_t d = (((kv >> bit) & 1u) == 0u) ? z : Z + ((uint64_t)i - z);
        kout[d] = kv;
        iout[d] = iin[i];
    }
}

gs_status stable_sort_desc(const uint32_t *key, uint32_t n, uint32_t max_key,
                           uint32_t *idx_out, cudaStream_t s)
{
    if (n == 0) return GS_OK;
    int bits = 0;
    while (bits < 32 && (max_key >> bits) != 0) bits++;
    DevBuf ka, kb, ib, z;
    GS_TRY(ka.alloc((size_t)n * 4));
    GS_TRY(kb.alloc((size_t)n * 4));
    GS_TRY(ib.alloc((size_t)n * 4));
    GS_TRY(z.alloc(((size_t)n + 1) * 8));
    uint32_t *kin = ka.as<uint32_t>(), *kout = kb.as<uint32_t>();
    uint32_t *iin = idx_out, *iout = ib.as<uint32_t>();
    unsigned g = (n + 255) / 256;
    k_sort_init<<<g, 256, 0, s>>>(key, n, max_key, kin, iin);
    GS_CHECK_LAUNCH();
    for (int b = 0; b < bits; b++) {
        CountDev f{4, nullptr, kin, (uint32_t)b};
        GS_TRY(scan_impl(f, n, z.as<uint64_t>(), nullptr, s));
        k_sort_scatter<<<g, 256, 0, s>>>(kin, iin, n, (uint32_t)b, z.as<uint64_t>(), kout,
                                         iout);
        GS_CHECK_LAUNCH();
        uint32_t *t = kin; kin = kout; kout = t;
        t = iin; iin = iout; iout = t;
    }
    if (iin != idx_out)
        GS_CUDA(cudaMemcpyAsync(idx_out, iin, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    GS_CUDA(cudaStreamSynchronize(s));  // scratch buffers are freed on return
    return GS_OK;
}

// ------------------------------------------------------------------ max reduce
__global__ void k_max_u32(const uint32_t *d, size_t n, uint32_t *out)
{
    uint32_t m = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        m = max(m, d[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

gs_status reduce_max_u32(const uint32_t *d, size_t n, uint32_t *out, cudaStream_t s)
{
    uint32_t *dm = nullptr;
    GS_CUDA(cudaMallocAsync(&dm, sizeof(uint32_t), s));
    GS_CUDA(cudaMemsetAsync(dm, 0, sizeof(uint32_t), s));
    if (n) k_max_u32<<<296, 256, 0, s>>>(d, n, dm);
    cudaError_t le = cudaGetLastError();
    cudaError_t ce = cudaMemcpyAsync(out, dm, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(dm, s);
    if (le != cudaSuccess || ce != cudaSuccess)
        return fail(GS_ERR_CUDA, "max reduce failed: %s",
                    cudaGetErrorString(le != cudaSuccess ? le : ce));
    GS_CUDA(cudaStreamSynchronize(s));
    return GS_OK;
}

}  // namespace gs
