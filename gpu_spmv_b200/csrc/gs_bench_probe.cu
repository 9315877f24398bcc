// gs_bench_probe.cu -- measurement helpers of the benchmark (libgs_bench_probe.so, built
// beside the engine library and loaded only by bench.py; not part of the engine's C ABI).
// No counterpart in the reference.
//
//   gsp_gather_rate   rate of independent random 8-byte reads from a vector through the SM's
//                     load path (ld.global.nc): each read of a uniformly random column is its
//                     own 128-byte line request, which bounds an SpMV whose x gathers are
//                     random (the roofline's gather ceiling).
//   gsp_gather4_rate  the same random reads issued as TMA tile gathers
//                     (cp.async.bulk.tensor.2d ... tile::gather4): x viewed as rows of two
//                     doubles (16 bytes), one instruction brings four such rows into shared
//                     memory and completes on an mbarrier.  Optionally some warps of every
//                     block issue load-path gathers at the same time, to see whether the two
//                     paths add up.  The tensor map covers only this GPU's x, no multicast.
//
// Every mbarrier wait is bounded in wall time; a wait that gives up sets *status and the
// kernel waits (bounded again) for the copies it issued before it returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "gs_bulk.cuh"

namespace {

char g_err[256];

int fail(const char *what, cudaError_t e)
{
    snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
    return 2;
}

__device__ __forceinline__ uint32_t mix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// per_thread reads per thread, 8 independent reads in flight, indices hash(..) % n
__global__ void __launch_bounds__(256) k_gather_rate(const double *__restrict__ x, uint32_t n,
                                                     uint32_t per_thread, double *sink)
{
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s = mix32(tid * 2654435761u + 17u);
    double acc = 0.0;
    for (uint32_t k = 0; k < per_thread; k += 8) {
        double v[8];
#pragma unroll
        for (int b = 0; b < 8; b++) {
            s = mix32(s + (uint32_t)b);
            v[b] = __ldg(x + s % n);
        }
#pragma unroll
        for (int b = 0; b < 8; b++) acc += v[b];
    }
    if (acc == 1.2345678e300) sink[0] = acc;  // never true for finite x: keeps the reads
}

constexpr int kG4Stages = 4;            // stages per warp
constexpr uint32_t kG4Bytes = 64u;       // one gather4: 4 rows x 16 bytes
constexpr uint32_t kG4Slot = 128u;       // a tensor copy's shared-memory destination is
                                         // 128-byte aligned: one slot per lane
constexpr uint32_t kG4StageBytes = 32u * kG4Slot;

__device__ __forceinline__ void gather4(void *dst, const CUtensorMap *tm, int32_t c, int32_t r0,
                                        int32_t r1, int32_t r2, int32_t r3, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        ::"r"(gs::bulk::smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(tm)), "r"(c), "r"(r0),
          "r"(r1), "r"(r2), "r"(r3), "r"(gs::bulk::smem_addr(bar))
        : "memory");
}

// Warps [0, lsu_warps) of each block gather through the load path (8 reads in flight per
// lane, per_lane reads per lane); the others issue per_lane / 4 gather4 instructions per lane
// (each four 16-byte rows), kG4Stages stages of 32 instructions in flight per warp.
__global__ void __launch_bounds__(256) k_gather4_rate(const __grid_constant__ CUtensorMap tm,
                                                      const double *__restrict__ x,
                                                      uint32_t nrow2, uint32_t per_lane,
                                                      uint32_t lsu_warps, double *sink,
                                                      uint32_t *status)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t nw = blockDim.x >> 5;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s = mix32(tid * 2654435761u + 17u);
    double acc = 0.0;
    if ((uint32_t)wid < lsu_warps) {
        const uint32_t n = 2u * nrow2;
        for (uint32_t k = 0; k < per_lane; k += 8) {
            double v[8];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                s = mix32(s + (uint32_t)b);
                v[b] = __ldg(x + s % n);
            }
#pragma unroll
            for (int b = 0; b < 8; b++) acc += v[b];
        }
    } else {
        const uint32_t tw = (uint32_t)wid - lsu_warps;  // index among the gather4 warps
        unsigned char *buf = smem + (size_t)tw * kG4Stages * kG4StageBytes;
        uint64_t *bars = reinterpret_cast<uint64_t *>(
                             smem + (size_t)(nw - lsu_warps) * kG4Stages * kG4StageBytes) +
                         tw * kG4Stages;
        if (lane == 0)
            for (int i = 0; i < kG4Stages; i++) gs::bulk::mbar_init(bars + i, 1);
        gs::bulk::fence_mbar_init();
        gs::bulk::fence_proxy_async();
        __syncwarp();
        const uint32_t iters = per_lane / 4u;
        bool ok = true;
        uint32_t issued = 0;
        for (uint32_t it = 0; it < iters && ok; it++) {
            const int st = (int)(it % kG4Stages);
            if (it >= (uint32_t)kG4Stages) {
                ok = gs::bulk::mbar_wait_bounded(bars + st, ((it / kG4Stages) - 1u) & 1u);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
                acc += *reinterpret_cast<const double *>(buf + st * kG4StageBytes + lane * kG4Slot);
            }
            unsigned char *dst = buf + st * kG4StageBytes + lane * kG4Slot;
            // a misaligned destination is recorded and the stage skipped, never issued
            if (!__all_sync(0xffffffffu, (gs::bulk::smem_addr(dst) & 127u) == 0u)) {
                if (lane == 0) atomicOr(status, 2u);
                break;
            }
            __syncwarp();
            if (lane == 0) gs::bulk::mbar_expect_tx(bars + st, 32u * kG4Bytes);
            __syncwarp();
            int32_t r[4];
#pragma unroll
            for (int b = 0; b < 4; b++) {
                s = mix32(s + (uint32_t)b);
                r[b] = (int32_t)(s % nrow2);
            }
            gather4(dst, &tm, 0, r[0], r[1], r[2], r[3], bars + st);
            issued = it + 1;
        }
        // drain: every stage still in flight (bounded; a second limit after a timeout)
        const uint32_t first = issued > (uint32_t)kG4Stages ? issued - kG4Stages : 0u;
        for (uint32_t it = first; it < issued; it++) {
            const int st = (int)(it % kG4Stages);
            if (!gs::bulk::mbar_wait_bounded(bars + st, (it / kG4Stages) & 1u)) ok = false;
            else acc += *reinterpret_cast<const double *>(buf + st * kG4StageBytes + lane * kG4Slot);
        }
        if (!ok && lane == 0) atomicOr(status, 1u);
    }
    if (acc == 1.2345678e300) sink[0] = acc;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

}  // namespace

extern "C" {

const char *gsp_last_error(void) { return g_err; }

// Random 8-byte reads per second from d_x[0..n) through the load path; 0 on success.
int gsp_gather_rate(const double *d_x, uint32_t n, uint32_t per_thread, double *reads_per_s,
                    void *stream)
{
    if (!d_x || !reads_per_s || n == 0 || per_thread == 0 || per_thread % 8) {
        snprintf(g_err, sizeof(g_err), "invalid argument");
        return 1;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 148;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail("device query", e);
    const unsigned blocks = (unsigned)sms * 8u;  // 8 blocks of 256 per SM: every SM busy
    double *sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    if ((e = cudaMalloc(&sink, 64)) != cudaSuccess) return fail("cudaMalloc", e);
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_gather_rate<<<blocks, 256, 0, s>>>(d_x, n, per_thread, sink);
    cudaEventRecord(a, s);
    k_gather_rate<<<blocks, 256, 0, s>>>(d_x, n, per_thread, sink);
    cudaEventRecord(b, s);
    e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return fail("gather probe", e);
    *reads_per_s = (double)blocks * 256.0 * (double)per_thread / ((double)ms * 1e-3);
    return 0;
}

// Random 8-byte reads per second from d_x[0..n) (n even, d_x 16-byte aligned) when
// `warps - lsu_warps` warps of each block issue TMA gather4 loads and `lsu_warps` warps
// load-path gathers, `blocks_per_sm` blocks of `warps` warps on every SM.  Each lane makes
// per_lane reads (a multiple of 8).  *timed_out is set when a bounded wait gave up.
int gsp_gather4_rate(const double *d_x, uint32_t n, uint32_t per_lane, uint32_t warps,
                     uint32_t lsu_warps, uint32_t blocks_per_sm, double *reads_per_s,
                     uint32_t *timed_out, void *stream)
{
    if (!d_x || !reads_per_s || !timed_out || n < 8 || (n & 1u) || per_lane == 0 ||
        per_lane % 8 || warps == 0 || warps > 8 || lsu_warps > warps || blocks_per_sm == 0 ||
        (reinterpret_cast<uintptr_t>(d_x) & 15u)) {
        snprintf(g_err, sizeof(g_err), "invalid argument");
        return 1;
    }
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (!enc) {
        snprintf(g_err, sizeof(g_err), "cuTensorMapEncodeTiled unavailable");
        return 2;
    }
    // x as a [n/2][2] FP64 tensor: rows of 16 bytes, a box of one row (gather4 takes four)
    CUtensorMap tm;
    const cuuint64_t dims[2] = {2, n / 2};
    const cuuint64_t strides[1] = {16};
    const cuuint32_t box[2] = {2, 1};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(d_x), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(g_err, sizeof(g_err), "cuTensorMapEncodeTiled failed (%d)", (int)r);
        return 2;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 148;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail("device query", e);
    const size_t tw = warps - lsu_warps;
    const size_t smem = tw * kG4Stages * kG4StageBytes + tw * kG4Stages * 8 + 8;
    e = cudaFuncSetAttribute(k_gather4_rate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fail("cudaFuncSetAttribute", e);
    const unsigned blocks = (unsigned)sms * blocks_per_sm;
    double *sink = nullptr;
    uint32_t *st = nullptr;
    if ((e = cudaMalloc(&sink, 64)) != cudaSuccess) return fail("cudaMalloc", e);
    if ((e = cudaMalloc(&st, 4)) != cudaSuccess) {
        cudaFree(sink);
        return fail("cudaMalloc", e);
    }
    cudaMemsetAsync(st, 0, 4, s);
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_gather4_rate<<<blocks, warps * 32, smem, s>>>(tm, d_x, n / 2, per_lane, lsu_warps, sink, st);
    cudaEventRecord(a, s);
    k_gather4_rate<<<blocks, warps * 32, smem, s>>>(tm, d_x, n / 2, per_lane, lsu_warps, sink, st);
    cudaEventRecord(b, s);
    e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    if (e == cudaSuccess) e = cudaGetLastError();
    uint32_t hst = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&hst, st, 4, cudaMemcpyDeviceToHost);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    cudaFree(st);
    if (e != cudaSuccess) return fail("gather4 probe", e);
    *timed_out = hst;
    *reads_per_s = (double)blocks * warps * 32.0 * (double)per_lane / ((double)ms * 1e-3);
    return 0;
}

}  // extern "C"
