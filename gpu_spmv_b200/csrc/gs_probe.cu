// gs_probe.cu -- gs_gather_rate: the rate of independent random 8-byte reads from a vector,
// the ceiling of an SpMV whose x gathers fall on random lines (each read is one line request
// through the SM's load path; see the bench's roofline).  No counterpart in the reference.
#include "gs_internal.cuh"

namespace gs {
namespace {

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

}  // namespace
}  // namespace gs

extern "C" gs_status gs_gather_rate(const double *d_x, UIN n, UIN per_thread,
                                    double *reads_per_s, gs_stream stream)
{
    if (!d_x || !reads_per_s || n == 0) return gs::fail(GS_ERR_INVALID, "NULL argument or n = 0");
    if (per_thread == 0 || per_thread % 8) return gs::fail(GS_ERR_INVALID, "per_thread must be a positive multiple of 8");
    cudaStream_t s = gs::cs(stream);
    int dev = 0, sms = 148;
    GS_CUDA(cudaGetDevice(&dev));
    GS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned blocks = (unsigned)sms * 8u;  // 8 blocks of 256 per SM: every SM busy
    gs::DevBuf sink;
    GS_TRY(sink.alloc(8));
    cudaEvent_t a, b;
    GS_CUDA(cudaEventCreate(&a));
    GS_CUDA(cudaEventCreate(&b));
    gs::k_gather_rate<<<blocks, 256, 0, s>>>(d_x, n, per_thread, sink.as<double>());
    cudaEventRecord(a, s);
    gs::k_gather_rate<<<blocks, 256, 0, s>>>(d_x, n, per_thread, sink.as<double>());
    cudaEventRecord(b, s);
    const cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return gs::fail(GS_ERR_CUDA, "gather probe: %s", cudaGetErrorString(e));
    GS_CHECK_LAUNCH();
    *reads_per_s = (double)blocks * 256.0 * (double)per_thread / ((double)ms * 1e-3);
    return GS_OK;
}
