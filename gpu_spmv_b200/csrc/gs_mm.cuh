// gs_mm.cuh -- device code shared by the multi-RHS K1 kernels (gs_spmm.cu, gs_batch.cu):
// arithmetic in the reference's order (separate multiply and add), 16/32-byte row access of
// row-major [*][ld] operands, and the work of one K1 unit (one kK1Split-step piece of a 32-row
// chunk) for a block of K right-hand sides.
#pragma once

#include "gs_internal.cuh"

namespace gs {
namespace mm {

constexpr uint32_t kNoSrc = 0xffffffffu;

template <class T> struct Arith;
template <> struct Arith<double> {
    __device__ __forceinline__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ __forceinline__ static double add(double a, double b) { return __dadd_rn(a, b); }
};
template <> struct Arith<float> {
    __device__ __forceinline__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ __forceinline__ static float add(float a, float b) { return __fadd_rn(a, b); }
};

// 32-byte loads / stores (one request for a 32-byte row; sm_100 256-bit vector access)
__device__ __forceinline__ void ld32(const float *p, float *v)
{
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]),
                   "=f"(v[6]), "=f"(v[7])
                 : "l"(p));
}
__device__ __forceinline__ void ld32(const double *p, double *v)
{
    asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
                 : "l"(p));
}
__device__ __forceinline__ void st32(float *p, const float *v)
{
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(v[0]),
                 "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
                 : "memory");
}
__device__ __forceinline__ void st32(double *p, const double *v)
{
    asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]),
                 "d"(v[2]), "d"(v[3])
                 : "memory");
}

// K consecutive values of row r of a row-major array with row stride ld: 32-byte accesses
// for K values of 32 bytes or more, 16-byte ones for 16 bytes (row starts aligned to that)
template <class T, int K>
__device__ __forceinline__ void load_row(const T *__restrict__ X, uint32_t r, uint32_t ld,
                                         T (&v)[K])
{
    const T *p = X + (size_t)r * ld;
    if constexpr (sizeof(T) * K >= 32) {
        constexpr int per = 32 / (int)sizeof(T);
#pragma unroll
        for (int i = 0; i < K / per; i++) ld32(p + i * per, v + i * per);
    } else if constexpr (sizeof(T) * K >= 16) {
        constexpr int per = 16 / (int)sizeof(T);
#pragma unroll
        for (int i = 0; i < K / per; i++) {
            if constexpr (sizeof(T) == 8) {
                const double2 w = __ldg(reinterpret_cast<const double2 *>(p) + i);
                v[2 * i] = w.x;
                v[2 * i + 1] = w.y;
            } else {
                const float4 w = __ldg(reinterpret_cast<const float4 *>(p) + i);
                v[4 * i] = w.x;
                v[4 * i + 1] = w.y;
                v[4 * i + 2] = w.z;
                v[4 * i + 3] = w.w;
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; k++) v[k] = __ldg(p + k);
    }
}

template <class T, int K>
__device__ __forceinline__ void store_row(T *__restrict__ Y, uint32_t r, uint32_t ld,
                                          const T (&v)[K])
{
    T *p = Y + (size_t)r * ld;
    if constexpr (sizeof(T) * K >= 32) {
        constexpr int per = 32 / (int)sizeof(T);
#pragma unroll
        for (int i = 0; i < K / per; i++) st32(p + i * per, v + i * per);
    } else if constexpr (sizeof(T) * K >= 16) {
        constexpr int per = 16 / (int)sizeof(T);
#pragma unroll
        for (int i = 0; i < K / per; i++) {
            if constexpr (sizeof(T) == 8)
                reinterpret_cast<double2 *>(p)[i] = make_double2(v[2 * i], v[2 * i + 1]);
            else
                reinterpret_cast<float4 *>(p)[i] =
                    make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; k++) p[k] = v[k];
    }
}

// slots in flight per lane: at most 8, and at most 128 bytes of gathered rows (more
// registers would cost occupancy, which the latency-bound gathers need more)
template <class T, int K, int BYTES = 128> constexpr int mm_batch()
{
    return (BYTES / (K * (int)sizeof(T))) < 1 ? 1
           : ((BYTES / (K * (int)sizeof(T))) > 8 ? 8 : BYTES / (K * (int)sizeof(T)));
}

struct MMArgs {
    uint32_t nrows;                            // rows of this layout (A: n, A^T: ncols)
    const uint32_t *permi, *nmc, *chp, *klen;  // K1 layout
    const void *val;
    const uint32_t *col;                       // gathered row index (A: col, A^T: row of A)
    const void *xin;                           // gathered operand (A: X, A^T: Ybar)
    const void *xrow;                          // A^T only: X, row j held for vbar
    void *yout;                                // A: Y, A^T: Xbar
    void *vbar;                                // A^T only, or nullptr: vbar in this
                                               // layout's slot order, padding slots zero
    const uint32_t *unit_chunk, *unit_base;
    uint32_t units, split_units;               // units < split_units may be pieces
    void *partial;                             // split_units * ld * 32 values
    uint32_t *count;                           // chunks * nrb arrival counters
    uint32_t ld;                               // row stride of X, Y (= K for one block)
    uint32_t nrb;                              // right-hand-side blocks per unit
};

// Unit u of the layout, right-hand-side block rb (columns rb*K .. rb*K+K-1 of X, Y), by
// one warp.  Split chunks: each piece leaves its partial sums in scratch; the piece that
// arrives last adds them in piece order and writes Y.
template <class T, int K, bool ADJ>
__device__ __forceinline__ void mm_unit(const MMArgs &a, uint32_t u, uint32_t rb)
{
    using A = Arith<T>;
    // the adjoint also holds X's row and the slot indices: half the gathered bytes in flight
    constexpr int B = mm_batch<T, K, ADJ ? 64 : 128>();
    const uint32_t off = rb * K;
    const T *__restrict__ val = static_cast<const T *>(a.val);
    const T *__restrict__ xin = static_cast<const T *>(a.xin) + off;
    T *__restrict__ yout = static_cast<T *>(a.yout) + off;
    T *__restrict__ partial = static_cast<T *>(a.partial);
    const int lane = threadIdx.x & 31;
    const uint32_t ld = a.ld;
    {
        const uint32_t c = __ldg(a.unit_chunk + u);
        const uint32_t ub = __ldg(a.unit_base + c);
        const uint32_t np = __ldg(a.unit_base + c + 1) - ub;
        const uint32_t piece = u - ub;
        const uint32_t g = 32u * c + (uint32_t)lane;
        const bool valid = g < a.nrows;
        const uint32_t len = valid ? __ldg(a.klen + g) : 0u;
        const uint32_t j0 = piece * kK1Split;
        const uint32_t j1 = min(len, j0 + kK1Split);
        const uint32_t base = __ldg(a.chp + c) + (uint32_t)lane;
        const uint32_t me = valid ? __ldg(a.permi + g) : 0u;
        T xr[K];
        if constexpr (ADJ) {
            if (a.vbar && j0 < j1) load_row<T, K>(static_cast<const T *>(a.xrow) + off, me, ld, xr);
        }
        T acc[K];
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = T(0);
        for (uint32_t j = j0; j < j1; j += B) {
            T v[B], gv[B][K];
            uint32_t cc[B];
#pragma unroll
            for (int b = 0; b < B; b++) {
                const bool in = j + b < j1;
                const uint32_t pos = base + 32u * (j + b);
                v[b] = in ? __ldcs(val + pos) : T(0);
                cc[b] = in ? __ldcs(a.col + pos) : 0u;
            }
#pragma unroll
            for (int b = 0; b < B; b++) {
                if (j + b < j1) load_row<T, K>(xin, cc[b], ld, gv[b]);
                else {
#pragma unroll
                    for (int k = 0; k < K; k++) gv[b][k] = T(0);
                }
            }
#pragma unroll
            for (int b = 0; b < B; b++) {
                if (j + b < j1) {
#pragma unroll
                    for (int k = 0; k < K; k++) acc[k] = A::add(acc[k], A::mul(v[b], gv[b][k]));
                }
            }
            if constexpr (ADJ) {
                if (a.vbar) {
#pragma unroll
                    for (int b = 0; b < B; b++) {
                        if (j + b < j1) {
                            T d = T(0);
#pragma unroll
                            for (int k = 0; k < K; k++) d = A::add(d, A::mul(gv[b][k], xr[k]));
                            static_cast<T *>(a.vbar)[base + 32u * (j + b)] = d;
                        }
                    }
                }
            }
        }
        if constexpr (ADJ) {
            // slot order: this piece's padding slots of the lane get a zero gradient
            if (a.vbar) {
                const uint32_t pend = min(__ldg(a.nmc + c), j0 + kK1Split);
                for (uint32_t j = max(j0, len); j < pend; j++)
                    static_cast<T *>(a.vbar)[base + 32u * j] = T(0);
            }
        }
        if (np == 1) {
            if (valid) store_row<T, K>(yout, me, ld, acc);
            return;
        }
        // split chunk: the pieces of chunk c are units ub .. ub+np-1 < split_units
#pragma unroll
        for (int k = 0; k < K; k++) partial[((size_t)u * ld + off + k) * 32 + lane] = acc[k];
        __threadfence();
        __syncwarp();
        uint32_t ticket = 0;
        if (lane == 0) ticket = atomicAdd(a.count + (size_t)c * a.nrb + rb, 1u);
        ticket = __shfl_sync(0xffffffffu, ticket, 0);
        if (ticket == np - 1) {
            __threadfence();
            T s[K];
#pragma unroll
            for (int k = 0; k < K; k++) s[k] = T(0);
            for (uint32_t q = 0; q < np; q++) {
#pragma unroll
                for (int k = 0; k < K; k++)
                    s[k] = A::add(s[k],
                                  __ldcg(partial + ((size_t)(ub + q) * ld + off + k) * 32 + lane));
            }
            if (valid) store_row<T, K>(yout, me, ld, s);
            if (lane == 0) a.count[(size_t)c * a.nrb + rb] = 0;
        }
    }
}


}  // namespace mm
}  // namespace gs
