// gs_internal.cuh -- internal declarations shared by the engine's translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstddef>
#include <type_traits>

#include "gpuspmv_b200.h"

namespace gs {

// ------------------------------------------------------------------ errors
// Records a formatted message for gs_last_error() on the calling thread and returns st.
gs_status fail(gs_status st, const char *fmt, ...);
void clear_error();

#define GS_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return ::gs::fail(GS_ERR_CUDA, "%s:%d: %s failed: %s", __FILE__, __LINE__,  \
                              #call, cudaGetErrorString(e_));                            \
    } while (0)

#define GS_TRY(call)                                                                     \
    do {                                                                                 \
        gs_status s_ = (call);                                                           \
        if (s_ != GS_OK) return s_;                                                      \
    } while (0)

#define GS_CHECK_LAUNCH() GS_CUDA(cudaGetLastError())

inline cudaStream_t cs(gs_stream s) { return reinterpret_cast<cudaStream_t>(s); }

inline size_t dtype_size(gs_dtype t) { return t == GS_F64 ? 8 : (t == GS_F32 ? 4 : 2); }

// ------------------------------------------------------------------ device buffers
// Owning device allocation (cudaMalloc / cudaFree).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) { reset(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { reset(); }
    void reset() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
    gs_status alloc(size_t nbytes);                       // rounds up, keeps 16 B of tail slack
    gs_status alloc_zero(size_t nbytes, cudaStream_t s);  // alloc + async memset 0
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// ------------------------------------------------------------------ scan primitives
// Exclusive prefix sum of n 32-bit counts produced by `count(i)`, written as 64-bit
// offsets out[0..n] (out[n] = total).  Implemented in gs_scan.cu for the functors listed
// there; `total` receives out[n] on the host (synchronises the stream).
enum class CountKind {
    RowLen,         // row[i+1]-row[i]
    RowTiles,       // ceil((row[i+1]-row[i]) / a)
    Array,          // arr[i]
    ArrayTimes,     // arr[i] * a
    BitZero,        // (arr[i] >> a) & 1 == 0   (radix sort pass)
    PiecesMin1,     // max(1, ceil(arr[i] / a))
    WindowPopc,     // popcount of the a words arr[i*a .. i*a+a)
    NonEmpty,       // row[i+1] > row[i]
};
struct CountSpec {
    CountKind kind;
    const uint32_t *row = nullptr;  // RowLen / RowTiles
    const uint32_t *arr = nullptr;  // Array / ArrayTimes
    uint32_t a = 1;
};
gs_status exclusive_scan(const CountSpec &spec, size_t n, uint64_t *out, uint64_t *total,
                         cudaStream_t s);

// Stable sort of row indices 0..n-1 by descending key (keys < 2^bits): idx_out[i] is the
// i-th row.  Ties keep ascending row order.  1-bit LSD radix passes built on the scan.
gs_status stable_sort_desc(const uint32_t *key, uint32_t n, uint32_t max_key,
                           uint32_t *idx_out, cudaStream_t s);

// Maximum of n u32 values (host result, synchronises).
gs_status reduce_max_u32(const uint32_t *d, size_t n, uint32_t *out, cudaStream_t s);

// ------------------------------------------------------------------ device helpers
__device__ __forceinline__ double ldcs_f64(const double *p) { return __ldcs(p); }
__device__ __forceinline__ uint32_t ldcs_u32(const uint32_t *p) { return __ldcs(p); }

template <class T> struct ValTraits;
template <> struct ValTraits<double> {
    __device__ __forceinline__ static double to_f64(double v) { return v; }
    __device__ __forceinline__ static float to_f32(double v) { return (float)v; }
};
template <> struct ValTraits<float> {
    __device__ __forceinline__ static double to_f64(float v) { return (double)v; }
    __device__ __forceinline__ static float to_f32(float v) { return v; }
};
template <> struct ValTraits<__nv_bfloat16> {
    __device__ __forceinline__ static double to_f64(__nv_bfloat16 v) {
        return (double)__bfloat162float(v);
    }
    __device__ __forceinline__ static float to_f32(__nv_bfloat16 v) { return __bfloat162float(v); }
};

}  // namespace gs

namespace gs {
// Execution plan of the row-stream kernel (gs_spmv_rows.cu), built once per matrix:
//  sbits  : bit p set <=> position p is the first position of a non-empty row
//  rbits  : bit p set <=> position p holds a real element (padded layouts only)
//  wcount : number of set start bits before each window of 32*V positions
//  ne     : rank -> row index of the non-empty rows (only when some rows are empty)
//  empty  : the empty rows (their y entries are written 0)
//  colbase: per-window base of the 16-bit column offsets (GS_IDX_U16 only)
//  status : device status word (bit 0: a bounded wait in a kernel timed out)
//  aligned: every row starts on a multiple of V positions (UNC / AXC layouts)
struct RowsPlan {
    uint32_t npos = 0, nwin = 0, V = 8, wpw = 4, n_empty = 0;
    bool padded = false, aligned = false, grouped = false;
    DevBuf sbits, rbits, wcount, ne, empty, colbase, status;
};
}  // namespace gs

// Streams, events and double buffers of the host-streaming product (gs_spmv_host_stream),
// made on its first call.
struct HostPipe {
    cudaStream_t in = nullptr, out = nullptr;
    cudaEvent_t xready[2] = {}, kdone[2] = {}, ydone[2] = {};
    gs::DevBuf x[2], y[2];
    bool ready = false;
    ~HostPipe()
    {
        for (int b = 0; b < 2; b++) {
            if (xready[b]) cudaEventDestroy(xready[b]);
            if (kdone[b]) cudaEventDestroy(kdone[b]);
            if (ydone[b]) cudaEventDestroy(ydone[b]);
        }
        if (in) cudaStreamDestroy(in);
        if (out) cudaStreamDestroy(out);
    }
};

// ------------------------------------------------------------------ the matrix handle
struct gs_matrix {
    HostPipe pipe;
    gs_convert_params p{};
    uint32_t nrows = 0, ncols = 0, nnz = 0;
    // reference-layout dimensions
    uint32_t tileHW = 0, tileH = 0, logTH = 0, tileN = 0, lenAX = 0, lenSEC = 0, lenCON = 0,
             log = 0, bs = 0;
    uint32_t hbs = 0, lenBRP = 0, lenMAPX = 0;
    uint32_t chunkNum = 0, lenVC = 0;
    // native streams
    uint32_t nslots = 0;
    gs::DevBuf val, col, colbase;
    gs::DevBuf sec, con, brp, mapx;
    gs::DevBuf permi, nmc, chp;
    gs::DevBuf rpos, rlen;  // row table for the row-stream kernels
    // K1 execution plan (split of long chunks) and its scratch
    gs::DevBuf k1len, k1unit_chunk, k1unit_base, k1partial, k1count, k1ck;
    // multi-RHS products (gs_spmm) and the adjoint (gs_matrix_prepare_adjoint)
    gs::DevBuf mmpartial;  // split pieces x 32 lanes x up to 32 RHS (FP64 sized)
    uint32_t k1split_units = 0;
    bool mm_ready = false, adj_ready = false;
    gs::DevBuf fsrc;    // forward slot -> CSR index
    gs::DevBuf ftslot;  // forward slot -> adjoint-layout slot
    gs::DevBuf csr2t;   // CSR index -> adjoint-layout slot
    gs::DevBuf csr2f;   // CSR index -> forward slot
    gs::DevBuf t2f;     // adjoint-layout slot -> forward slot (padding: none)
    gs::DevBuf vslots;  // vbar in slot order before it is gathered into CSR order
    gs::DevBuf tpermi, tnmc, tchp, tlen, trow, tsrc, tval;  // K1 layout of A^T
    gs::DevBuf tunit_chunk, tunit_base, tpartial1, tcount, tpartial;
    uint32_t tchunkNum = 0, tlenVC = 0, tunits = 0, tsplit_units = 0;
    uint32_t k1units = 0;
    // row-stream kernel configuration
    uint32_t tiled = 0;  // 1: positions map to tile slots (tileH > 1 layouts)
    gs::RowsPlan plan;
    // FP64 layouts of whole tiles per row (UNC tileH = 1, AXC) of width 4..32: the same rows
    // planned over tiles, for the tile kernel (launch_tiles); tile_w 0 otherwise
    gs::RowsPlan tplan;
    uint32_t tile_w = 0;
    double conv_ms = 0, mfp = 0, beta = 0;
};

namespace gs {

// Row-stream SpMV (see gs_spmv_rows.cu).
struct RowsArgs {
    uint32_t npos, nwin, wpw, V;   // positions, windows of 32*V positions, windows per warp
    uint32_t thw, th;              // tile shape of tiled (tileH > 1) layouts
    uint32_t axw;                  // baked layouts: ax half width (tileHW or hbs)
    uint32_t nslots;               // length of the value/column streams
    uint32_t n_empty;
    uint32_t aligned;              // rows start on multiples of V (aligned kernel applies)
    uint32_t wide;                 // val and col 32-byte aligned: 32-byte stream loads
    uint32_t grouped;              // x gathers close to random: owned tiles go two at a time
    const uint32_t *sbits, *rbits, *wcount, *ne, *empty, *colbase;
    uint32_t *status;  // device status word (bounded-wait timeouts)
    const void *val;   // value stream (or the baked ax)
    const void *col;  // column stream (u32, or u16 offsets from colbase)
    const void *x;
    void *y;
};
// Positions per lane of the direct (tileH = 1) layouts.
constexpr uint32_t kDirectV = 8;
// Positions per lane of an FP64 direct layout with x gathered at run time (CSR, COM
// tileH = 1), from the CSR row pointers and columns: 4 when rows average fewer than 8
// elements or fewer than a quarter of a sample of in-row column steps stay within 16
// columns (the x gathers are random: 4 positions hold 40 registers, 6 blocks per SM, and a
// lane's 4 values and 4 columns are one 32-byte and one 16-byte request), else 8 (streams
// with local columns: more bytes in flight per warp).
gs_status direct_lane_positions(const uint32_t *d_row, const uint32_t *d_col, uint32_t n,
                                uint64_t nnz, uint32_t *V, cudaStream_t s);
// Whether the x gathers of a CSR matrix are close to random: fewer than a quarter of a
// sample of in-row column steps (up to 32 steps of 65,536 rows) stay within 16 columns.
gs_status random_columns(const uint32_t *d_row, const uint32_t *d_col, uint32_t n,
                         bool *random, cudaStream_t s);
// Positions per lane for a layout whose rows start on multiples of `align` positions
// (0: no alignment): returns the V that makes the aligned kernel apply, or kDirectV.
uint32_t aligned_lane_positions(uint32_t align, bool *aligned);
// Build the plan from a row table: rpos[0..n] first position of each row (rpos[n] = total
// positions), rlen[r] real length (nullptr when rows carry no padding).
gs_status build_rows_plan(const uint32_t *d_rpos, const uint32_t *d_rlen, uint32_t n,
                          uint32_t V, RowsPlan &P, cudaStream_t s, bool tiled = false);
// 16-bit column offsets: per-window base over real positions, col16 = col32 - base.
gs_status build_u16_columns(const uint32_t *d_col32, uint32_t nslots, RowsPlan &P,
                            uint16_t *d_col16, cudaStream_t s);
RowsArgs rows_args(const RowsPlan &P);
// FP64 layouts of whole tiles per row (UNC tileH = 1, AXC), thw in {4, 8, 16, 32}: baked
// (a.val = ax: [thw values | thw x] per tile) or with value / column streams (a.val, a.col,
// a.x; a.rbits the slot-level real bits of a padded layout, or null).  The plan is built over
// tiles (its positions are tiles, its row starts the first tile of each row; windows of 32 V
// tiles); y FP64.
gs_status launch_tiles(const RowsArgs &a, uint32_t thw, bool baked, cudaStream_t s);
gs_status launch_rows(const RowsArgs &a, gs_dtype vtype, gs_itype itype, gs_dtype ytype,
                      uint32_t flags, bool tiled, bool baked, bool padded, cudaStream_t s);

// Slot of step j of lane `lane` in the K1 chunk that starts at slot cbase and has nmc
// steps.  The reference's order is cbase + 32 j + lane (a warp's loads of one step are
// consecutive).  The 16-bit-step layouts use a lane-blocked order instead: steps below
// 8 floor(nmc / 8) in groups of 8, each lane's 8 slots of a group consecutive
// (cbase + 256 (j / 8) + 8 lane + j % 8), so that one 16-byte load brings a lane 8 steps;
// the remaining steps keep the reference's order after them.
__host__ __device__ __forceinline__ uint32_t k1_slot(uint32_t cbase, uint32_t nmc, uint32_t j,
                                                     uint32_t lane, bool blocked)
{
    if (blocked && j < (nmc & ~7u)) return cbase + (j >> 3) * 256u + lane * 8u + (j & 7u);
    return cbase + 32u * j + lane;
}

// K1 SpMV (see gs_spmv_k1.cu).
struct K1Args {
    uint32_t nrows, chunkNum;
    const uint32_t *permi, *nmc, *chp, *klen;  // klen: per sorted row length or nullptr
    const void *val;  // double / float / __nv_bfloat16
    const void *col;  // uint32_t columns, or uint16_t steps with checkpoints ck
    const uint32_t *ck;
    const void *x;    // double for FP64 values, float otherwise
    void *y;          // double or float
    const uint32_t *unit_chunk, *unit_base;  // plan
    uint32_t units;
    double *partial;
    uint32_t *count;
};
gs_status launch_k1(const K1Args &a, gs_dtype vtype, gs_itype itype, gs_dtype ytype, bool acc64,
                    cudaStream_t s);
// 16-bit column steps + per-unit checkpoints from 32-bit K1 columns (plan and klen needed).
gs_status build_k1_deltas(const K1Args &a, const uint32_t *d_col32, uint16_t *d_col16,
                          uint32_t *d_ck, cudaStream_t s);
// Build the K1 plan for chunk lengths nmc (device) into the given buffers.
constexpr uint32_t kK1Split = 128;  // j-steps per K1 work unit (a piece is a critical path of
                                     // kK1Split/8 dependent gather rounds: 128 keeps it short)
gs_status build_k1_plan(const uint32_t *d_nmc, uint32_t chunkNum, DevBuf &unit_chunk,
                        DevBuf &unit_base, DevBuf &partial, DevBuf &count, uint32_t *units,
                        cudaStream_t s);

// Sizes a K1 matrix's multi-RHS scratch once (gs_spmm.cu; allocates, synchronises).
gs_status prepare_mm_scratch(gs_matrix *A, cudaStream_t s);

// Conversion entry (gs_convert.cu).  x/ax optional: bake x into a reference-layout ax.
gs_status convert(gs_matrix *A, const gs_convert_params &p, uint32_t nrows, uint32_t ncols,
                  uint32_t nnz, const uint32_t *d_row, const uint32_t *d_col,
                  const void *d_val, gs_dtype val_type, const double *d_xbake,
                  DevBuf *ax_out, cudaStream_t s);

}  // namespace gs
