// gs_spmm.cu -- multi-RHS K1 products and the adjoint of y = A(v) x.
//
// Forward: Y = A X for k right-hand sides (X row-major [ncols][k], Y row-major [nrows][k],
// k in {1, 2, 4, 8, 16, 32}) on the K1 layout.  Each lane owns one sorted row, as in the
// single-RHS kernel (gs_spmv_k1.cu), and one gather of a column fetches all k values of
// X's row at once (32 bytes for k = 8 in FP32), so the gather cost is paid once per
// stored element for every right-hand side.  Long chunks are cut into the same kK1Split-step
// pieces, whose partial sums meet in scratch memory in piece order.
//
// Adjoint, for a loss L(Y) with Ybar = dL/dY:
//   Xbar = A^T Ybar                      (ncols x k)
//   vbar_e = sum_r Ybar[row_e][r] X[col_e][r]   for every stored element e (CSR order)
// Deterministic mode: the transpose is stored as its own K1 layout, built once by
// gs_matrix_prepare_adjoint (columns of A sorted by decreasing length, each transposed slot
// remembering the CSR index of its element and its row), and Xbar is the forward kernel run
// on it; the same pass gathers Ybar[row_e] for Xbar and forms vbar_e against X[col] held in
// registers, so vbar costs no extra gather.  Atomic mode: the forward layout, with Xbar
// accumulated by atomic adds (its rounding order varies between runs).
//
// The reference has no multi-RHS product and no adjoint; these extend its K1 format.
#include <mutex>

#include "gs_mm.cuh"

namespace gs {

namespace {

using namespace mm;

template <class T, int K, bool ADJ>
__global__ void __launch_bounds__(256) k_k1_mm(const MMArgs a)
{
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < a.units;
         u += warps)
        mm_unit<T, K, ADJ>(a, u, 0);
}

// Atomic-mode adjoint on the forward layout, over the same kK1Split-step work units: lane = row
// r of A with Ybar[r] in registers; per stored element e: Xbar[col_e] += v_e Ybar[r] (atomic
// adds; Xbar zeroed first) and, when vbar is wanted, vbar_e = Ybar[r] . X[col_e] (one more
// gather of X's row per element).
struct AtomicArgs {
    uint32_t nrows;
    const uint32_t *permi, *chp, *klen, *col, *unit_chunk, *unit_base;
    uint32_t units;
    const void *val, *x, *ybar;
    void *xbar, *vbar;  // vbar (or nullptr) in forward slot order
};

template <class T, int K>
__device__ __forceinline__ void red_row(T *__restrict__ X, uint32_t r, const T (&v)[K])
{
    T *p = X + (size_t)r * K;
    if constexpr (sizeof(T) == 4 && K % 4 == 0) {
#pragma unroll
        for (int i = 0; i < K / 4; i++)
            atomicAdd(reinterpret_cast<float4 *>(p) + i,
                      make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]));
    } else {
#pragma unroll
        for (int k = 0; k < K; k++) atomicAdd(p + k, v[k]);
    }
}

template <class T, int K>
__global__ void __launch_bounds__(256) k_k1_adj_atomic(const AtomicArgs a)
{
    using A = Arith<T>;
    constexpr int B = mm_batch<T, K>();
    const T *__restrict__ val = static_cast<const T *>(a.val);
    const T *__restrict__ x = static_cast<const T *>(a.x);
    T *__restrict__ vbar = static_cast<T *>(a.vbar);
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < a.units;
         u += warps) {
        const uint32_t c = __ldg(a.unit_chunk + u);
        const uint32_t piece = u - __ldg(a.unit_base + c);
        const uint32_t g = 32u * c + (uint32_t)lane;
        const uint32_t len = g < a.nrows ? __ldg(a.klen + g) : 0u;
        const uint32_t j0 = piece * kK1Split;
        const uint32_t j1 = min(len, j0 + kK1Split);
        if (j0 >= j1) continue;
        T yb[K];
        load_row<T, K>(static_cast<const T *>(a.ybar), __ldg(a.permi + g), K, yb);
        const uint32_t base = __ldg(a.chp + c) + (uint32_t)lane;
        for (uint32_t j = j0; j < j1; j += B) {
            T v[B], xg[B][K];
            uint32_t cc[B], sr[B];
#pragma unroll
            for (int b = 0; b < B; b++) {
                const bool in = j + b < j1;
                const uint32_t pos = base + 32u * (j + b);
                v[b] = in ? __ldcs(val + pos) : T(0);
                cc[b] = in ? __ldcs(a.col + pos) : 0u;
                sr[b] = pos;  // vbar in forward slot order
            }
            if (vbar) {
#pragma unroll
                for (int b = 0; b < B; b++) {
                    if (j + b < j1) load_row<T, K>(x, cc[b], K, xg[b]);
                }
            }
#pragma unroll
            for (int b = 0; b < B; b++) {
                if (j + b < j1) {
                    T contrib[K];
#pragma unroll
                    for (int k = 0; k < K; k++) contrib[k] = A::mul(v[b], yb[k]);
                    if (vbar) {
                        T d = T(0);
#pragma unroll
                        for (int k = 0; k < K; k++) d = A::add(d, A::mul(yb[k], xg[b][k]));
                        vbar[sr[b]] = d;
                    }
                    red_row<T, K>(static_cast<T *>(a.xbar), cc[b], contrib);
                }
            }
        }
    }
}

// ------------------------------------------------------------------ layout helpers
// fsrc[slot] = CSR index of the element in K1 slot `slot` (kNoSrc for padding)
__global__ void k_k1_fsrc(uint32_t n, const uint32_t *row, const uint32_t *permi,
                          const uint32_t *chp, uint32_t *fsrc)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t r = permi[g], b = row[r], len = row[r + 1] - b;
    const uint32_t base = chp[g / 32] + (g % 32);
    for (uint32_t e = 0; e < len; e++) fsrc[base + 32u * e] = b + e;
}

template <class T>
__global__ void k_gather_vals(size_t nslots, const uint32_t *src, const T *v, T *out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nslots;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t s = src[i];
        out[i] = s == kNoSrc ? T(0) : v[s];
    }
}

template <class T>
__global__ void k_scatter_vals(size_t nslots, const uint32_t *src, const T *v, T *out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nslots;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t s = src[i];
        if (s != kNoSrc) out[s] = v[i];
    }
}

// inv[map[i]] = i for the real entries of map
__global__ void k_invert_map(size_t n, const uint32_t *map, uint32_t *inv)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t m = map[i];
        if (m != kNoSrc) inv[m] = (uint32_t)i;
    }
}

// out[i] = b[a[i]] (kNoSrc stays kNoSrc)
__global__ void k_compose_map(size_t n, const uint32_t *a, const uint32_t *b, uint32_t *out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t m = a[i];
        out[i] = m == kNoSrc ? kNoSrc : b[m];
    }
}

__global__ void k_expand_rows(uint32_t n, const uint32_t *row, uint32_t *rowidx)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    for (uint32_t e = row[r]; e < row[r + 1]; e++) rowidx[e] = r;
}

__global__ void k_col_keys(uint32_t nnz, uint32_t ncols, const uint32_t *col, uint32_t *key,
                           uint32_t *count)
{
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    key[e] = ncols - 1u - col[e];  // descending key = ascending column
    atomicAdd(count + col[e], 1u);
}

__global__ void k_t_meta(uint32_t m, const uint32_t *tl, const uint32_t *tperm, uint32_t *nmc,
                         uint32_t *klen)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= m) return;
    const uint32_t l = tl[tperm[g]];
    klen[g] = l;
    if ((g & 31) == 0) nmc[g >> 5] = l;
}

__global__ void k_narrow(uint32_t n, const uint64_t *a, uint32_t *b)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (uint32_t)a[i];
}

// transposed slot (chunk of sorted column g, step e) <- e-th element of column tperm[g]
__global__ void k_t_fill(uint32_t m, const uint32_t *tperm, const uint64_t *cptr,
                         const uint32_t *csc, const uint32_t *rowidx, const uint32_t *chp,
                         uint32_t *trow, uint32_t *tsrc)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= m) return;
    const uint32_t j = tperm[g];
    const uint64_t b = cptr[j], len = cptr[j + 1] - b;
    const uint32_t base = chp[g / 32] + (g % 32);
    for (uint32_t e = 0; e < len; e++) {
        const uint32_t k = csc[b + e];
        tsrc[base + 32u * e] = k;
        trow[base + 32u * e] = rowidx[k];
    }
}

// largest u + 1 over units of split chunks (the prefix the partial sums need)
__global__ void k_split_extent(uint32_t units, const uint32_t *unit_chunk,
                               const uint32_t *unit_base, uint32_t *out)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= units) return;
    const uint32_t c = unit_chunk[u];
    if (unit_base[c + 1] - unit_base[c] > 1) atomicMax(out, u + 1);
}

unsigned blocks_of(size_t n) { return (unsigned)((n + 255) / 256); }

gs_status split_extent(uint32_t units, const uint32_t *uc, const uint32_t *ub, uint32_t *out,
                       cudaStream_t s)
{
    *out = 0;
    if (!units) return GS_OK;
    DevBuf d;
    GS_TRY(d.alloc_zero(4, s));
    k_split_extent<<<blocks_of(units), 256, 0, s>>>(units, uc, ub, d.as<uint32_t>());
    GS_CHECK_LAUNCH();
    GS_CUDA(cudaMemcpyAsync(out, d.p, 4, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    return GS_OK;
}

template <class T, bool ADJ>
gs_status launch_mm(const MMArgs &a, uint32_t k, cudaStream_t s)
{
    if (!a.units) return GS_OK;
    const uint32_t blocks = min((a.units + 7) / 8, 148u * 64u);
    switch (k) {
    case 1: k_k1_mm<T, 1, ADJ><<<blocks, 256, 0, s>>>(a); break;
    case 2: k_k1_mm<T, 2, ADJ><<<blocks, 256, 0, s>>>(a); break;
    case 4: k_k1_mm<T, 4, ADJ><<<blocks, 256, 0, s>>>(a); break;
    case 8: k_k1_mm<T, 8, ADJ><<<blocks, 256, 0, s>>>(a); break;
    case 16: k_k1_mm<T, 16, ADJ><<<blocks, 256, 0, s>>>(a); break;
    case 32: k_k1_mm<T, 32, ADJ><<<blocks, 256, 0, s>>>(a); break;
    default: return fail(GS_ERR_UNSUPPORTED, "k = %u right-hand sides (1, 2, 4, 8, 16, 32)", k);
    }
    GS_CHECK_LAUNCH();
    return GS_OK;
}

template <class T>
gs_status launch_atomic(const AtomicArgs &a, uint32_t k, cudaStream_t s)
{
    if (!a.units) return GS_OK;
    const uint32_t blocks = min((a.units + 7) / 8, 148u * 64u);
    switch (k) {
    case 1: k_k1_adj_atomic<T, 1><<<blocks, 256, 0, s>>>(a); break;
    case 2: k_k1_adj_atomic<T, 2><<<blocks, 256, 0, s>>>(a); break;
    case 4: k_k1_adj_atomic<T, 4><<<blocks, 256, 0, s>>>(a); break;
    case 8: k_k1_adj_atomic<T, 8><<<blocks, 256, 0, s>>>(a); break;
    case 16: k_k1_adj_atomic<T, 16><<<blocks, 256, 0, s>>>(a); break;
    case 32: k_k1_adj_atomic<T, 32><<<blocks, 256, 0, s>>>(a); break;
    default: return fail(GS_ERR_UNSUPPORTED, "k = %u right-hand sides (1, 2, 4, 8, 16, 32)", k);
    }
    GS_CHECK_LAUNCH();
    return GS_OK;
}

bool valid_k(uint32_t k) { return k == 1 || k == 2 || k == 4 || k == 8 || k == 16 || k == 32; }

gs_status check_mm_matrix(const gs_matrix *A)
{
    if (A->p.format != GS_FMT_K1)
        return fail(GS_ERR_UNSUPPORTED, "multi-RHS products and adjoints run on K1 matrices");
    if (A->p.vtype != GS_F64 && A->p.vtype != GS_F32)
        return fail(GS_ERR_UNSUPPORTED, "multi-RHS products take FP64 or FP32 values");
    if (A->p.itype != GS_IDX_U32)
        return fail(GS_ERR_UNSUPPORTED, "multi-RHS products take 32-bit columns");
    return GS_OK;
}

bool aligned32(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 31u) == 0; }

std::mutex g_mm_mutex;  // guards the lazily sized multi-RHS scratch of a matrix

gs_status ensure_mm_scratch(gs_matrix *A, cudaStream_t s)
{
    std::lock_guard<std::mutex> lock(g_mm_mutex);
    if (A->mm_ready) return GS_OK;
    GS_TRY(split_extent(A->k1units, A->k1unit_chunk.as<uint32_t>(), A->k1unit_base.as<uint32_t>(),
                        &A->k1split_units, s));
    GS_TRY(A->mmpartial.alloc((size_t)A->k1split_units * 32 * 32 * 8 + 8));
    A->mm_ready = true;
    return GS_OK;
}

template <class T>
void refresh_values(gs_matrix *A, const T *v, gs_value_order order, cudaStream_t s)
{
    const unsigned gb = 148u * 16u;
    if (order == GS_VALUES_CSR) {
        k_gather_vals<T><<<gb, 256, 0, s>>>(A->lenVC, A->fsrc.as<uint32_t>(), v, A->val.as<T>());
        k_gather_vals<T><<<gb, 256, 0, s>>>(A->tlenVC, A->tsrc.as<uint32_t>(), v, A->tval.as<T>());
    } else {
        k_gather_vals<T><<<gb, 256, 0, s>>>(A->lenVC, A->ftslot.as<uint32_t>(), v, A->val.as<T>());
        cudaMemcpyAsync(A->tval.p, v, (size_t)A->tlenVC * sizeof(T), cudaMemcpyDeviceToDevice, s);
    }
}

}  // namespace

gs_status prepare_mm_scratch(gs_matrix *A, cudaStream_t s) { return ensure_mm_scratch(A, s); }

}  // namespace gs

using namespace gs;

extern "C" {

gs_status gs_spmm(gs_matrix *A, const void *d_X, void *d_Y, gs_dtype dtype, UIN k,
                  gs_stream stream)
{
    if (!A || !d_X || !d_Y) return fail(GS_ERR_INVALID, "NULL argument");
    GS_TRY(check_mm_matrix(A));
    if (dtype != A->p.vtype) return fail(GS_ERR_UNSUPPORTED, "X and Y take the value type");
    if (!valid_k(k)) return fail(GS_ERR_UNSUPPORTED, "k = %u right-hand sides (1, 2, 4, 8, 16, 32)", k);
    if (!aligned32(d_X) || !aligned32(d_Y)) return fail(GS_ERR_INVALID, "X and Y must be 32-byte aligned");
    cudaStream_t s = cs(stream);
    GS_TRY(ensure_mm_scratch(A, s));
    MMArgs a{};
    a.nrows = A->nrows;
    a.permi = A->permi.as<uint32_t>();
    a.nmc = A->nmc.as<uint32_t>();
    a.chp = A->chp.as<uint32_t>();
    a.klen = A->k1len.as<uint32_t>();
    a.val = A->val.p;
    a.col = A->col.as<uint32_t>();
    a.xin = d_X;
    a.yout = d_Y;
    a.unit_chunk = A->k1unit_chunk.as<uint32_t>();
    a.unit_base = A->k1unit_base.as<uint32_t>();
    a.units = A->k1units;
    a.split_units = A->k1split_units;
    a.partial = A->mmpartial.p;
    a.count = A->k1count.as<uint32_t>();
    a.ld = k;
    a.nrb = 1;
    if (A->p.vtype == GS_F64) return launch_mm<double, false>(a, k, s);
    return launch_mm<float, false>(a, k, s);
}

gs_status gs_matrix_prepare_adjoint(gs_matrix *A, const UIN *d_row, const UIN *d_col,
                                    gs_stream stream)
{
    if (!A || !d_row || (A->nnz && !d_col)) return fail(GS_ERR_INVALID, "NULL argument");
    GS_TRY(check_mm_matrix(A));
    cudaStream_t s = cs(stream);
    GS_TRY(ensure_mm_scratch(A, s));
    if (A->adj_ready) return GS_OK;
    const uint32_t n = A->nrows, m = A->ncols, nnz = A->nnz;
    // forward slot -> CSR index
    GS_TRY(A->fsrc.alloc((size_t)A->lenVC * 4));
    GS_CUDA(cudaMemsetAsync(A->fsrc.p, 0xff, (size_t)A->lenVC * 4, s));
    if (n) {
        k_k1_fsrc<<<blocks_of(n), 256, 0, s>>>(n, d_row, A->permi.as<uint32_t>(),
                                                A->chp.as<uint32_t>(), A->fsrc.as<uint32_t>());
        GS_CHECK_LAUNCH();
    }
    // CSC order of the elements: stable sort of CSR indices by ascending column
    DevBuf rowidx, key, ccount, csc, cptr;
    GS_TRY(rowidx.alloc((size_t)nnz * 4));
    GS_TRY(key.alloc((size_t)nnz * 4));
    GS_TRY(ccount.alloc_zero((size_t)m * 4, s));
    GS_TRY(csc.alloc((size_t)nnz * 4));
    if (n) {
        k_expand_rows<<<blocks_of(n), 256, 0, s>>>(n, d_row, rowidx.as<uint32_t>());
        GS_CHECK_LAUNCH();
    }
    if (nnz) {
        k_col_keys<<<blocks_of(nnz), 256, 0, s>>>(nnz, m, d_col, key.as<uint32_t>(),
                                                  ccount.as<uint32_t>());
        GS_CHECK_LAUNCH();
        GS_TRY(stable_sort_desc(key.as<uint32_t>(), nnz, m ? m - 1 : 0, csc.as<uint32_t>(), s));
    }
    GS_TRY(cptr.alloc(((size_t)m + 1) * 8));
    {
        CountSpec cc{CountKind::Array};
        cc.arr = ccount.as<uint32_t>();
        GS_TRY(exclusive_scan(cc, m, cptr.as<uint64_t>(), nullptr, s));
    }
    // K1 layout of A^T: columns of A sorted by decreasing length
    const uint32_t tchunks = (m + 31) / 32;
    A->tchunkNum = tchunks;
    uint32_t maxlen = 0;
    GS_TRY(reduce_max_u32(ccount.as<uint32_t>(), m, &maxlen, s));
    GS_TRY(A->tpermi.alloc_zero(((size_t)tchunks + 1) * 32 * 4, s));
    GS_TRY(stable_sort_desc(ccount.as<uint32_t>(), m, maxlen, A->tpermi.as<uint32_t>(), s));
    GS_TRY(A->tnmc.alloc_zero((size_t)tchunks * 4 + 4, s));
    GS_TRY(A->tlen.alloc((size_t)m * 4 + 4));
    if (m) {
        k_t_meta<<<blocks_of(m), 256, 0, s>>>(m, ccount.as<uint32_t>(), A->tpermi.as<uint32_t>(),
                                              A->tnmc.as<uint32_t>(), A->tlen.as<uint32_t>());
        GS_CHECK_LAUNCH();
    }
    DevBuf P;
    GS_TRY(P.alloc(((size_t)tchunks + 1) * 8));
    uint64_t lenvc = 0;
    {
        CountSpec cs{CountKind::ArrayTimes};
        cs.arr = A->tnmc.as<uint32_t>();
        cs.a = 32;
        GS_TRY(exclusive_scan(cs, tchunks, P.as<uint64_t>(), &lenvc, s));
    }
    if (lenvc > 0xffffffffull) return fail(GS_ERR_OVERFLOW, "transposed K1 exceeds 32-bit slots");
    A->tlenVC = (uint32_t)lenvc;
    GS_TRY(A->tchp.alloc((size_t)tchunks * 4 + 4));
    if (tchunks) {
        k_narrow<<<blocks_of(tchunks), 256, 0, s>>>(tchunks, P.as<uint64_t>(), A->tchp.as<uint32_t>());
        GS_CHECK_LAUNCH();
    }
    const size_t vsz = A->p.vtype == GS_F64 ? 8 : 4;
    GS_TRY(A->trow.alloc_zero((size_t)A->tlenVC * 4, s));
    GS_TRY(A->tsrc.alloc((size_t)A->tlenVC * 4));
    GS_CUDA(cudaMemsetAsync(A->tsrc.p, 0xff, (size_t)A->tlenVC * 4, s));
    GS_TRY(A->tval.alloc_zero((size_t)A->tlenVC * vsz, s));
    if (m) {
        k_t_fill<<<blocks_of(m), 256, 0, s>>>(m, A->tpermi.as<uint32_t>(), cptr.as<uint64_t>(),
                                              csc.as<uint32_t>(), rowidx.as<uint32_t>(),
                                              A->tchp.as<uint32_t>(), A->trow.as<uint32_t>(),
                                              A->tsrc.as<uint32_t>());
        GS_CHECK_LAUNCH();
    }
    GS_TRY(build_k1_plan(A->tnmc.as<uint32_t>(), tchunks, A->tunit_chunk, A->tunit_base,
                         A->tpartial1, A->tcount, &A->tunits, s));
    GS_TRY(split_extent(A->tunits, A->tunit_chunk.as<uint32_t>(), A->tunit_base.as<uint32_t>(),
                        &A->tsplit_units, s));
    GS_TRY(A->tpartial.alloc((size_t)A->tsplit_units * 32 * 32 * 8 + 8));
    // transposed values from the stored ones: forward slots -> CSR order (each CSR index
    // sits in exactly one forward slot) -> transposed slots
    DevBuf vcsr;
    GS_TRY(vcsr.alloc((size_t)nnz * vsz + 8));
    const unsigned gb = 148u * 16u;
    if (A->p.vtype == GS_F64) {
        k_scatter_vals<double><<<gb, 256, 0, s>>>(A->lenVC, A->fsrc.as<uint32_t>(),
                                                  A->val.as<double>(), vcsr.as<double>());
        k_gather_vals<double><<<gb, 256, 0, s>>>(A->tlenVC, A->tsrc.as<uint32_t>(),
                                                 vcsr.as<double>(), A->tval.as<double>());
    } else {
        k_scatter_vals<float><<<gb, 256, 0, s>>>(A->lenVC, A->fsrc.as<uint32_t>(),
                                                 A->val.as<float>(), vcsr.as<float>());
        k_gather_vals<float><<<gb, 256, 0, s>>>(A->tlenVC, A->tsrc.as<uint32_t>(),
                                                vcsr.as<float>(), A->tval.as<float>());
    }
    GS_CHECK_LAUNCH();
    // forward slot -> adjoint-layout slot, through the CSR index; the CSR index -> slot maps
    // stay: a value gradient in CSR order is formed in slot order (coalesced writes) and then
    // gathered into CSR order, instead of scattering one 4- or 8-byte write per element
    GS_TRY(A->csr2t.alloc((size_t)nnz * 4 + 4));
    GS_TRY(A->csr2f.alloc((size_t)nnz * 4 + 4));
    GS_TRY(A->ftslot.alloc((size_t)A->lenVC * 4 + 4));
    k_invert_map<<<gb, 256, 0, s>>>(A->tlenVC, A->tsrc.as<uint32_t>(), A->csr2t.as<uint32_t>());
    k_invert_map<<<gb, 256, 0, s>>>(A->lenVC, A->fsrc.as<uint32_t>(), A->csr2f.as<uint32_t>());
    k_compose_map<<<gb, 256, 0, s>>>(A->lenVC, A->fsrc.as<uint32_t>(), A->csr2t.as<uint32_t>(),
                                     A->ftslot.as<uint32_t>());
    GS_TRY(A->t2f.alloc((size_t)A->tlenVC * 4 + 4));
    k_compose_map<<<gb, 256, 0, s>>>(A->tlenVC, A->tsrc.as<uint32_t>(), A->csr2f.as<uint32_t>(),
                                     A->t2f.as<uint32_t>());
    GS_CHECK_LAUNCH();
    GS_TRY(A->vslots.alloc((size_t)max(A->lenVC, A->tlenVC) * vsz + 8));
    A->adj_ready = true;
    GS_CUDA(cudaStreamSynchronize(s));
    return GS_OK;
}

gs_status gs_matrix_set_values(gs_matrix *A, const void *d_val, gs_dtype dtype,
                               gs_value_order order, gs_stream stream)
{
    if (!A || (A->nnz && !d_val)) return fail(GS_ERR_INVALID, "NULL argument");
    GS_TRY(check_mm_matrix(A));
    if (!A->adj_ready)
        return fail(GS_ERR_INVALID, "gs_matrix_prepare_adjoint must run first");
    if (dtype != A->p.vtype) return fail(GS_ERR_UNSUPPORTED, "values take the matrix value type");
    if (order != GS_VALUES_CSR && order != GS_VALUES_SLOTS)
        return fail(GS_ERR_INVALID, "unknown value order %d", (int)order);
    cudaStream_t s = cs(stream);
    if (dtype == GS_F64) refresh_values(A, static_cast<const double *>(d_val), order, s);
    else refresh_values(A, static_cast<const float *>(d_val), order, s);
    GS_CHECK_LAUNCH();
    return GS_OK;
}

gs_status gs_matrix_value_slots(const gs_matrix *A, UIN *nslots)
{
    if (!A || !nslots) return fail(GS_ERR_INVALID, "NULL argument");
    if (!A->adj_ready) return fail(GS_ERR_INVALID, "gs_matrix_prepare_adjoint must run first");
    *nslots = A->tlenVC;
    return GS_OK;
}

gs_status gs_matrix_convert_values(const gs_matrix *A, const void *d_in, gs_value_order in_order,
                                   void *d_out, gs_dtype dtype, gs_stream stream)
{
    if (!A || !d_in || !d_out) return fail(GS_ERR_INVALID, "NULL argument");
    if (!A->adj_ready) return fail(GS_ERR_INVALID, "gs_matrix_prepare_adjoint must run first");
    if (dtype != A->p.vtype) return fail(GS_ERR_UNSUPPORTED, "values take the matrix value type");
    cudaStream_t s = cs(stream);
    const unsigned gb = 148u * 16u;
    const bool f64 = dtype == GS_F64;
    if (in_order == GS_VALUES_CSR) {  // slots[t] = csr[tsrc[t]], padding 0
        if (f64)
            k_gather_vals<double><<<gb, 256, 0, s>>>(A->tlenVC, A->tsrc.as<uint32_t>(),
                                                     static_cast<const double *>(d_in),
                                                     static_cast<double *>(d_out));
        else
            k_gather_vals<float><<<gb, 256, 0, s>>>(A->tlenVC, A->tsrc.as<uint32_t>(),
                                                    static_cast<const float *>(d_in),
                                                    static_cast<float *>(d_out));
    } else if (in_order == GS_VALUES_SLOTS) {  // csr[tsrc[t]] = slots[t]
        if (f64)
            k_scatter_vals<double><<<gb, 256, 0, s>>>(A->tlenVC, A->tsrc.as<uint32_t>(),
                                                      static_cast<const double *>(d_in),
                                                      static_cast<double *>(d_out));
        else
            k_scatter_vals<float><<<gb, 256, 0, s>>>(A->tlenVC, A->tsrc.as<uint32_t>(),
                                                     static_cast<const float *>(d_in),
                                                     static_cast<float *>(d_out));
    } else {
        return fail(GS_ERR_INVALID, "unknown value order %d", (int)in_order);
    }
    GS_CHECK_LAUNCH();
    return GS_OK;
}

gs_status gs_spmm_adjoint(gs_matrix *A, const void *d_Ybar, const void *d_X, void *d_Xbar,
                          void *d_vbar, gs_dtype dtype, UIN k, gs_adjoint_mode mode,
                          gs_value_order vbar_order, gs_stream stream)
{
    if (vbar_order != GS_VALUES_CSR && vbar_order != GS_VALUES_SLOTS)
        return fail(GS_ERR_INVALID, "unknown value order %d", (int)vbar_order);
    if (!A || !d_Ybar || !d_Xbar || (d_vbar && !d_X)) return fail(GS_ERR_INVALID, "NULL argument");
    GS_TRY(check_mm_matrix(A));
    if (!A->adj_ready)
        return fail(GS_ERR_INVALID, "gs_matrix_prepare_adjoint must run first");
    if (dtype != A->p.vtype) return fail(GS_ERR_UNSUPPORTED, "operands take the value type");
    if (!valid_k(k)) return fail(GS_ERR_UNSUPPORTED, "k = %u right-hand sides (1, 2, 4, 8, 16, 32)", k);
    if (!aligned32(d_Ybar) || !aligned32(d_Xbar) || (d_X && !aligned32(d_X)))
        return fail(GS_ERR_INVALID, "Ybar, X and Xbar must be 32-byte aligned");
    cudaStream_t s = cs(stream);
    const bool f64 = A->p.vtype == GS_F64;
    const unsigned gb = 148u * 16u;
    if (mode == GS_ADJ_ATOMIC) {
        GS_CUDA(cudaMemsetAsync(d_Xbar, 0, (size_t)A->ncols * k * (f64 ? 8 : 4), s));
        AtomicArgs a{};
        a.nrows = A->nrows;
        a.permi = A->permi.as<uint32_t>();
        a.chp = A->chp.as<uint32_t>();
        a.klen = A->k1len.as<uint32_t>();
        a.col = A->col.as<uint32_t>();
        // vbar in forward slot order first (coalesced), then gathered into the asked order
        const bool via_slots = d_vbar != nullptr;
        a.unit_chunk = A->k1unit_chunk.as<uint32_t>();
        a.unit_base = A->k1unit_base.as<uint32_t>();
        a.units = A->k1units;
        a.val = A->val.p;
        a.x = d_X;
        a.ybar = d_Ybar;
        a.xbar = d_Xbar;
        a.vbar = via_slots ? A->vslots.p : d_vbar;
        GS_TRY((f64 ? launch_atomic<double>(a, k, s) : launch_atomic<float>(a, k, s)));
        if (via_slots) {
            const bool csr = vbar_order == GS_VALUES_CSR;
            const size_t n_out = csr ? A->nnz : A->tlenVC;
            const uint32_t *map = csr ? A->csr2f.as<uint32_t>() : A->t2f.as<uint32_t>();
            if (f64)
                k_gather_vals<double><<<gb, 256, 0, s>>>(n_out, map, A->vslots.as<double>(),
                                                         static_cast<double *>(d_vbar));
            else
                k_gather_vals<float><<<gb, 256, 0, s>>>(n_out, map, A->vslots.as<float>(),
                                                        static_cast<float *>(d_vbar));
            GS_CHECK_LAUNCH();
        }
        return GS_OK;
    }
    if (mode != GS_ADJ_DETERMINISTIC) return fail(GS_ERR_INVALID, "unknown adjoint mode %d", (int)mode);
    MMArgs a{};
    a.nrows = A->ncols;
    a.permi = A->tpermi.as<uint32_t>();
    a.nmc = A->tnmc.as<uint32_t>();
    a.chp = A->tchp.as<uint32_t>();
    a.klen = A->tlen.as<uint32_t>();
    a.val = A->tval.p;
    a.col = A->trow.as<uint32_t>();
    a.xin = d_Ybar;
    a.xrow = d_X;
    a.yout = d_Xbar;
    // CSR order: vbar in the adjoint layout's slot order first, then gathered into CSR order
    const bool via_slots = d_vbar && vbar_order == GS_VALUES_CSR;
    a.vbar = via_slots ? A->vslots.p : d_vbar;
    a.unit_chunk = A->tunit_chunk.as<uint32_t>();
    a.unit_base = A->tunit_base.as<uint32_t>();
    a.units = A->tunits;
    a.split_units = A->tsplit_units;
    a.partial = A->tpartial.p;
    a.count = A->tcount.as<uint32_t>();
    a.ld = k;
    a.nrb = 1;
    GS_TRY((f64 ? launch_mm<double, true>(a, k, s) : launch_mm<float, true>(a, k, s)));
    if (via_slots) {
        if (f64)
            k_gather_vals<double><<<gb, 256, 0, s>>>(A->nnz, A->csr2t.as<uint32_t>(),
                                                     A->vslots.as<double>(),
                                                     static_cast<double *>(d_vbar));
        else
            k_gather_vals<float><<<gb, 256, 0, s>>>(A->nnz, A->csr2t.as<uint32_t>(),
                                                    A->vslots.as<float>(),
                                                    static_cast<float *>(d_vbar));
        GS_CHECK_LAUNCH();
    }
    return GS_OK;
}

}  // extern "C"
