// gs_gen.cpp -- seeded synthetic matrices and vectors for the benchmark workloads.
//
// The reference reads SuiteSparse-style matrices from files (jobLauncher.sh:58-70) that
// are not available here; these generators produce the workloads the engine is measured
// on, deterministically for a seed regardless of the thread count (every row, element or
// vector entry draws from its own counter-based stream).
//
//   laplacian2d : 5-point Laplacian on a grid x grid mesh, diagonal 4, off-diagonals -1
//   powerlaw    : lognormal(mu, sigma) row lengths clipped to [1, max_len], rescaled so
//                 the total is exactly target_nnz; columns uniform without replacement,
//                 sorted within the row; values N(0,1)
//   stencil27   : 27-point stencil on grid^3, diagonal 26, off-diagonals -1 + U(-0.1,0.1)
//   banded      : lengths U[min_len, max_len] clipped to the band, columns uniform without
//                 replacement inside [r-half_bw, r+half_bw], values N(0,1)
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gpuspmv_b200.h"

namespace {

inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// splitmix64 stream keyed by (seed, stream id)
struct Rng {
    uint64_t s;
    Rng(uint64_t seed, uint64_t stream) : s(mix64(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull) ^ mix64(stream + 0x3C6EF372FE94F82Bull)) {}
    uint64_t next() { s += 0x9E3779B97F4A7C15ull; return mix64(s); }
    double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }  // [0, 1)
    double normal()
    {
        double u1 = 1.0 - uniform();  // (0, 1]
        double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};

constexpr uint64_t kColStream = 0x100000000ull;
constexpr uint64_t kValStream = 0x200000000ull;

// k distinct values in [lo, lo+width), sorted ascending, drawn from rng
void distinct_sorted(Rng &rng, uint32_t lo, uint32_t width, uint32_t k, uint32_t *out)
{
    if (k == 0) return;
    if ((uint64_t)k * 2 >= width) {
        // dense case: partial Fisher-Yates over the whole range
        std::vector<uint32_t> pool(width);
        for (uint32_t i = 0; i < width; i++) pool[i] = lo + i;
        for (uint32_t i = 0; i < k; i++) {
            uint32_t j = i + (uint32_t)rng.below(width - i);
            std::swap(pool[i], pool[j]);
        }
        std::copy(pool.begin(), pool.begin() + k, out);
        std::sort(out, out + k);
        return;
    }
    uint32_t have = 0;
    while (have < k) {
        for (uint32_t i = have; i < k; i++) out[i] = lo + (uint32_t)rng.below(width);
        std::sort(out, out + k);
        have = (uint32_t)(std::unique(out, out + k) - out);
    }
}

gs_status alloc_csr(uint32_t n, uint64_t nnz, UIN **row, UIN **col, double **val)
{
    if (nnz > 0xffffffffull) return GS_ERR_OVERFLOW;
    *row = (UIN *)malloc(((size_t)n + 1) * sizeof(UIN));
    *col = (UIN *)malloc((size_t)(nnz ? nnz : 1) * sizeof(UIN));
    *val = (double *)malloc((size_t)(nnz ? nnz : 1) * sizeof(double));
    if (!*row || !*col || !*val) {
        free(*row); free(*col); free(*val);
        *row = nullptr; *col = nullptr; *val = nullptr;
        return GS_ERR_ALLOC;
    }
    return GS_OK;
}

void prefix(uint32_t n, const std::vector<uint32_t> &len, UIN *row)
{
    row[0] = 0;
    for (uint32_t r = 0; r < n; r++) row[r + 1] = row[r] + len[r];
}

}  // namespace

extern "C" {

void gs_free_host(void *p) { free(p); }

gs_status gs_gen_vector(uint64_t n, int dist, double lo, double hi, uint64_t seed, double *v)
{
    if (!v) return GS_ERR_INVALID;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        Rng g(seed, (uint64_t)i);
        v[i] = dist == 0 ? lo + (hi - lo) * g.uniform() : g.normal();
    }
    return GS_OK;
}

gs_status gs_gen_laplacian2d(UIN grid, UIN **row, UIN **col, double **val, UIN *nrows, UIN *nnz)
{
    if (!grid || (uint64_t)grid * grid > 0xffffffffull) return GS_ERR_INVALID;
    const uint32_t n = grid * grid;
    std::vector<uint32_t> len(n);
    for (uint32_t r = 0; r < n; r++) {
        uint32_t i = r / grid, j = r % grid;
        len[r] = 1 + (i > 0) + (j > 0) + (j + 1 < grid) + (i + 1 < grid);
    }
    uint64_t tot = 0;
    for (uint32_t l : len) tot += l;
    gs_status st = alloc_csr(n, tot, row, col, val);
    if (st) return st;
    prefix(n, len, *row);
#pragma omp parallel for schedule(static)
    for (int64_t rr = 0; rr < (int64_t)n; rr++) {
        uint32_t r = (uint32_t)rr, i = r / grid, j = r % grid, p = (*row)[r];
        auto put = [&](uint32_t c, double v) { (*col)[p] = c; (*val)[p] = v; p++; };
        if (i > 0) put(r - grid, -1.0);
        if (j > 0) put(r - 1, -1.0);
        put(r, 4.0);
        if (j + 1 < grid) put(r + 1, -1.0);
        if (i + 1 < grid) put(r + grid, -1.0);
    }
    *nrows = n;
    *nnz = (UIN)tot;
    return GS_OK;
}

gs_status gs_gen_powerlaw(UIN n, uint64_t target, double mu, double sigma, UIN max_len,
                          uint64_t seed, UIN **row, UIN **col, double **val, UIN *nnz)
{
    if (!n || !max_len || target > 0xffffffffull) return GS_ERR_INVALID;
    const uint32_t cap = std::min<uint32_t>(max_len, n);
    if (target < n || target > (uint64_t)cap * n) return GS_ERR_INVALID;
    std::vector<double> L(n);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < (int64_t)n; r++) {
        Rng g(seed, (uint64_t)r);
        double l = std::exp(mu + sigma * g.normal());
        L[r] = std::min(std::max(l, 1.0), (double)max_len);
    }
    auto total_at = [&](double s) {
        uint64_t t = 0;
#pragma omp parallel for reduction(+ : t) schedule(static)
        for (int64_t r = 0; r < (int64_t)n; r++) {
            double v = std::rint(L[r] * s);
            t += (uint64_t)std::min(std::max(v, 1.0), (double)cap);
        }
        return t;
    };
    double lo = 0.0, hi = 1.0;
    while (total_at(hi) < target && hi < 1e12) hi *= 2;
    for (int it = 0; it < 100; it++) {
        double mid = 0.5 * (lo + hi);
        if (total_at(mid) < target) lo = mid; else hi = mid;
    }
    std::vector<uint32_t> len(n);
    uint64_t tot = 0;
    for (uint32_t r = 0; r < n; r++) {
        double v = std::rint(L[r] * hi);
        len[r] = (uint32_t)std::min(std::max(v, 1.0), (double)cap);
        tot += len[r];
    }
    // settle the rounding residue deterministically so the total is exactly target
    for (uint32_t r = 0; tot > target; r = (r + 1) % n)
        if (len[r] > 1) { len[r]--; tot--; }
    for (uint32_t r = 0; tot < target; r = (r + 1) % n)
        if (len[r] < cap) { len[r]++; tot++; }
    gs_status st = alloc_csr(n, tot, row, col, val);
    if (st) return st;
    prefix(n, len, *row);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t r = 0; r < (int64_t)n; r++) {
        Rng gc(seed, kColStream + (uint64_t)r), gv(seed, kValStream + (uint64_t)r);
        const uint32_t p = (*row)[r];
        distinct_sorted(gc, 0, n, len[r], *col + p);
        for (uint32_t e = 0; e < len[r]; e++) (*val)[p + e] = gv.normal();
    }
    *nnz = (UIN)tot;
    return GS_OK;
}

gs_status gs_gen_stencil27(UIN grid, uint64_t seed, UIN **row, UIN **col, double **val,
                           UIN *nrows, UIN *nnz)
{
    if (!grid || (uint64_t)grid * grid * grid > 0xffffffffull) return GS_ERR_INVALID;
    const uint32_t g = grid, n = g * g * g;
    std::vector<uint32_t> len(n);
    auto span = [&](uint32_t a) { return (uint32_t)(1 + (a > 0) + (a + 1 < g)); };
#pragma omp parallel for schedule(static)
    for (int64_t rr = 0; rr < (int64_t)n; rr++) {
        uint32_t r = (uint32_t)rr, i = r % g, j = (r / g) % g, k = r / (g * g);
        len[r] = span(i) * span(j) * span(k);
    }
    uint64_t tot = 0;
    for (uint32_t l : len) tot += l;
    gs_status st = alloc_csr(n, tot, row, col, val);
    if (st) return st;
    prefix(n, len, *row);
#pragma omp parallel for schedule(static)
    for (int64_t rr = 0; rr < (int64_t)n; rr++) {
        uint32_t r = (uint32_t)rr, i = r % g, j = (r / g) % g, k = r / (g * g), p = (*row)[r];
        Rng gv(seed, (uint64_t)r);
        for (int dk = -1; dk <= 1; dk++)
            for (int dj = -1; dj <= 1; dj++)
                for (int di = -1; di <= 1; di++) {
                    int64_t ii = (int64_t)i + di, jj = (int64_t)j + dj, kk = (int64_t)k + dk;
                    if (ii < 0 || jj < 0 || kk < 0 || ii >= g || jj >= g || kk >= g) continue;
                    (*col)[p] = (uint32_t)(ii + (int64_t)g * (jj + (int64_t)g * kk));
                    (*val)[p] = (di == 0 && dj == 0 && dk == 0)
                                    ? 26.0
                                    : -1.0 + 0.1 * (2.0 * gv.uniform() - 1.0);
                    p++;
                }
    }
    *nrows = n;
    *nnz = (UIN)tot;
    return GS_OK;
}

gs_status gs_gen_banded(UIN n, UIN half_bw, UIN min_len, UIN max_len, uint64_t seed, UIN **row,
                        UIN **col, double **val, UIN *nnz)
{
    if (!n || min_len > max_len) return GS_ERR_INVALID;
    std::vector<uint32_t> len(n);
    for (uint32_t r = 0; r < n; r++) {
        Rng g(seed, (uint64_t)r);
        uint32_t lo = r > half_bw ? r - half_bw : 0;
        uint32_t hi = std::min<uint64_t>((uint64_t)r + half_bw, (uint64_t)n - 1);
        uint32_t l = min_len + (uint32_t)g.below((uint64_t)max_len - min_len + 1);
        len[r] = std::min(l, hi - lo + 1);
    }
    uint64_t tot = 0;
    for (uint32_t l : len) tot += l;
    gs_status st = alloc_csr(n, tot, row, col, val);
    if (st) return st;
    prefix(n, len, *row);
#pragma omp parallel for schedule(static)
    for (int64_t rr = 0; rr < (int64_t)n; rr++) {
        uint32_t r = (uint32_t)rr;
        uint32_t lo = r > half_bw ? r - half_bw : 0;
        uint32_t hi = std::min<uint64_t>((uint64_t)r + half_bw, (uint64_t)n - 1);
        Rng gc(seed, kColStream + r), gv(seed, kValStream + r);
        const uint32_t p = (*row)[r];
        distinct_sorted(gc, lo, hi - lo + 1, len[r], *col + p);
        for (uint32_t e = 0; e < len[r]; e++) (*val)[p + e] = gv.normal();
    }
    *nnz = (UIN)tot;
    return GS_OK;
}

}  // extern "C"
