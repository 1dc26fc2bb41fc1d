// The tile-aware reorder planner of the reference (TASA; build_reorder_plan,
// src/reorder.h:2044-2428), behind the same entry point and ReorderInfo.
//
// What it computes, by problem and matrix:
//   * AA with a symmetric matrix (src/reorder.h:2205-2279): one order shared
//     by all three axes, chosen from the rows' tile sets (the distinct tile
//     columns of each row) --
//       - n <= 50,000 whose natural tile rows hold < 32 tiles on average:
//         identity ("identity_narrow_tiles");
//       - n <= 50,000 otherwise: reverse Cuthill-McKee over the pattern
//         with seeds and neighbours taken by (tile count, degree, id), each
//         component reversed on its own, then a windowed greedy refinement
//         that pulls forward the row sharing most tiles with its
//         predecessor (window 32);
//       - n > 50,000: windowed packing of the natural order into groups of
//         up to 16 rows, each next row the one adding the fewest new tiles
//         to its group (score 96 overlap - 64 added - 48 distance/16).
//   * AA with a general matrix, A*B and A*A^T (:2166-2204, :2046-2152): each
//     axis sorted by a tile signature of its rows / columns -- distinct
//     tiles, first three and last tile, degree and two order hashes -- by
//     (band of the first tile, first, second, third tile, tile-count bucket
//     descending, span, last tile, degree bucket descending, hashes, id);
//     the inner axis by the signature of A's columns combined with B's
//     rows (A's rows for AA).
//   * every plan: the sampled tile estimates before and after, then the
//     structural risk guard (:1989-2042), which falls back to identity when
//     the estimates grow (thresholds as the reference's; TASA_FORCE_ACTIVE=1
//     accepts any plan, TASA_AB_SHARED_SYM=1 lets an A*B of two symmetric
//     matrices take the symmetric plan).
//
// B200 design: the signatures of the general path are computed on the GPU
// (a thread per row; the columns through one radix sort of (column, row)
// keys) and each axis is ordered by five stable 64-bit radix-sort passes
// over packed keys (least significant first), which gives the comparator's
// total order exactly.  The symmetric path is host code as in the
// reference -- its RCM is over n <= 50,000 -- with the packing windows,
// which are independent, spread over host threads.
#include <limits.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <algorithm>
#include <numeric>
#include <thread>
#include <vector>

#include "tsg_internal.h"

int tsg_axis_alloc(AxisPermutation *p, int n);
int tsg_axis_from_order(AxisPermutation *p, const int *order, int n);
int tsg_axis_copy(AxisPermutation *dst, const AxisPermutation *src);
void tsg_info_text(char *dst, size_t size, const char *src);
long long tsg_estimate_input_tiles(const SMatrix *M, const AxisPermutation *row, const AxisPermutation *col);
long long tsg_estimate_c_tiles(const SMatrix *A, const SMatrix *B, const AxisPermutation *row,
                               const AxisPermutation *inner, const AxisPermutation *col, bool one);
tsg_context *tsg_dropin_context(void);

namespace
{

double now_ms()
{
    timeval t;
    gettimeofday(&t, nullptr);
    return t.tv_sec * 1000.0 + t.tv_usec / 1000.0;
}

// SplitMix64's output function (Steele, Lea, Flood 2014; Vigna's constants)
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long x)
{
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// floor(log2(v)) for v >= 1, 0 below, at most 31
__host__ __device__ __forceinline__ int log2_bucket(int v)
{
    int b = 0;
    for (v = v > 0 ? v : 0; v > 1 && b < 31; v >>= 1)
        b++;
    return b;
}

constexpr unsigned long long FNV_BASIS = 1469598103934665603ULL, FNV_PRIME = 1099511628211ULL;

// ---------------------------------------------------------------------------
// general path: signatures on the device
// ---------------------------------------------------------------------------
struct Sig
{
    int n = 0;
    int *count = nullptr, *first = nullptr, *last = nullptr, *second = nullptr, *third = nullptr, *degree = nullptr;
    unsigned long long *h1 = nullptr, *h2 = nullptr;
};

int sig_alloc(tsg_context *ctx, Sig *s, int n)
{
    s->n = n;
    const size_t c = (size_t)(n > 0 ? n : 1);
    TSG_TRY(tsg_alloc(ctx, &s->count, c));
    TSG_TRY(tsg_alloc(ctx, &s->first, c));
    TSG_TRY(tsg_alloc(ctx, &s->last, c));
    TSG_TRY(tsg_alloc(ctx, &s->second, c));
    TSG_TRY(tsg_alloc(ctx, &s->third, c));
    TSG_TRY(tsg_alloc(ctx, &s->degree, c));
    TSG_TRY(tsg_alloc(ctx, &s->h1, c));
    TSG_TRY(tsg_alloc(ctx, &s->h2, c));
    return TSG_OK;
}

void sig_free(tsg_context *ctx, Sig *s)
{
    tsg_release(ctx, s->count);
    tsg_release(ctx, s->first);
    tsg_release(ctx, s->last);
    tsg_release(ctx, s->second);
    tsg_release(ctx, s->third);
    tsg_release(ctx, s->degree);
    tsg_release(ctx, s->h1);
    tsg_release(ctx, s->h2);
}

// A signature from the ascending tile sequence of one row or column
// (repeats skipped); ordered: the row form chains two order-dependent
// hashes, the column form XORs two per-tile hashes.
struct SigAcc
{
    int count = 0, first = INT_MAX, last = -1, second = INT_MAX, third = INT_MAX, prev = -1;
    unsigned long long h1, h2;
    __device__ void add_row(int t)
    {
        if (t == prev)
            return;
        if (count == 1)
            second = t;
        else if (count == 2)
            third = t;
        count++;
        first = min(first, t);
        last = max(last, t);
        const unsigned long long m = mix64((unsigned long long)t);
        h1 = (h1 ^ m) * FNV_PRIME;
        h2 ^= m + (h2 << 6) + (h2 >> 2);
        prev = t;
    }
    __device__ void add_col(int t)
    {
        if (t == prev)
            return;
        if (count == 1)
            second = t;
        else if (count == 2)
            third = t;
        count++;
        first = min(first, t);
        last = max(last, t);
        h1 ^= mix64((unsigned long long)t);
        h2 ^= mix64((unsigned long long)t ^ 0x9e3779b97f4a7c15ULL);
        prev = t;
    }
    __device__ void store(const Sig &s, int i, int degree) const
    {
        s.count[i] = count;
        s.first[i] = count > 0 ? first : INT_MAX;
        s.last[i] = last;
        s.second[i] = second;
        s.third[i] = third;
        s.degree[i] = degree;
        s.h1[i] = h1;
        s.h2[i] = h2;
    }
};

// thread per row: the tiles of its columns in CSR order (rows sorted)
__global__ void k_row_signatures(int m, const int *__restrict__ rp, const int *__restrict__ ci, Sig s)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m)
        return;
    SigAcc a;
    a.h1 = FNV_BASIS;
    a.h2 = FNV_PRIME ^ (unsigned long long)i;
    for (int p = rp[i]; p < rp[i + 1]; p++)
        a.add_row(ci[p] / TSG_BS);
    a.store(s, i, rp[i + 1] - rp[i]);
}

__global__ void k_col_keys(int m, const int *__restrict__ rp, const int *__restrict__ ci,
                           unsigned long long *__restrict__ keys, int *__restrict__ vals, int *__restrict__ cdeg)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m)
        return;
    for (int p = rp[i]; p < rp[i + 1]; p++)
    {
        keys[p] = ((unsigned long long)(unsigned)ci[p] << 32) | (unsigned)i;
        vals[p] = p;
        atomicAdd(cdeg + ci[p], 1);
    }
}

// thread per column over its rows, ascending (the sorted keys' segment)
__global__ void k_col_signatures(int n, const int *__restrict__ cptr, const unsigned long long *__restrict__ keys, Sig s)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n)
        return;
    SigAcc a;
    a.h1 = 0;
    a.h2 = 0;
    for (int p = cptr[c]; p < cptr[c + 1]; p++)
        a.add_col((int)(unsigned)(keys[p] & 0xffffffffULL) / TSG_BS);
    a.store(s, c, cptr[c + 1] - cptr[c]);
}

int row_signatures(tsg_context *ctx, int m, const int *d_rp, const int *d_ci, Sig *s)
{
    TSG_TRY(sig_alloc(ctx, s, m));
    if (m > 0)
    {
        k_row_signatures<<<tsg_blocks(m, 256), 256, 0, ctx->stream>>>(m, d_rp, d_ci, *s);
        TSG_LAUNCH_CHECK();
    }
    return TSG_OK;
}

__global__ void k_sig_empty(int n, Sig s)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        s.count[i] = 0;
        s.first[i] = INT_MAX;
        s.last[i] = -1;
        s.second[i] = INT_MAX;
        s.third[i] = INT_MAX;
        s.degree[i] = 0;
        s.h1[i] = 0;
        s.h2[i] = 0;
    }
}

int col_signatures(tsg_context *ctx, int m, int n, int nnz, const int *d_rp, const int *d_ci, Sig *s)
{
    TSG_TRY(sig_alloc(ctx, s, n));
    if (n <= 0)
        return TSG_OK;
    if (m <= 0 || nnz <= 0)
    {
        k_sig_empty<<<tsg_blocks(n, 256), 256, 0, ctx->stream>>>(n, *s);
        TSG_LAUNCH_CHECK();
        return TSG_OK;
    }
    unsigned long long *keys;
    int *vals, *cptr;
    TSG_TRY(tsg_alloc(ctx, &keys, (size_t)nnz));
    TSG_TRY(tsg_alloc(ctx, &vals, (size_t)nnz));
    TSG_TRY(tsg_alloc(ctx, &cptr, (size_t)n + 1));
    TSG_CUDA(cudaMemsetAsync(cptr, 0, ((size_t)n + 1) * sizeof(int), ctx->stream));
    k_col_keys<<<tsg_blocks(m, 256), 256, 0, ctx->stream>>>(m, d_rp, d_ci, keys, vals, cptr);
    TSG_LAUNCH_CHECK();
    TSG_TRY(tsg_scan_counts(ctx, cptr, cptr, n, nullptr));
    TSG_TRY(tsg_sort_pairs_u64(ctx, keys, vals, nnz, 64));
    k_col_signatures<<<tsg_blocks(n, 256), 256, 0, ctx->stream>>>(n, cptr, keys, *s);
    TSG_LAUNCH_CHECK();
    tsg_release(ctx, keys);
    tsg_release(ctx, vals);
    tsg_release(ctx, cptr);
    return TSG_OK;
}

// Sort keys of the signature order, most significant first:
//   k[0] = band << 31 | first        k[1] = second << 31 | third
//   k[2] = (31 - count bucket) << 59 | span << 32 | (last + 1) << 5 | (31 - degree bucket)
//   k[3] = hash1                      k[4] = hash2
// (tile indices below 2^27, so span and last + 1 fit 27 bits); ties of all
// five keep the id order.
__global__ void k_sig_keys(int n, int dim, Sig l, Sig r, bool combined, unsigned long long *__restrict__ k)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int count = l.count[i], first = l.first[i], last = l.last[i], second = l.second[i], third = l.third[i];
    int degree = l.degree[i];
    unsigned long long h1 = l.h1[i], h2 = l.h2[i];
    if (combined)
    {
        count += r.count[i];
        first = min(first, r.first[i]);
        last = max(last, r.last[i]);
        second = min(second, r.second[i]);
        third = min(third, r.third[i]);
        degree += r.degree[i];
        h1 = l.h1[i] ^ mix64(r.h1[i]);
        h2 = r.h2[i] ^ mix64(l.h2[i]);
    }
    const int span = last >= first ? last - first + 1 : 0;
    int band = INT_MAX;
    if (count > 0 && first < dim)
        band = first / (span <= 8 ? 4 : (span <= 32 ? 8 : 16));
    const int f = count > 0 ? first : INT_MAX;
    k[i] = ((unsigned long long)band << 31) | (unsigned)f;
    k[(size_t)n + i] = ((unsigned long long)(unsigned)second << 31) | (unsigned)third;
    k[2 * (size_t)n + i] = ((unsigned long long)(31 - log2_bucket(count)) << 59) | ((unsigned long long)span << 32) |
                           ((unsigned long long)(unsigned)(last + 1) << 5) | (unsigned long long)(31 - log2_bucket(degree));
    k[3 * (size_t)n + i] = h1;
    k[4 * (size_t)n + i] = h2;
}

__global__ void k_gather_key(int n, const unsigned long long *__restrict__ k, const int *__restrict__ perm,
                             unsigned long long *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = k[perm[i]];
}

__global__ void k_iota(int n, int *__restrict__ p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        p[i] = i;
}

// new -> old order of the signatures l (combined with r when given)
int order_by_signature(tsg_context *ctx, const Sig &l, const Sig *r, int dim, AxisPermutation *perm)
{
    const int n = l.n;
    if (dim >= (1 << 27) - 1)
        return tsg_set_error(TSG_ERR_INVALID, "TASA planner: more than 2^27 tiles on an axis");
    std::vector<int> h((size_t)(n > 0 ? n : 1));
    if (n > 0)
    {
        unsigned long long *k, *g;
        int *p;
        TSG_TRY(tsg_alloc(ctx, &k, 5 * (size_t)n));
        TSG_TRY(tsg_alloc(ctx, &g, (size_t)n));
        TSG_TRY(tsg_alloc(ctx, &p, (size_t)n));
        k_sig_keys<<<tsg_blocks(n, 256), 256, 0, ctx->stream>>>(n, dim, l, r ? *r : l, r != nullptr, k);
        TSG_LAUNCH_CHECK();
        k_iota<<<tsg_blocks(n, 256), 256, 0, ctx->stream>>>(n, p);
        TSG_LAUNCH_CHECK();
        for (int pass = 4; pass >= 0; pass--) // least significant key first; each sort is stable
        {
            k_gather_key<<<tsg_blocks(n, 256), 256, 0, ctx->stream>>>(n, k + (size_t)pass * n, p, g);
            TSG_LAUNCH_CHECK();
            TSG_TRY(tsg_sort_pairs_u64(ctx, g, p, n, 64));
        }
        TSG_CUDA(cudaMemcpyAsync(h.data(), p, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        TSG_CUDA(cudaStreamSynchronize(ctx->stream));
        tsg_release(ctx, k);
        tsg_release(ctx, g);
        tsg_release(ctx, p);
    }
    return tsg_axis_from_order(perm, h.data(), n) == 0 ? TSG_OK : tsg_set_error(TSG_ERR_OOM, "permutation");
}

struct DevPattern
{
    int m = 0, n = 0, nnz = 0;
    int *rp = nullptr, *ci = nullptr;
};

int upload_pattern(tsg_context *ctx, const SMatrix *M, DevPattern *d)
{
    d->m = M->m;
    d->n = M->n;
    d->nnz = M->nnz;
    TSG_TRY(tsg_alloc(ctx, &d->rp, (size_t)M->m + 1));
    TSG_TRY(tsg_alloc(ctx, &d->ci, (size_t)(M->nnz > 0 ? M->nnz : 1)));
    TSG_CUDA(cudaMemcpyAsync(d->rp, M->rowpointer, ((size_t)M->m + 1) * sizeof(int), cudaMemcpyHostToDevice,
                             ctx->stream));
    if (M->nnz > 0)
        TSG_CUDA(cudaMemcpyAsync(d->ci, M->columnindex, (size_t)M->nnz * sizeof(int), cudaMemcpyHostToDevice,
                                 ctx->stream));
    return TSG_OK;
}

void free_pattern(tsg_context *ctx, DevPattern *d)
{
    tsg_release(ctx, d->rp);
    tsg_release(ctx, d->ci);
}

int tile_dim(int n) { return (n + TSG_BS - 1) / TSG_BS; }

// row, inner and column orders of A*B by signatures: rows by A's rows,
// columns by B's columns, the inner axis by A's columns with B's rows
int signature_plan(const SMatrix *A, const SMatrix *B, bool same, ReorderInfo *info)
{
    tsg_context *ctx = tsg_dropin_context();
    if (!ctx)
        return -2;
    double t0 = now_ms();
    DevPattern a, b;
    Sig a_row, a_col, b_row, b_col;
    int st = upload_pattern(ctx, A, &a);
    if (st == TSG_OK && !same)
        st = upload_pattern(ctx, B, &b);
    const DevPattern &bb = same ? a : b;
    if (st == TSG_OK)
        st = row_signatures(ctx, a.m, a.rp, a.ci, &a_row);
    if (st == TSG_OK)
        st = col_signatures(ctx, a.m, a.n, a.nnz, a.rp, a.ci, &a_col);
    if (st == TSG_OK && !same)
        st = row_signatures(ctx, bb.m, bb.rp, bb.ci, &b_row);
    if (st == TSG_OK && !same)
        st = col_signatures(ctx, bb.m, bb.n, bb.nnz, bb.rp, bb.ci, &b_col);
    if (st == TSG_OK)
        st = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? TSG_OK : TSG_ERR_CUDA;
    info->signature_time_ms = now_ms() - t0;
    const Sig &br = same ? a_row : b_row, &bc = same ? a_col : b_col;
    t0 = now_ms();
    const int comb = std::max(tile_dim(A->m), tile_dim(B->n));
    if (st == TSG_OK)
        st = order_by_signature(ctx, a_row, nullptr, tile_dim(A->n), &info->row_perm);
    const int st_row = st;
    if (st == TSG_OK)
        st = order_by_signature(ctx, a_col, &br, comb, &info->inner_perm);
    const int st_inner = st;
    if (st == TSG_OK)
        st = order_by_signature(ctx, bc, nullptr, tile_dim(B->m), &info->col_perm);
    info->sort_time_ms = now_ms() - t0;
    sig_free(ctx, &a_row);
    sig_free(ctx, &a_col);
    free_pattern(ctx, &a);
    if (!same)
    {
        sig_free(ctx, &b_row);
        sig_free(ctx, &b_col);
        free_pattern(ctx, &b);
    }
    if (st_row != TSG_OK)
        return -2;
    if (st_inner != TSG_OK)
        return -3;
    return st == TSG_OK ? 0 : -4;
}

// ---------------------------------------------------------------------------
// symmetric path: rows' tile sets on the host
// ---------------------------------------------------------------------------
struct TileSets
{
    std::vector<int> ptr, idx, count, degree;
};

void row_tile_sets(const SMatrix *M, TileSets *s)
{
    const int m = M->m;
    s->ptr.assign((size_t)m + 1, 0);
    s->count.assign(m, 0);
    s->degree.assign(m, 0);
    std::vector<std::vector<int>> lists(m);
    for (int i = 0; i < m; i++)
    {
        auto &v = lists[i];
        for (int p = M->rowpointer[i]; p < M->rowpointer[i + 1]; p++)
            v.push_back(M->columnindex[p] / TSG_BS);
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        s->count[i] = (int)v.size();
        s->degree[i] = M->rowpointer[i + 1] - M->rowpointer[i];
        s->ptr[i + 1] = s->ptr[i] + (int)v.size();
    }
    s->idx.resize(s->ptr[m]);
    for (int i = 0; i < m; i++)
        std::copy(lists[i].begin(), lists[i].end(), s->idx.begin() + s->ptr[i]);
}

// tiles of M in its natural order: distinct tile columns per tile row
long long natural_tiles(const TileSets &s, int m)
{
    long long total = 0;
    std::vector<int> seen;
    for (int tr = 0; tr < tile_dim(m); tr++)
    {
        seen.clear();
        for (int i = tr * TSG_BS; i < std::min(m, tr * TSG_BS + TSG_BS); i++)
            seen.insert(seen.end(), s.idx.begin() + s.ptr[i], s.idx.begin() + s.ptr[i + 1]);
        std::sort(seen.begin(), seen.end());
        total += std::unique(seen.begin(), seen.end()) - seen.begin();
    }
    return total;
}

int shared_tiles(const TileSets &s, int a, int b)
{
    int pa = s.ptr[a], pb = s.ptr[b], k = 0;
    while (pa < s.ptr[a + 1] && pb < s.ptr[b + 1])
    {
        const int va = s.idx[pa], vb = s.idx[pb];
        k += va == vb;
        pa += va <= vb;
        pb += vb <= va;
    }
    return k;
}

// RCM with (tile count, degree, id) seeds and neighbour order, each
// component reversed in place, then the windowed refinement
void rcm_refined(const SMatrix *M, const TileSets &s, int window, std::vector<int> *order, double *sort_ms,
                 double *aff_ms, double *ref_ms)
{
    const int n = M->m;
    auto before = [&](int a, int b) {
        if (s.count[a] != s.count[b])
            return s.count[a] < s.count[b];
        if (s.degree[a] != s.degree[b])
            return s.degree[a] < s.degree[b];
        return a < b;
    };
    double t0 = now_ms();
    std::vector<int> seeds(n);
    std::iota(seeds.begin(), seeds.end(), 0);
    std::sort(seeds.begin(), seeds.end(), before);
    *sort_ms += now_ms() - t0;
    t0 = now_ms();
    std::vector<char> seen(n, 0);
    std::vector<int> queue, next;
    order->clear();
    order->reserve(n);
    for (int sd : seeds)
    {
        if (seen[sd])
            continue;
        seen[sd] = 1;
        queue.assign(1, sd);
        for (size_t h = 0; h < queue.size(); h++)
        {
            const int v = queue[h];
            next.clear();
            for (int p = M->rowpointer[v]; p < M->rowpointer[v + 1]; p++)
            {
                const int u = M->columnindex[p];
                if (u >= 0 && u < n && !seen[u])
                {
                    seen[u] = 1;
                    next.push_back(u);
                }
            }
            std::sort(next.begin(), next.end(), before);
            queue.insert(queue.end(), next.begin(), next.end());
        }
        order->insert(order->end(), queue.rbegin(), queue.rend());
    }
    *aff_ms += now_ms() - t0;
    t0 = now_ms();
    // greedy: each position takes, from the rest of its window, the row
    // scoring best against its predecessor (16 shared tiles - tile count gap)
    auto score = [&](int a, int b) { return shared_tiles(s, a, b) * 16 - abs(s.count[a] - s.count[b]); };
    for (int w0 = 0; window > 1 && w0 < n; w0 += window)
    {
        const int w1 = std::min(n, w0 + window);
        for (int pos = w0 + 1; pos < w1; pos++)
        {
            const int prev = (*order)[pos - 1];
            int best = pos, best_score = score(prev, (*order)[pos]);
            for (int c = pos + 1; c < w1; c++)
            {
                const int sc = score(prev, (*order)[c]);
                if (sc > best_score)
                {
                    best_score = sc;
                    best = c;
                }
            }
            std::swap((*order)[pos], (*order)[best]);
        }
    }
    *ref_ms += now_ms() - t0;
}

// one packing window [w0, w1) of the natural order: groups of up to 16
// rows, each seeded by the first row left, grown by the best-scoring row
void pack_window(const TileSets &s, int w0, int w1, std::vector<int> &group_mark, int *out)
{
    const int len = w1 - w0;
    std::vector<char> used(len, 0);
    int left = len, o = 0;
    std::vector<int> marked;
    while (left > 0)
    {
        for (int t : marked)
            group_mark[t] = 0;
        marked.clear();
        int seed = 0;
        while (used[seed])
            seed++;
        used[seed] = 1;
        left--;
        const int seed_id = w0 + seed;
        out[o++] = seed_id;
        auto mark = [&](int id) {
            for (int p = s.ptr[id]; p < s.ptr[id + 1]; p++)
                if (!group_mark[s.idx[p]])
                {
                    group_mark[s.idx[p]] = 1;
                    marked.push_back(s.idx[p]);
                }
        };
        mark(seed_id);
        for (int g = 1; g < TSG_BS && left > 0; g++)
        {
            int best = -1, best_score = INT_MIN;
            for (int i = 0; i < len; i++)
            {
                if (used[i])
                    continue;
                const int id = w0 + i;
                int overlap = 0;
                for (int p = s.ptr[id]; p < s.ptr[id + 1]; p++)
                    overlap += group_mark[s.idx[p]];
                const int added = s.count[id] - overlap;
                const int sc = overlap * 96 - added * 64 - (abs(id - seed_id) / TSG_BS) * 48;
                if (sc > best_score)
                {
                    best_score = sc;
                    best = i;
                }
            }
            used[best] = 1;
            left--;
            out[o++] = w0 + best;
            mark(w0 + best);
        }
    }
    for (int t : marked)
        group_mark[t] = 0;
}

void banded_pack(const TileSets &s, int n, int window, std::vector<int> *order)
{
    order->resize(n);
    std::iota(order->begin(), order->end(), 0);
    if (window <= TSG_BS || n == 0)
        return;
    const int windows = (n + window - 1) / window;
    const int tiles = tile_dim(n);
    int threads = (int)std::thread::hardware_concurrency();
    threads = std::max(1, std::min(threads, std::min(16, windows)));
    auto work = [&](int t) {
        std::vector<int> mark((size_t)std::max(tiles, 1), 0);
        for (int w = t; w < windows; w += threads)
        {
            const int w0 = w * window, w1 = std::min(n, w0 + window);
            pack_window(s, w0, w1, mark, order->data() + w0);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; t++)
        pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool)
        th.join();
}

int pack_window_for(int n) { return n <= 50000 ? 32 : (n <= 1000000 ? 64 : 32); }

// ---------------------------------------------------------------------------
// estimates and the risk guard
// ---------------------------------------------------------------------------
void plan_estimates(const SMatrix *A, const SMatrix *B, bool ab, ReorderInfo *info)
{
    const double t0 = now_ms();
    info->input_tiles_A_before = tsg_estimate_input_tiles(A, nullptr, nullptr);
    info->input_tiles_B_before = ab ? tsg_estimate_input_tiles(B, nullptr, nullptr) : info->input_tiles_A_before;
    info->input_tiles_A_after = tsg_estimate_input_tiles(A, &info->row_perm, &info->inner_perm);
    info->input_tiles_B_after = tsg_estimate_input_tiles(ab ? B : A, &info->inner_perm, &info->col_perm);
    info->estimated_c_tiles_before = tsg_estimate_c_tiles(A, ab ? B : A, nullptr, nullptr, nullptr, !ab);
    info->estimated_c_tiles_after =
        tsg_estimate_c_tiles(A, ab ? B : A, &info->row_perm, &info->inner_perm, &info->col_perm, !ab);
    info->proxy_time_ms += now_ms() - t0;
}

bool env_is_1(const char *name)
{
    const char *v = getenv(name);
    return v && strcmp(v, "1") == 0;
}

int identity_axes(ReorderInfo *info, int rows, int inner, int cols)
{
    std::vector<int> id((size_t)std::max(std::max(rows, inner), std::max(cols, 1)));
    std::iota(id.begin(), id.end(), 0);
    return (tsg_axis_from_order(&info->row_perm, id.data(), rows) || tsg_axis_from_order(&info->inner_perm, id.data(), inner) ||
            tsg_axis_from_order(&info->col_perm, id.data(), cols))
               ? -1
               : 0;
}

void to_identity(ReorderInfo *info, int rows, int inner, int cols, const char *mode, const char *reason)
{
    identity_axes(info, rows, inner, cols);
    info->guard_degraded_to_identity = 1;
    info->structural_conservative = 1;
    info->shared_symmetric_csr = 0;
    tsg_info_text(info->mode, sizeof(info->mode), mode);
    tsg_info_text(info->risk_reason, sizeof(info->risk_reason), reason);
    info->input_tiles_A_after = info->input_tiles_A_before;
    info->input_tiles_B_after = info->input_tiles_B_before;
    info->estimated_c_tiles_after = info->estimated_c_tiles_before;
}

double ratio(long long after, long long before) { return before <= 0 ? 1.0 : (double)after / (double)before; }

// identity when the estimated tiles grow (input growth limit: 0.95 of C for
// AA, 0.98 for A*B), or when a small product gains nothing
void risk_guard(ReorderInfo *info, int rows, int inner, int cols, double input_growth_c_limit)
{
    const double ra = ratio(info->input_tiles_A_after, info->input_tiles_A_before);
    const double rb = ratio(info->input_tiles_B_after, info->input_tiles_B_before);
    const int max_dim = std::max(rows, std::max(inner, cols));
    info->risk_input_tile_ratio = ra > rb ? ra : rb;
    info->risk_c_tile_ratio = ratio(info->estimated_c_tiles_after, info->estimated_c_tiles_before);
    const double ri = info->risk_input_tile_ratio, rc = info->risk_c_tile_ratio;
    const char *why = nullptr;
    if (env_is_1("TASA_FORCE_ACTIVE"))
    {
        info->structural_conservative = 0;
        tsg_info_text(info->risk_reason, sizeof(info->risk_reason), "accepted_force");
        return;
    }
    if (rc > 1.15 && ri > 1.10)
        why = "c_and_input_tile_growth";
    else if (rc > 1.20)
        why = "c_tile_growth";
    else if (ri > 1.25 && rc > input_growth_c_limit)
        why = "input_tile_growth";
    else if (max_dim <= 50000 && rc > 0.98 && ri > 0.95)
        why = "small_no_tile_gain";
    if (why)
    {
        to_identity(info, rows, inner, cols, "conservative_identity", why);
        return;
    }
    info->structural_conservative = 0;
    tsg_info_text(info->risk_reason, sizeof(info->risk_reason), "accepted");
}

void begin_plan(ReorderInfo *info, int n, const char *mode)
{
    reorder_info_destroy(info);
    info->enabled = 1;
    info->n = n;
    info->guard_degraded_to_identity = 0;
    tsg_info_text(info->mode, sizeof(info->mode), mode);
    tsg_info_text(info->risk_reason, sizeof(info->risk_reason), "pending");
}

// A*A (src/reorder.h:2153-2405)
int plan_aa(const SMatrix *M, ReorderInfo *info)
{
    if (M->m != M->n)
        return -1;
    const int n = M->m;
    begin_plan(info, n, "active");
    if (!M->isSymmetric)
    {
        const int st = signature_plan(M, M, true, info);
        if (st != 0)
            return st;
        plan_estimates(M, M, false, info);
        tsg_info_text(info->mode, sizeof(info->mode), "active_general");
        risk_guard(info, n, n, n, 0.95);
        return 0;
    }
    double t0 = now_ms();
    TileSets s;
    row_tile_sets(M, &s);
    info->signature_time_ms = now_ms() - t0;
    std::vector<int> order;
    if (n <= 50000)
    {
        const long long nat = natural_tiles(s, n);
        const int td = tile_dim(n);
        if ((td > 0 ? (double)nat / td : 0.0) < 32.0)
        {
            info->local_refine_window = 0;
            if (identity_axes(info, n, n, n))
                return -2;
            info->input_tiles_A_before = info->input_tiles_B_before = nat;
            info->input_tiles_A_after = info->input_tiles_B_after = nat;
            info->estimated_c_tiles_before = info->estimated_c_tiles_after = 0;
            to_identity(info, n, n, n, "identity_narrow_tiles", "natural_tile_rows_compact");
            info->risk_input_tile_ratio = 1.0;
            info->risk_c_tile_ratio = 1.0;
            return 0;
        }
        info->local_refine_window = 32;
        rcm_refined(M, s, 32, &order, &info->sort_time_ms, &info->affinity_time_ms, &info->local_refine_time_ms);
    }
    else
    {
        info->local_refine_window = pack_window_for(n);
        t0 = now_ms();
        banded_pack(s, n, info->local_refine_window, &order);
        info->local_refine_time_ms += now_ms() - t0;
    }
    if (tsg_axis_from_order(&info->inner_perm, order.data(), n))
        return -2;
    if (tsg_axis_copy(&info->row_perm, &info->inner_perm))
        return -3;
    if (tsg_axis_copy(&info->col_perm, &info->inner_perm))
        return -4;
    plan_estimates(M, M, false, info);
    tsg_info_text(info->mode, sizeof(info->mode), "active_symmetric");
    risk_guard(info, n, n, n, 0.95);
    if (!info->guard_degraded_to_identity)
        info->shared_symmetric_csr = 1;
    return 0;
}

// A*B (src/reorder.h:2046-2135)
int plan_ab(const SMatrix *A, const SMatrix *B, ReorderInfo *info)
{
    if (A->n != B->m)
        return -1;
    const int rows = A->m, inner = A->n, cols = B->n;
    if (env_is_1("TASA_AB_SHARED_SYM") && A->m == A->n && B->m == B->n && A->m == B->m && A->isSymmetric &&
        B->isSymmetric)
    {
        const int st = plan_aa(A, info);
        if (st != 0)
            return st;
        info->shared_symmetric_csr = 0;
        plan_estimates(A, B, true, info);
        tsg_info_text(info->mode, sizeof(info->mode), "active_ab_shared_symmetric");
        risk_guard(info, rows, inner, cols, 0.98);
        if (!info->guard_degraded_to_identity)
            tsg_info_text(info->mode, sizeof(info->mode), "active_ab_shared_symmetric");
        return 0;
    }
    begin_plan(info, inner, "active_ab");
    info->shared_symmetric_csr = 0;
    const int st = signature_plan(A, B, false, info);
    if (st != 0)
        return st;
    plan_estimates(A, B, true, info);
    risk_guard(info, rows, inner, cols, 0.98);
    if (!info->guard_degraded_to_identity)
        tsg_info_text(info->mode, sizeof(info->mode), "active_ab");
    return 0;
}

} // namespace

extern "C" int build_reorder_plan(const ReorderProblem *problem, ReorderInfo *info)
{
    if (!problem || !info || !problem->matrixA)
        return -1;
    switch (problem->kind)
    {
    case REORDER_PROBLEM_AA:
        return plan_aa(problem->matrixA, info);
    case REORDER_PROBLEM_AAT:
    {
        const SMatrix *A = problem->matrixA, *AT = problem->matrixB;
        if (!AT)
            return -3;
        if (A->n != AT->m || A->m != AT->n)
            return -2;
        const int st = plan_ab(A, AT, info);
        if (st != 0)
            return st;
        if (!info->guard_degraded_to_identity)
            tsg_info_text(info->mode, sizeof(info->mode), "active_aat");
        return 0;
    }
    case REORDER_PROBLEM_AB:
        if (!problem->matrixB)
            return -3;
        return plan_ab(problem->matrixA, problem->matrixB, info);
    default:
        return -2;
    }
}
