// Device-wide scans, sorts, CSR validation and small reductions.
#include <stdarg.h>
#include <string.h>

#include <cub/device/device_radix_sort.cuh>

#include "tsg_internal.h"

static thread_local char g_last_error[512] = "";

int tsg_set_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

extern "C" const char *tsg_last_error(void) { return g_last_error; }

// ---------------------------------------------------------------------------
// Exclusive scan: reduce-then-scan over blocks of SCAN_ITEMS * SCAN_THREADS.
// ---------------------------------------------------------------------------
#define SCAN_THREADS 1024
#define SCAN_ITEMS 8
#define SCAN_TILE (SCAN_THREADS * SCAN_ITEMS)

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
    {
        T o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d)
            v += o;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread (SCAN_THREADS threads).
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *s_warp, T *block_total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = warp_incl_scan(v);
    if (lane == 31)
        s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0)
    {
        T w = s_warp[lane];
        T wi = warp_incl_scan(w);
        s_warp[lane] = wi - w;
        if (lane == 31)
            s_warp[32] = wi;
    }
    __syncthreads();
    T res = incl - v + s_warp[warp];
    *block_total = s_warp[32];
    __syncthreads();
    return res;
}

template <typename TIn>
__global__ void k_scan_reduce(const TIn *__restrict__ in, long long n, long long *__restrict__ partial)
{
    __shared__ long long s_warp[33];
    long long base = (long long)blockIdx.x * SCAN_TILE;
    long long sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
    {
        long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        if (i < n)
            sum += (long long)in[i];
    }
    long long tot;
    block_excl_scan<long long>(sum, s_warp, &tot);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = tot;
}

// Exclusive scan of each tile; offset[blockIdx] added (nullptr = 0).  Writes
// out[n] = grand total from the last block.  in/out may alias.
template <typename TIn, typename TOut>
__global__ void k_scan_apply(const TIn *in, long long n, const long long *__restrict__ offset,
                             TOut *out, long long *total_out)
{
    __shared__ long long s_warp[33];
    long long base = (long long)blockIdx.x * SCAN_TILE;
    long long v[SCAN_ITEMS];
    long long sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
    {
        long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        v[k] = i < n ? (long long)in[i] : 0;
        sum += v[k];
    }
    long long tot;
    long long run = block_excl_scan<long long>(sum, s_warp, &tot);
    long long off = offset ? offset[blockIdx.x] : 0;
    run += off;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
    {
        long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        if (i < n)
            out[i] = (TOut)run;
        run += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == SCAN_THREADS - 1)
    {
        out[n] = (TOut)(off + tot);
        if (total_out)
            *total_out = off + tot;
    }
}

// In-place exclusive scan of n long longs (n <= SCAN_TILE per level).
static int scan_partials(tsg_context *ctx, long long *p, long long nb)
{
    if (nb <= SCAN_TILE)
    {
        k_scan_apply<long long, long long><<<1, SCAN_THREADS, 0, ctx->stream>>>(p, nb, nullptr, p, nullptr);
        TSG_LAUNCH_CHECK();
        return TSG_OK;
    }
    long long nb2 = (nb + SCAN_TILE - 1) / SCAN_TILE;
    long long *p2;
    TSG_TRY(tsg_alloc(ctx, &p2, (size_t)nb2 + 1));
    k_scan_reduce<long long><<<(unsigned)nb2, SCAN_THREADS, 0, ctx->stream>>>(p, nb, p2);
    TSG_LAUNCH_CHECK();
    TSG_TRY(scan_partials(ctx, p2, nb2));
    k_scan_apply<long long, long long><<<(unsigned)nb2, SCAN_THREADS, 0, ctx->stream>>>(p, nb, p2, p, nullptr);
    TSG_LAUNCH_CHECK();
    tsg_release(ctx, p2);
    return TSG_OK;
}

int tsg_scan_counts(tsg_context *ctx, const int *in, int *out, long long n, long long *total)
{
    long long *d_total = nullptr;
    if (total)
        TSG_TRY(tsg_alloc(ctx, &d_total, 1));
    if (n <= SCAN_TILE)
    {
        k_scan_apply<int, int><<<1, SCAN_THREADS, 0, ctx->stream>>>(in, n, nullptr, out, d_total);
        TSG_LAUNCH_CHECK();
    }
    else
    {
        long long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
        long long *partial;
        TSG_TRY(tsg_alloc(ctx, &partial, (size_t)nb + 1));
        k_scan_reduce<int><<<(unsigned)nb, SCAN_THREADS, 0, ctx->stream>>>(in, n, partial);
        TSG_LAUNCH_CHECK();
        TSG_TRY(scan_partials(ctx, partial, nb));
        k_scan_apply<int, int><<<(unsigned)nb, SCAN_THREADS, 0, ctx->stream>>>(in, n, partial, out, d_total);
        TSG_LAUNCH_CHECK();
        tsg_release(ctx, partial);
    }
    if (total)
    {
        TSG_CUDA(cudaMemcpyAsync(ctx->h_pinned, d_total, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
        tsg_release(ctx, d_total);
        TSG_CUDA(cudaStreamSynchronize(ctx->stream));
        *total = ctx->h_pinned[0];
        if (*total > 2147483647LL)
            return tsg_set_error(TSG_ERR_OVERFLOW, "scan total %lld exceeds 32-bit offsets", *total);
    }
    return TSG_OK;
}

int tsg_read_int(tsg_context *ctx, const int *dptr, long long *out)
{
    int *h = (int *)ctx->h_pinned;
    TSG_CUDA(cudaMemcpyAsync(h, dptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = h[0];
    return TSG_OK;
}

// ---------------------------------------------------------------------------
// Stable radix sort of (key, int) pairs.
// ---------------------------------------------------------------------------
template <typename K>
static int sort_pairs(tsg_context *ctx, K *keys, int *vals, long long n, int end_bit)
{
    if (n <= 1)
        return TSG_OK;
    K *k2;
    int *v2;
    TSG_TRY(tsg_alloc(ctx, &k2, (size_t)n));
    TSG_TRY(tsg_alloc(ctx, &v2, (size_t)n));
    cub::DoubleBuffer<K> dk(keys, k2);
    cub::DoubleBuffer<int> dv(vals, v2);
    size_t temp = 0;
    TSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, dk, dv, (int)n, 0, end_bit, ctx->stream));
    char *d_temp;
    TSG_TRY(tsg_alloc(ctx, &d_temp, temp));
    TSG_CUDA(cub::DeviceRadixSort::SortPairs(d_temp, temp, dk, dv, (int)n, 0, end_bit, ctx->stream));
    if (dk.Current() != keys)
        TSG_CUDA(cudaMemcpyAsync(keys, dk.Current(), (size_t)n * sizeof(K), cudaMemcpyDeviceToDevice, ctx->stream));
    if (dv.Current() != vals)
        TSG_CUDA(cudaMemcpyAsync(vals, dv.Current(), (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
    tsg_release(ctx, d_temp);
    tsg_release(ctx, k2);
    tsg_release(ctx, v2);
    return TSG_OK;
}

int tsg_sort_pairs_u64(tsg_context *ctx, unsigned long long *keys, int *vals, long long n, int end_bit)
{
    return sort_pairs<unsigned long long>(ctx, keys, vals, n, end_bit);
}

int tsg_sort_pairs_u32(tsg_context *ctx, unsigned int *keys, int *vals, long long n, int end_bit)
{
    return sort_pairs<unsigned int>(ctx, keys, vals, n, end_bit);
}

// ---------------------------------------------------------------------------
// CSR validation: one warp per row.
// ---------------------------------------------------------------------------
__global__ void k_check_csr(int m, int n, int nnz, const int *__restrict__ rowptr,
                            const int *__restrict__ col, int *__restrict__ err)
{
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= m)
        return;
    const int r = (int)gw;
    int s = rowptr[r], e = rowptr[r + 1];
    int bad = 0;
    if (r == 0 && s != 0)
        bad |= 1;
    if (r == m - 1 && e != nnz)
        bad |= 1;
    if (s < 0 || e < s || e > nnz)
        bad |= 1;
    if (!bad)
    {
        for (int p = s + lane; p < e; p += 32)
        {
            int c = col[p];
            if (c < 0 || c >= n)
                bad |= 2;
            else if (p + 1 < e && col[p + 1] <= c)
                bad |= 4;
        }
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0 && bad)
        atomicOr(err, bad);
}

int tsg_check_csr(tsg_context *ctx, int m, int n, int nnz, const int *rowptr, const int *colidx)
{
    if (m < 0 || n < 0 || nnz < 0)
        return tsg_set_error(TSG_ERR_INVALID, "negative CSR dimension");
    if (m == 0)
        return nnz == 0 ? TSG_OK : tsg_set_error(TSG_ERR_INPUT, "m = 0 with nnz > 0");
    int *d_err;
    TSG_TRY(tsg_alloc(ctx, &d_err, 1));
    TSG_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream));
    k_check_csr<<<tsg_blocks((long long)m * 32, 256), 256, 0, ctx->stream>>>(m, n, nnz, rowptr, colidx, d_err);
    TSG_LAUNCH_CHECK();
    long long err;
    TSG_TRY(tsg_read_int(ctx, d_err, &err));
    tsg_release(ctx, d_err);
    if (err & 1)
        return tsg_set_error(TSG_ERR_INPUT, "CSR row pointer malformed (rowptr[0]=0, monotone, rowptr[m]=nnz)");
    if (err & 2)
        return tsg_set_error(TSG_ERR_INPUT, "CSR column index out of range [0, %d)", n);
    if (err & 4)
        return tsg_set_error(TSG_ERR_INPUT, "CSR rows must be sorted by strictly increasing column");
    return TSG_OK;
}

// ---------------------------------------------------------------------------
// nnzCub = sum over A nonzeros of |B row|.
// ---------------------------------------------------------------------------
__global__ void k_count_products(long long nnzA, const int *__restrict__ a_col,
                                 const int *__restrict__ b_rowptr, unsigned long long *out)
{
    unsigned long long s = 0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < nnzA;
         p += (long long)gridDim.x * blockDim.x)
    {
        int k = a_col[p];
        s += (unsigned long long)(b_rowptr[k + 1] - b_rowptr[k]);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, d);
    if ((threadIdx.x & 31) == 0 && s)
        atomicAdd(out, s);
}

int tsg_count_products_dev(tsg_context *ctx, int nnzA, const int *a_col, const int *b_rowptr, long long *out)
{
    unsigned long long *d;
    TSG_TRY(tsg_alloc(ctx, &d, 1));
    TSG_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), ctx->stream));
    if (nnzA > 0)
    {
        unsigned blocks = tsg_blocks(nnzA, 256);
        unsigned cap = (unsigned)ctx->num_sms * 8;
        k_count_products<<<blocks < cap ? blocks : cap, 256, 0, ctx->stream>>>(nnzA, a_col, b_rowptr, d);
        TSG_LAUNCH_CHECK();
    }
    TSG_CUDA(cudaMemcpyAsync(ctx->h_pinned, d, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = ctx->h_pinned[0];
    tsg_release(ctx, d);
    return TSG_OK;
}
