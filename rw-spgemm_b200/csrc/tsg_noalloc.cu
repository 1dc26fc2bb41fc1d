// Tiles -> CSR without any allocation: the row-pointer scan keeps its
// per-block partial sums in a fixed file-scope device array instead of in
// memory taken from the context's stream-ordered pool.
//
// The work is the same as tsg_tiled_to_csr (tsg_convert.cu): row lengths of C
// (k_t2c_rowlen), an exclusive scan of them into rowptr, then the copy of
// every tile row's entries into (colidx, val) (k_t2c_fill).  Only the scan
// differs: a reduce-then-scan whose partials live in g_t2c_partials.
//
// Limits and sharing:
//  - the scan covers SCAN_TILE rows per block and the scratch holds
//    NA_MAX_PARTIALS block sums, so C may have at most
//    NA_MAX_PARTIALS * SCAN_TILE = 33,554,432 rows; larger C is rejected
//    with TSG_ERR_INVALID before anything is launched;
//  - nothing in the scratch needs to start at zero: each call writes every
//    partial it later reads (reduce kernel, then the partial scan, then the
//    apply kernel, in stream order);
//  - the scratch is one array per device, shared by every context, stream and
//    thread of the process: two calls that can run at the same time on one
//    device (different streams without an event between them, or different
//    host threads) race on it and must be serialised by the caller;
//  - the scratch's address is looked up with cudaGetSymbolAddress (with the
//    device current) when a context is created on the device
//    (tsg_noalloc_prepare), so the conversion itself makes no runtime call
//    but its launches and may be captured in a graph.
#include <mutex>

#include "tsg_internal.h"

#define SCAN_THREADS 1024
#define SCAN_ITEMS 8
#define SCAN_TILE (SCAN_THREADS * SCAN_ITEMS)
#define NA_MAX_PARTIALS 4096
#define NA_PART_ITEMS (NA_MAX_PARTIALS / SCAN_THREADS)
#define NA_MAX_DEVICES 64

static __device__ __align__(256) long long g_t2c_partials[NA_MAX_PARTIALS];

// Row lengths and the final copy: the kernels of tsg_tiled_to_csr.
__global__ void k_t2c_rowlen(int m, int tilem, const int *__restrict__ tile_ptr, const int *__restrict__ tnnz,
                             const unsigned char *__restrict__ Ptr, int *__restrict__ rowlen);
__global__ void k_t2c_fill(int m, int tilem, const int *__restrict__ tile_ptr, const int *__restrict__ tile_col,
                           const int *__restrict__ tnnz, const unsigned char *__restrict__ Ptr,
                           const unsigned char *__restrict__ Col, const double *__restrict__ Val,
                           const int *__restrict__ rowptr, int *__restrict__ ccol, double *__restrict__ cval);

__device__ __forceinline__ long long na_warp_incl(long long v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
    {
        long long o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d)
            v += o;
    }
    return v;
}

// Exclusive scan of one value per thread over SCAN_THREADS threads.
__device__ __forceinline__ long long na_block_excl(long long v, long long *s_warp, long long *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long incl = na_warp_incl(v);
    if (lane == 31)
        s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0)
    {
        long long w = s_warp[lane];
        long long wi = na_warp_incl(w);
        s_warp[lane] = wi - w;
        if (lane == 31)
            s_warp[32] = wi;
    }
    __syncthreads();
    const long long res = incl - v + s_warp[warp];
    *total = s_warp[32];
    return res;
}

// partial[b] = sum of rowlen[b * SCAN_TILE .. (b + 1) * SCAN_TILE)
__global__ void __launch_bounds__(SCAN_THREADS) k_na_reduce(const int *__restrict__ rowlen, int m,
                                                            long long *__restrict__ partial)
{
    __shared__ long long s_warp[33];
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    long long sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
        if (base + k < m)
            sum += rowlen[base + k];
    long long tot;
    na_block_excl(sum, s_warp, &tot);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = tot;
}

// One block: exclusive scan of partial[0 .. nb) in place; rowptr[m] = total.
__global__ void __launch_bounds__(SCAN_THREADS) k_na_partials(long long *__restrict__ partial, int nb, int m,
                                                              int *__restrict__ rowptr)
{
    __shared__ long long s_warp[33];
    const int base = threadIdx.x * NA_PART_ITEMS;
    long long v[NA_PART_ITEMS], sum = 0;
#pragma unroll
    for (int k = 0; k < NA_PART_ITEMS; k++)
    {
        v[k] = base + k < nb ? partial[base + k] : 0;
        sum += v[k];
    }
    long long tot;
    long long run = na_block_excl(sum, s_warp, &tot);
#pragma unroll
    for (int k = 0; k < NA_PART_ITEMS; k++)
    {
        if (base + k < nb)
            partial[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0)
        rowptr[m] = (int)tot;
}

// Exclusive scan of each block's rows (in place) plus the block's offset.
__global__ void __launch_bounds__(SCAN_THREADS) k_na_apply(int *rowptr, int m, const long long *__restrict__ partial)
{
    __shared__ long long s_warp[33];
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    long long v[SCAN_ITEMS], sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
    {
        v[k] = base + k < m ? rowptr[base + k] : 0;
        sum += v[k];
    }
    long long tot;
    long long run = na_block_excl(sum, s_warp, &tot) + partial[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
    {
        if (base + k < m)
            rowptr[base + k] = (int)run;
        run += v[k];
    }
}

// Scratch address per device, looked up with that device current: at every
// context creation (refresh: a cudaDeviceReset since the last lookup moves
// it), and on a conversion only if no context ever looked it up.
static std::mutex g_na_mutex;
static long long *g_na_scratch[NA_MAX_DEVICES];

static int na_lookup(int device, bool refresh)
{
    if (device < 0 || device >= NA_MAX_DEVICES)
        return tsg_set_error(TSG_ERR_INVALID, "tsg_tiled_to_csr_noalloc: device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (refresh || !g_na_scratch[device])
    {
        int cur = -1;
        TSG_CUDA(cudaGetDevice(&cur));
        if (cur != device)
            TSG_CUDA(cudaSetDevice(device));
        long long *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_t2c_partials);
        if (cur != device)
            cudaSetDevice(cur);
        if (e != cudaSuccess || !ptr)
            return tsg_set_error(TSG_ERR_CUDA, "tsg_tiled_to_csr_noalloc: cudaGetSymbolAddress failed: %s",
                                 cudaGetErrorString(e));
        g_na_scratch[device] = ptr;
    }
    return TSG_OK;
}

int tsg_noalloc_prepare(int device) { return na_lookup(device, true); }

static int na_scratch(int device, long long **out)
{
    TSG_TRY(na_lookup(device, false));
    *out = g_na_scratch[device];
    return TSG_OK;
}

extern "C" int tsg_tiled_to_csr_noalloc(tsg_context *ctx, const tsg_tiled *C, int *d_rowptr, int *d_colidx,
                                        double *d_val)
{
    if (!ctx || !C || !d_rowptr)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    const int m = C->m, tilem = C->tilem;
    if (m < 0 || (long long)m > (long long)NA_MAX_PARTIALS * SCAN_TILE)
        return tsg_set_error(TSG_ERR_INVALID,
                             "tsg_tiled_to_csr_noalloc: C has %d rows; the fixed scratch covers at most %lld rows "
                             "(use tsg_tiled_to_csr)",
                             m, (long long)NA_MAX_PARTIALS * SCAN_TILE);
    if (C->nnz > 0 && (!d_colidx || !d_val))
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    long long *partial = nullptr;
    TSG_TRY(na_scratch(ctx->device, &partial));
    if (m == 0)
    {
        TSG_CUDA(cudaMemsetAsync(d_rowptr, 0, sizeof(int), ctx->stream));
        return TSG_OK;
    }
    const int nb = (m + SCAN_TILE - 1) / SCAN_TILE;
    k_t2c_rowlen<<<tsg_blocks((long long)tilem * 16, 256), 256, 0, ctx->stream>>>(m, tilem, C->tile_ptr, C->tile_nnz,
                                                                                 C->tile_csr_Ptr, d_rowptr);
    TSG_LAUNCH_CHECK();
    k_na_reduce<<<nb, SCAN_THREADS, 0, ctx->stream>>>(d_rowptr, m, partial);
    TSG_LAUNCH_CHECK();
    k_na_partials<<<1, SCAN_THREADS, 0, ctx->stream>>>(partial, nb, m, d_rowptr);
    TSG_LAUNCH_CHECK();
    k_na_apply<<<nb, SCAN_THREADS, 0, ctx->stream>>>(d_rowptr, m, partial);
    TSG_LAUNCH_CHECK();
    k_t2c_fill<<<tsg_blocks((long long)tilem * 16, 256), 256, 0, ctx->stream>>>(
        m, tilem, C->tile_ptr, C->tile_columnidx, C->tile_nnz, C->tile_csr_Ptr, C->tile_csr_Col, C->tile_csr_Value,
        d_rowptr, d_colidx, d_val);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}
