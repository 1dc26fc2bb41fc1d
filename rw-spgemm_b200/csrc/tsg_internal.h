// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "tilespgemm_b200.h"

#define TSG_BS 16
// SPA schedule: C values per tile (on average) from which the numeric step's
// tile kernel is faster than the sparse accumulator (the default threshold)
#define TSG_SPA_DENSE_DEFAULT 64

struct tsg_context
{
    int device;
    int num_sms;
    cudaStream_t stream;
    int own_stream;
    int timing;
    cudaEvent_t ev[8];
    long long *h_pinned; // small pinned buffer for scalar read-backs
    long long launches;  // kernels this library launched on the context
    int sched;           // TSG_SCHED_TILES / TSG_SCHED_ROWS for steps 2-3
    int seg_tiles;       // row schedule: C tiles per work item (8 or 16)
    int acc_cap;         // row schedule: FP64 accumulator slots per half-warp
    int fuse12;          // step-1 emit fused with step 2 for narrow tile rows
    cudaStream_t copy_stream; // device-to-host copies overlapping compute (created on first use)
    cudaEvent_t copy_ev;      // orders a chunk's copy after its fill
    int *d_status;            // device error word kernels set (TSG_ERR_TIMEOUT, TSG_ERR_OVERFLOW), 0 when clear
    long long allocs;         // device allocations tsg_alloc made on the context
    int spa_dense;            // SPA schedule: C values per tile from which a product takes the tile kernel
    int last_step3;           // TSG_STEP3_* of the last numeric step launched
};

// Looks up the no-alloc conversion's scratch address on a device (that
// device current); run at context creation.
int tsg_noalloc_prepare(int device);

// Reads and clears the context's device error word (synchronises the
// context's stream); returns TSG_OK or the code a kernel recorded.
int tsg_take_device_status(tsg_context *ctx);

// C tile rows are copied to the host in at most TSG_MAX_CHUNKS chunks of at
// least TSG_CHUNK_NNZ nonzeros (tsg_spgemm_to_host).
#define TSG_MAX_CHUNKS 8
#define TSG_CHUNK_NNZ (1LL << 20)

// Creates the context's copy stream and event if needed.
int tsg_copy_stream(tsg_context *ctx);

// C = A*B (device operands) into host CSR buffers of nnz_cap entries, the
// copy overlapping the numeric step; TSG_ERR_OVERFLOW (with *nnzC set) when
// nnz(C) > nnz_cap.  Synchronous.
int tsg_spgemm_to_host(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B, int *h_rowptr, int *h_colidx,
                       double *h_val, long long nnz_cap, int *nnzC, tsg_spgemm_info *info);

// Records a formatted message as the thread's last error and returns code.
int tsg_set_error(int code, const char *fmt, ...);

#define TSG_CUDA(call)                                                                      \
    do                                                                                      \
    {                                                                                       \
        cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess)                                                              \
            return tsg_set_error(_e == cudaErrorMemoryAllocation ? TSG_ERR_OOM : TSG_ERR_CUDA, \
                                 "%s:%d %s: %s", __FILE__, __LINE__, #call,                \
                                 cudaGetErrorString(_e));                                   \
    } while (0)

#define TSG_TRY(expr)      \
    do                     \
    {                      \
        int _s = (expr);   \
        if (_s != TSG_OK)  \
            return _s;     \
    } while (0)

#define TSG_LAUNCH_CHECK()     \
    do                         \
    {                          \
        ctx->launches++;       \
        TSG_CUDA(cudaGetLastError()); \
    } while (0)

// Device allocation on the context's stream.  Every allocation is rounded
// up to 16 bytes and given 16 bytes of slack, so kernels may copy a range
// with its end rounded up to a 16-byte boundary (bulk copies) without
// leaving the allocation.
template <typename T>
static inline int tsg_alloc(tsg_context *ctx, T **p, size_t count)
{
    *p = nullptr;
    if (count == 0)
        count = 1;
    const size_t bytes = ((count * sizeof(T) + 15) & ~(size_t)15) + 16;
    ctx->allocs++;
    cudaError_t e = cudaMallocAsync((void **)p, bytes, ctx->stream);
    if (e != cudaSuccess)
    {
        *p = nullptr;
        return tsg_set_error(TSG_ERR_OOM, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    return TSG_OK;
}

template <typename T>
static inline void tsg_release(tsg_context *ctx, T *&p)
{
    if (p)
        cudaFreeAsync((void *)p, ctx->stream);
    p = nullptr;
}

static inline unsigned int tsg_blocks(long long work, int per_block)
{
    long long b = (work + per_block - 1) / per_block;
    return (unsigned int)(b < 1 ? 1 : b);
}

// Exclusive scan of n int32 counts into out[0..n] (out[n] = total).  in and
// out may alias.  The total is also returned through *total (synchronous
// read-back) when total != nullptr.
int tsg_scan_counts(tsg_context *ctx, const int *in, int *out, long long n, long long *total);

// Stable sort of (key, value) pairs by the low end_bit bits of the keys.
int tsg_sort_pairs_u64(tsg_context *ctx, unsigned long long *keys, int *vals, long long n, int end_bit);
int tsg_sort_pairs_u32(tsg_context *ctx, unsigned int *keys, int *vals, long long n, int end_bit);

// Validates a device CSR (ptr monotone, rowptr[0]=0, rowptr[m]=nnz, columns
// in range and strictly increasing per row).
int tsg_check_csr(tsg_context *ctx, int m, int n, int nnz, const int *rowptr, const int *colidx);

// Column view of a row-major tiled matrix (csc_tile_ptr / rowidx / pos).
int tsg_build_csc_view(tsg_context *ctx, tsg_tiled *mat);

// Readback helper: copies one long long / int from device to host (syncs).
int tsg_read_int(tsg_context *ctx, const int *dptr, long long *out);

// Product count over device CSR arrays.
int tsg_count_products_dev(tsg_context *ctx, int nnzA, const int *a_col, const int *b_rowptr,
                           long long *out);

int tsg_tiled_alloc_arrays(tsg_context *ctx, tsg_tiled *t, int with_csc);
