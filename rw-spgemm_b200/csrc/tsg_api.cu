// Context management, host<->device transfer of tiled matrices, the drop-in
// entry points of the reference (csr2tile_row_major, csr2tile_col_major,
// tilespgemm, tile2csr, matrix_destroy) and the end-to-end CSR call.
#include <stdlib.h>

#include "tsg_internal.h"

int tsg_gather_colmajor(tsg_context *ctx, const tsg_tiled *src, int *tnnz_cm, unsigned char *Ptr_cm,
                        unsigned short *mask_cm, unsigned char *Col_cm, double *Val_cm);
int tsg_colmajor_data_to_rowmajor(tsg_context *ctx, tsg_tiled *mat);

extern "C" const char *tsg_last_error(void);

extern "C" const char *tsg_status_string(int status)
{
    switch (status)
    {
    case TSG_OK:
        return "ok";
    case TSG_ERR_INVALID:
        return "invalid argument";
    case TSG_ERR_CUDA:
        return "CUDA error";
    case TSG_ERR_OOM:
        return "out of device memory";
    case TSG_ERR_INPUT:
        return "malformed input matrix";
    case TSG_ERR_OVERFLOW:
        return "result exceeds 32-bit offsets";
    case TSG_ERR_UNSUPPORTED:
        return "unsupported";
    case TSG_ERR_TIMEOUT:
        return "device wait timed out";
    case TSG_ERR_REJECTED:
        return "admission rejected";
    default:
        return "unknown status";
    }
}

extern "C" int tsg_context_create(int device, tsg_context **out)
{
    if (!out)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    *out = nullptr;
    TSG_CUDA(cudaSetDevice(device));
    tsg_context *ctx = (tsg_context *)calloc(1, sizeof(tsg_context));
    if (!ctx)
        return tsg_set_error(TSG_ERR_OOM, "host allocation failed");
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaMallocHost((void **)&ctx->h_pinned, 64 * sizeof(long long));
    for (int i = 0; i < 8 && e == cudaSuccess; i++)
        e = cudaEventCreate(&ctx->ev[i]);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&ctx->d_status, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemset(ctx->d_status, 0, sizeof(int));
    if (e == cudaSuccess && tsg_noalloc_prepare(device) != TSG_OK)
        e = cudaErrorUnknown;
    if (e != cudaSuccess)
    {
        free(ctx);
        return tsg_set_error(TSG_ERR_CUDA, "context creation failed: %s", cudaGetErrorString(e));
    }
    ctx->own_stream = 1;
    ctx->sched = TSG_SCHED_SPA;
    ctx->seg_tiles = 8;
    ctx->acc_cap = 512;
    ctx->fuse12 = 1;
    ctx->spa_dense = TSG_SPA_DENSE_DEFAULT;
    // keep freed pool memory cached so repeated products do not return pages
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess)
    {
        unsigned long long thr = ~0ULL;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    *out = ctx;
    return TSG_OK;
}

extern "C" int tsg_context_destroy(tsg_context *ctx)
{
    if (!ctx)
        return TSG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < 8; i++)
        cudaEventDestroy(ctx->ev[i]);
    if (ctx->copy_stream)
    {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
        cudaEventDestroy(ctx->copy_ev);
    }
    if (ctx->own_stream)
        cudaStreamDestroy(ctx->stream);
    cudaFreeHost(ctx->h_pinned);
    cudaFree(ctx->d_status);
    free(ctx);
    return TSG_OK;
}

int tsg_take_device_status(tsg_context *ctx)
{
    int *h = (int *)(ctx->h_pinned + 63);
    TSG_CUDA(cudaMemcpyAsync(h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    const int code = *h;
    if (code == TSG_OK)
        return TSG_OK;
    TSG_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    if (code == TSG_ERR_TIMEOUT)
        return tsg_set_error(code, "a kernel's bounded wait ran out (numeric step pipeline)");
    if (code == TSG_ERR_OVERFLOW)
        return tsg_set_error(code, "a numeric step's accumulator slot fell outside its segment");
    return tsg_set_error(code, "a kernel recorded error %d", code);
}

extern "C" int tsg_context_set_stream(tsg_context *ctx, void *stream)
{
    if (!ctx)
        return tsg_set_error(TSG_ERR_INVALID, "null context");
    if (stream)
    {
        if (ctx->own_stream)
        {
            cudaStreamSynchronize(ctx->stream);
            cudaStreamDestroy(ctx->stream);
        }
        ctx->stream = (cudaStream_t)stream;
        ctx->own_stream = 0;
    }
    else if (!ctx->own_stream)
    {
        TSG_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = 1;
    }
    return TSG_OK;
}

extern "C" int tsg_context_set_schedule(tsg_context *ctx, int schedule, int seg_tiles, int acc_cap)
{
    if (!ctx)
        return tsg_set_error(TSG_ERR_INVALID, "null context");
    if (schedule != TSG_SCHED_TILES && schedule != TSG_SCHED_ROWS && schedule != TSG_SCHED_ELEMS &&
        schedule != TSG_SCHED_SPA)
        return tsg_set_error(TSG_ERR_INVALID, "unknown schedule %d", schedule);
    if (schedule == TSG_SCHED_ROWS)
    {
        const bool ok = (seg_tiles == 8 && (acc_cap == 256 || acc_cap == 512 || acc_cap == 1024)) ||
                        (seg_tiles == 16 && (acc_cap == 512 || acc_cap == 1024 || acc_cap == 2048)) ||
                        (seg_tiles == 32 && (acc_cap == 1024 || acc_cap == 2048));
        if (!ok)
            return tsg_set_error(TSG_ERR_INVALID, "unsupported (seg_tiles, acc_cap) = (%d, %d)", seg_tiles, acc_cap);
        ctx->seg_tiles = seg_tiles;
        ctx->acc_cap = acc_cap;
    }
    ctx->sched = schedule;
    return TSG_OK;
}

extern "C" int tsg_context_set_dense_threshold(tsg_context *ctx, int values_per_tile)
{
    if (!ctx)
        return tsg_set_error(TSG_ERR_INVALID, "null context");
    if (values_per_tile < 0 || values_per_tile > 257)
        return tsg_set_error(TSG_ERR_INVALID, "dense threshold %d outside [0, 257]", values_per_tile);
    ctx->spa_dense = values_per_tile ? values_per_tile : TSG_SPA_DENSE_DEFAULT;
    return TSG_OK;
}

extern "C" int tsg_context_set_fusion(tsg_context *ctx, int fuse_step12)
{
    if (!ctx)
        return tsg_set_error(TSG_ERR_INVALID, "null context");
    ctx->fuse12 = fuse_step12 ? 1 : 0;
    return TSG_OK;
}

extern "C" int tsg_context_query(tsg_context *ctx)
{
    if (!ctx)
        return tsg_set_error(TSG_ERR_INVALID, "null context");
    const cudaError_t e = cudaStreamQuery(ctx->stream);
    if (e == cudaSuccess)
        return 0;
    if (e == cudaErrorNotReady)
        return 1;
    return tsg_set_error(TSG_ERR_CUDA, "stream query: %s", cudaGetErrorString(e));
}

extern "C" int tsg_context_synchronize(tsg_context *ctx)
{
    if (!ctx)
        return tsg_set_error(TSG_ERR_INVALID, "null context");
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    return tsg_take_device_status(ctx);
}

extern "C" long long tsg_context_launches(tsg_context *ctx) { return ctx ? ctx->launches : 0; }

extern "C" long long tsg_context_allocations(tsg_context *ctx) { return ctx ? ctx->allocs : 0; }

extern "C" int tsg_context_set_timing(tsg_context *ctx, int enabled)
{
    if (!ctx)
        return tsg_set_error(TSG_ERR_INVALID, "null context");
    ctx->timing = enabled ? 1 : 0;
    return TSG_OK;
}

extern "C" int tsg_tiled_free(tsg_context *ctx, tsg_tiled *t)
{
    if (!ctx || !t)
        return TSG_OK;
    if (t->_alloc) // borrowed view (batch arena): nothing to release
    {
        memset(t, 0, sizeof(*t));
        return TSG_OK;
    }
    tsg_release(ctx, t->tile_ptr);
    tsg_release(ctx, t->tile_columnidx);
    tsg_release(ctx, t->tile_rowidx);
    tsg_release(ctx, t->tile_nnz);
    tsg_release(ctx, t->tile_csr_Ptr);
    tsg_release(ctx, t->tile_csr_Col);
    tsg_release(ctx, t->tile_csr_Value);
    tsg_release(ctx, t->mask);
    tsg_release(ctx, t->csc_tile_ptr);
    tsg_release(ctx, t->csc_tile_rowidx);
    tsg_release(ctx, t->csc_tile_pos);
    tsg_release(ctx, t->mask_t);
    tsg_release(ctx, t->row_ptr);
    tsg_release(ctx, t->row_col);
    tsg_release(ctx, t->row_val);
    memset(t, 0, sizeof(*t));
    return TSG_OK;
}

static long long padded_bytes(const void *p, long long bytes)
{
    return p ? ((bytes + 15) & ~15LL) + 16 : 0; // tsg_alloc's size for `bytes`
}

extern "C" long long tsg_tiled_device_bytes(const tsg_tiled *t)
{
    if (!t || t->_alloc)
        return 0;
    const long long T = t->numtile, nnz = t->nnz;
    return padded_bytes(t->tile_ptr, 4 * ((long long)t->tilem + 1)) + padded_bytes(t->tile_columnidx, 4 * T) +
           padded_bytes(t->tile_rowidx, 4 * T) + padded_bytes(t->tile_nnz, 4 * (T + 1)) +
           padded_bytes(t->tile_csr_Ptr, TSG_BS * T) + padded_bytes(t->tile_csr_Col, nnz) +
           padded_bytes(t->tile_csr_Value, 8 * nnz) + padded_bytes(t->mask, 2 * TSG_BS * T) +
           padded_bytes(t->csc_tile_ptr, 4 * ((long long)t->tilen + 1)) + padded_bytes(t->csc_tile_rowidx, 4 * T) +
           padded_bytes(t->csc_tile_pos, 4 * T) + padded_bytes(t->mask_t, 2 * TSG_BS * T) +
           padded_bytes(t->row_ptr, 4 * ((long long)t->m + 1)) + padded_bytes(t->row_col, 4 * nnz) +
           padded_bytes(t->row_val, 8 * nnz);
}

extern "C" int tsg_context_pool_used(tsg_context *ctx, unsigned long long *bytes)
{
    if (!ctx || !bytes)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    cudaMemPool_t pool;
    TSG_CUDA(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
    unsigned long long used = 0; // the attribute is a 64-bit unsigned integer
    TSG_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
    *bytes = (unsigned long long)used;
    return TSG_OK;
}

extern "C" int tsg_count_products(tsg_context *ctx, int nnzA, const int *d_a_colidx, const int *d_b_rowptr,
                                  long long *nnzCub)
{
    if (!ctx || !nnzCub)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    return tsg_count_products_dev(ctx, nnzA, d_a_colidx, d_b_rowptr, nnzCub);
}

// ---------------------------------------------------------------------------
// Host <-> device copies of tiled matrices.
// ---------------------------------------------------------------------------
template <typename T>
static int h2d(tsg_context *ctx, T **dst, const T *src, size_t count)
{
    TSG_TRY(tsg_alloc(ctx, dst, count));
    if (count && src)
        TSG_CUDA(cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return TSG_OK;
}

template <typename T>
static int d2h(tsg_context *ctx, T **dst, const T *src, size_t count)
{
    *dst = (T *)malloc(count ? count * sizeof(T) : 1);
    if (!*dst)
        return tsg_set_error(TSG_ERR_OOM, "host allocation failed");
    if (count && src)
        TSG_CUDA(cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    return TSG_OK;
}

// masks from in-tile CSR when a host matrix carries none
__global__ void k_masks_from_csr(int T, const int *__restrict__ tnnz, const unsigned char *__restrict__ Ptr,
                                 const unsigned char *__restrict__ Col, unsigned short *__restrict__ mask)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int t = (int)(gid >> 4), r = threadIdx.x & 15;
    if (t >= T)
        return;
    const int base = tnnz[t], n = tnnz[t + 1] - base;
    const int s = Ptr[(long long)t * TSG_BS + r];
    const int e = r == TSG_BS - 1 ? n : Ptr[(long long)t * TSG_BS + r + 1];
    unsigned mk = 0;
    for (int q = s; q < e; q++)
        mk |= 0x8000u >> (Col[base + q] & 15);
    mask[(long long)t * TSG_BS + r] = (unsigned short)mk;
}

static int upload_common(tsg_context *ctx, const SMatrix *h, tsg_tiled *out)
{
    out->m = h->m;
    out->n = h->n;
    out->nnz = h->nnz;
    out->tilem = h->tilem;
    out->tilen = h->tilen;
    out->numtile = h->numtile;
    const size_t T = (size_t)h->numtile;
    TSG_TRY(h2d(ctx, &out->tile_ptr, h->tile_ptr, (size_t)h->tilem + 1));
    TSG_TRY(h2d(ctx, &out->tile_columnidx, h->tile_columnidx, T));
    TSG_TRY(h2d(ctx, &out->tile_nnz, h->tile_nnz, T + 1));
    TSG_TRY(h2d(ctx, &out->tile_csr_Ptr, h->tile_csr_Ptr, T * TSG_BS));
    TSG_TRY(h2d(ctx, &out->tile_csr_Col, h->tile_csr_Col, (size_t)h->nnz));
    TSG_TRY(h2d(ctx, &out->tile_csr_Value, h->tile_csr_Value, (size_t)h->nnz));
    if (h->mask)
        TSG_TRY(h2d(ctx, &out->mask, h->mask, T * TSG_BS));
    else
    {
        TSG_TRY(tsg_alloc(ctx, &out->mask, T * TSG_BS));
        if (T)
        {
            k_masks_from_csr<<<tsg_blocks((long long)T * 16, 256), 256, 0, ctx->stream>>>(
                (int)T, out->tile_nnz, out->tile_csr_Ptr, out->tile_csr_Col, out->mask);
            TSG_LAUNCH_CHECK();
        }
    }
    return TSG_OK;
}

extern "C" int tsg_tiled_upload_rowmajor(tsg_context *ctx, const SMatrix *h, tsg_tiled *out)
{
    if (!ctx || !h || !out)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    memset(out, 0, sizeof(*out));
    TSG_TRY(upload_common(ctx, h, out));
    out->col_packed = 1;
    TSG_TRY(h2d(ctx, &out->tile_rowidx, h->tile_rowidx, (size_t)h->numtile));
    return TSG_OK;
}

extern "C" int tsg_tiled_upload_colmajor(tsg_context *ctx, const SMatrix *h, tsg_tiled *out)
{
    if (!ctx || !h || !out)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    if (!h->csc_tile_ptr || !h->csc_tile_rowidx)
        return tsg_set_error(TSG_ERR_INVALID, "column-major matrix without csc_tile_ptr/csc_tile_rowidx");
    memset(out, 0, sizeof(*out));
    TSG_TRY(upload_common(ctx, h, out));
    out->col_packed = 0;
    TSG_TRY(h2d(ctx, &out->csc_tile_ptr, h->csc_tile_ptr, (size_t)h->tilen + 1));
    TSG_TRY(h2d(ctx, &out->csc_tile_rowidx, h->csc_tile_rowidx, (size_t)h->numtile));
    TSG_TRY(tsg_alloc(ctx, &out->tile_rowidx, (size_t)h->numtile));
    // internal layout: row-major tile data plus the column view
    return tsg_colmajor_data_to_rowmajor(ctx, out);
}

extern "C" int tsg_tiled_download(tsg_context *ctx, const tsg_tiled *src, int colmajor, SMatrix *dst)
{
    if (!ctx || !src || !dst)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    const size_t T = (size_t)src->numtile, nnz = (size_t)src->nnz;
    dst->m = src->m;
    dst->n = src->n;
    dst->nnz = src->nnz;
    dst->tilem = src->tilem;
    dst->tilen = src->tilen;
    dst->numtile = src->numtile;
    TSG_TRY(d2h(ctx, &dst->tile_ptr, src->tile_ptr, (size_t)src->tilem + 1));
    TSG_TRY(d2h(ctx, &dst->tile_columnidx, src->tile_columnidx, T));
    if (!colmajor)
    {
        TSG_TRY(d2h(ctx, &dst->tile_rowidx, src->tile_rowidx, T));
        TSG_TRY(d2h(ctx, &dst->tile_nnz, src->tile_nnz, T + 1));
        TSG_TRY(d2h(ctx, &dst->tile_csr_Ptr, src->tile_csr_Ptr, T * TSG_BS));
        TSG_TRY(d2h(ctx, &dst->mask, src->mask, T * TSG_BS));
        TSG_TRY(d2h(ctx, &dst->tile_csr_Col, src->tile_csr_Col, nnz));
        TSG_TRY(d2h(ctx, &dst->tile_csr_Value, src->tile_csr_Value, nnz));
        dst->csc_tile_ptr = nullptr;
        dst->csc_tile_rowidx = nullptr;
    }
    else
    {
        if (!src->csc_tile_ptr)
            return tsg_set_error(TSG_ERR_INVALID, "column-major download needs the column view");
        int *tnnz;
        unsigned char *Ptr, *Col;
        unsigned short *mask;
        double *Val;
        TSG_TRY(tsg_alloc(ctx, &tnnz, T + 1));
        TSG_TRY(tsg_alloc(ctx, &Ptr, T * TSG_BS));
        TSG_TRY(tsg_alloc(ctx, &mask, T * TSG_BS));
        TSG_TRY(tsg_alloc(ctx, &Col, nnz));
        TSG_TRY(tsg_alloc(ctx, &Val, nnz));
        TSG_TRY(tsg_gather_colmajor(ctx, src, tnnz, Ptr, mask, Col, Val));
        // the reference leaves B's tile_rowidx zero-filled (src/csr2tile.h:318-319)
        dst->tile_rowidx = (int *)calloc(T ? T : 1, sizeof(int));
        TSG_TRY(d2h(ctx, &dst->tile_nnz, tnnz, T + 1));
        TSG_TRY(d2h(ctx, &dst->tile_csr_Ptr, Ptr, T * TSG_BS));
        TSG_TRY(d2h(ctx, &dst->mask, mask, T * TSG_BS));
        TSG_TRY(d2h(ctx, &dst->tile_csr_Col, Col, nnz));
        TSG_TRY(d2h(ctx, &dst->tile_csr_Value, Val, nnz));
        TSG_TRY(d2h(ctx, &dst->csc_tile_ptr, src->csc_tile_ptr, (size_t)src->tilen + 1));
        TSG_TRY(d2h(ctx, &dst->csc_tile_rowidx, src->csc_tile_rowidx, T));
        TSG_CUDA(cudaStreamSynchronize(ctx->stream));
        tsg_release(ctx, tnnz);
        tsg_release(ctx, Ptr);
        tsg_release(ctx, mask);
        tsg_release(ctx, Col);
        tsg_release(ctx, Val);
    }
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    return TSG_OK;
}

// ---------------------------------------------------------------------------
// End-to-end CSR call with host buffers.
// ---------------------------------------------------------------------------
template <typename T>
static int d2h_pinned(tsg_context *ctx, T **dst, const T *src, size_t count)
{
    TSG_CUDA(cudaMallocHost((void **)dst, (count ? count : 1) * sizeof(T)));
    if (count && src)
        TSG_CUDA(cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    return TSG_OK;
}

extern "C" void tsg_host_free(void *p)
{
    if (p)
        cudaFreeHost(p);
}

extern "C" int tsg_spgemm_csr_host(tsg_context *ctx, int m, int k, int n, int nnzA, const int *a_rowptr,
                                   const int *a_colidx, const double *a_val, int nnzB, const int *b_rowptr,
                                   const int *b_colidx, const double *b_val, int *nnzC, int **c_rowptr,
                                   int **c_colidx, double **c_val, tsg_spgemm_info *info)
{
    return tsg_spgemm_csr_host_ex(ctx, m, k, n, nnzA, a_rowptr, a_colidx, a_val, nnzB, b_rowptr, b_colidx, b_val,
                                  nnzC, c_rowptr, c_colidx, c_val, info, 0);
}

extern "C" int tsg_spgemm_csr_host_ex(tsg_context *ctx, int m, int k, int n, int nnzA, const int *a_rowptr,
                                      const int *a_colidx, const double *a_val, int nnzB, const int *b_rowptr,
                                      const int *b_colidx, const double *b_val, int *nnzC, int **c_rowptr,
                                      int **c_colidx, double **c_val, tsg_spgemm_info *info, int flags)
{
    if (!ctx || !a_rowptr || !b_rowptr || !nnzC || !c_rowptr || !c_colidx || !c_val)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    const bool alias =
        (a_rowptr == b_rowptr && a_colidx == b_colidx && a_val == b_val && m == k && k == n && nnzA == nnzB);
    int *dA_rp, *dA_ci, *dB_rp = nullptr, *dB_ci = nullptr;
    double *dA_v, *dB_v = nullptr;
    TSG_TRY(h2d(ctx, &dA_rp, a_rowptr, (size_t)m + 1));
    TSG_TRY(h2d(ctx, &dA_ci, a_colidx, (size_t)nnzA));
    TSG_TRY(h2d(ctx, &dA_v, a_val, (size_t)nnzA));
    if (!alias)
    {
        TSG_TRY(h2d(ctx, &dB_rp, b_rowptr, (size_t)k + 1));
        TSG_TRY(h2d(ctx, &dB_ci, b_colidx, (size_t)nnzB));
        TSG_TRY(h2d(ctx, &dB_v, b_val, (size_t)nnzB));
    }
    tsg_tiled A, B, C;
    memset(&A, 0, sizeof(A));
    memset(&B, 0, sizeof(B));
    memset(&C, 0, sizeof(C));
    int st;
    if (alias)
    {
        // one conversion serves both roles: plain bytes + column view
        st = tsg_csr_to_tiled(ctx, m, k, nnzA, dA_rp, dA_ci, dA_v, TSG_TILED_CSC_VIEW, &A);
    }
    else
    {
        st = tsg_csr_to_tiled(ctx, m, k, nnzA, dA_rp, dA_ci, dA_v, TSG_TILED_PACKED_COL, &A);
        if (st == TSG_OK)
            st = tsg_csr_to_tiled(ctx, k, n, nnzB, dB_rp, dB_ci, dB_v, TSG_TILED_CSC_VIEW, &B);
    }
    if (st == TSG_OK)
        st = tsg_spgemm(ctx, &A, alias ? &A : &B, &C, info);
    int *dC_rp = nullptr, *dC_ci = nullptr;
    double *dC_v = nullptr;
    if (st == TSG_OK)
    {
        st = tsg_alloc(ctx, &dC_rp, (size_t)m + 1);
        if (st == TSG_OK)
            st = tsg_alloc(ctx, &dC_ci, (size_t)C.nnz);
        if (st == TSG_OK)
            st = tsg_alloc(ctx, &dC_v, (size_t)C.nnz);
        if (st == TSG_OK)
            st = tsg_tiled_to_csr(ctx, &C, dC_rp, dC_ci, dC_v);
    }
    if (st == TSG_OK)
    {
        *nnzC = C.nnz;
        if (flags & TSG_HOST_PINNED_OUTPUT)
        {
            st = d2h_pinned(ctx, c_rowptr, dC_rp, (size_t)m + 1);
            if (st == TSG_OK)
                st = d2h_pinned(ctx, c_colidx, dC_ci, (size_t)C.nnz);
            if (st == TSG_OK)
                st = d2h_pinned(ctx, c_val, dC_v, (size_t)C.nnz);
        }
        else
        {
            st = d2h(ctx, c_rowptr, dC_rp, (size_t)m + 1);
            if (st == TSG_OK)
                st = d2h(ctx, c_colidx, dC_ci, (size_t)C.nnz);
            if (st == TSG_OK)
                st = d2h(ctx, c_val, dC_v, (size_t)C.nnz);
        }
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (st == TSG_OK && e != cudaSuccess)
            st = tsg_set_error(TSG_ERR_CUDA, "%s", cudaGetErrorString(e));
    }
    tsg_tiled_free(ctx, &A);
    tsg_tiled_free(ctx, &B);
    tsg_tiled_free(ctx, &C);
    tsg_release(ctx, dA_rp);
    tsg_release(ctx, dA_ci);
    tsg_release(ctx, dA_v);
    tsg_release(ctx, dB_rp);
    tsg_release(ctx, dB_ci);
    tsg_release(ctx, dB_v);
    tsg_release(ctx, dC_rp);
    tsg_release(ctx, dC_ci);
    tsg_release(ctx, dC_v);
    return st;
}

// ---------------------------------------------------------------------------
// Drop-in entry points (host buffers, void return, abort on error).
// ---------------------------------------------------------------------------
static tsg_context *g_ctx = nullptr;
static int g_ctx_device = -1;

tsg_context *tsg_dropin_context(void)
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (g_ctx && g_ctx_device == dev)
        return g_ctx;
    if (g_ctx)
        tsg_context_destroy(g_ctx);
    g_ctx = nullptr;
    if (tsg_context_create(dev, &g_ctx) != TSG_OK)
    {
        fprintf(stderr, "tilespgemm_b200: cannot create a context on device %d: %s\n", dev, tsg_last_error());
        abort();
    }
    g_ctx_device = dev;
    return g_ctx;
}

static void dropin_check(int st, const char *what)
{
    if (st != TSG_OK)
    {
        fprintf(stderr, "tilespgemm_b200: %s failed: %s (%s)\n", what, tsg_status_string(st), tsg_last_error());
        abort();
    }
}

static void dropin_convert(SMatrix *matrix, int colmajor)
{
    tsg_context *ctx = tsg_dropin_context();
    int *rp, *ci;
    double *v;
    dropin_check(h2d(ctx, &rp, matrix->rowpointer, (size_t)matrix->m + 1), "upload");
    dropin_check(h2d(ctx, &ci, matrix->columnindex, (size_t)matrix->nnz), "upload");
    dropin_check(h2d(ctx, &v, matrix->value, (size_t)matrix->nnz), "upload");
    tsg_tiled t;
    dropin_check(tsg_csr_to_tiled(ctx, matrix->m, matrix->n, matrix->nnz, rp, ci, v,
                                  colmajor ? TSG_TILED_CSC_VIEW : TSG_TILED_PACKED_COL, &t),
                 colmajor ? "csr2tile_col_major" : "csr2tile_row_major");
    dropin_check(tsg_tiled_download(ctx, &t, colmajor, matrix), "download");
    tsg_tiled_free(ctx, &t);
    tsg_release(ctx, rp);
    tsg_release(ctx, ci);
    tsg_release(ctx, v);
    cudaStreamSynchronize(ctx->stream);
}

extern "C" void csr2tile_row_major(SMatrix *matrix) { dropin_convert(matrix, 0); }

extern "C" void csr2tile_col_major(SMatrix *matrix) { dropin_convert(matrix, 1); }

extern "C" void matrix_destroy(SMatrix *matrix)
{
    free(matrix->tile_ptr);
    free(matrix->tile_columnidx);
    free(matrix->tile_nnz);
    free(matrix->tile_csr_Value);
    free(matrix->tile_csr_Col);
    free(matrix->tile_csr_Ptr);
    free(matrix->mask);
}

extern "C" void tile2csr(SMatrix *matrix)
{
    tsg_context *ctx = tsg_dropin_context();
    tsg_tiled t;
    memset(&t, 0, sizeof(t));
    t.m = matrix->m;
    t.n = matrix->n;
    t.tilem = matrix->tilem;
    t.tilen = matrix->tilen;
    t.numtile = matrix->numtile;
    const size_t T = (size_t)matrix->numtile;
    int nnz_tiles = T ? matrix->tile_nnz[T] : 0;
    dropin_check(h2d(ctx, &t.tile_ptr, matrix->tile_ptr, (size_t)matrix->tilem + 1), "upload");
    dropin_check(h2d(ctx, &t.tile_columnidx, matrix->tile_columnidx, T), "upload");
    dropin_check(h2d(ctx, &t.tile_nnz, matrix->tile_nnz, T + 1), "upload");
    dropin_check(h2d(ctx, &t.tile_csr_Ptr, matrix->tile_csr_Ptr, T * TSG_BS), "upload");
    dropin_check(h2d(ctx, &t.tile_csr_Col, matrix->tile_csr_Col, (size_t)nnz_tiles), "upload");
    dropin_check(h2d(ctx, &t.tile_csr_Value, matrix->tile_csr_Value, (size_t)nnz_tiles), "upload");
    int *rp, *ci;
    double *v;
    dropin_check(tsg_alloc(ctx, &rp, (size_t)matrix->m + 1), "alloc");
    dropin_check(tsg_alloc(ctx, &ci, (size_t)nnz_tiles), "alloc");
    dropin_check(tsg_alloc(ctx, &v, (size_t)nnz_tiles), "alloc");
    dropin_check(tsg_tiled_to_csr(ctx, &t, rp, ci, v), "tile2csr");
    long long nnz = 0;
    dropin_check(tsg_read_int(ctx, rp + matrix->m, &nnz), "tile2csr");
    matrix->nnz = (int)nnz;
    dropin_check(d2h(ctx, &matrix->rowpointer, rp, (size_t)matrix->m + 1), "download");
    dropin_check(d2h(ctx, &matrix->columnindex, ci, (size_t)nnz), "download");
    dropin_check(d2h(ctx, &matrix->value, v, (size_t)nnz), "download");
    cudaStreamSynchronize(ctx->stream);
    tsg_tiled_free(ctx, &t);
    tsg_release(ctx, rp);
    tsg_release(ctx, ci);
    tsg_release(ctx, v);
    cudaStreamSynchronize(ctx->stream);
}

// ---------------------------------------------------------------------------
// Intersection bitmaps of the reference's driver (src/main.cu:430-465): a
// warp per tile row (A) or tile column (B), its lanes over the row's tiles,
// each setting bit 31 - idx % 32 of word idx / 32 of the row's words.
// ---------------------------------------------------------------------------
__global__ void k_tile_bitmaps(int rows, int len, const int *__restrict__ ptr, const int *__restrict__ idx,
                               unsigned *__restrict__ bits)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= rows)
        return;
    unsigned *row = bits + w * (long long)len;
    for (int j = ptr[w] + lane; j < ptr[w + 1]; j += 32)
    {
        const int c = idx[j];
        if (c >= 0 && (c >> 5) < len) // validated on the host; kept inside the row regardless
            atomicOr(&row[c >> 5], 1u << (31 - (c & 31)));
    }
}

static int bitmaps_of(tsg_context *ctx, int rows, int len, const int *h_ptr, const int *h_idx, unsigned **out)
{
    *out = (unsigned *)calloc((size_t)rows * len > 0 ? (size_t)rows * len : 1, sizeof(unsigned));
    if (!*out)
        return tsg_set_error(TSG_ERR_OOM, "host allocation failed");
    if (rows == 0 || len == 0)
        return TSG_OK;
    const int n = h_ptr[rows];
    int *d_ptr, *d_idx;
    unsigned *d_bits;
    TSG_TRY(tsg_alloc(ctx, &d_ptr, (size_t)rows + 1));
    TSG_TRY(tsg_alloc(ctx, &d_idx, (size_t)(n > 0 ? n : 1)));
    TSG_TRY(tsg_alloc(ctx, &d_bits, (size_t)rows * len));
    TSG_CUDA(cudaMemcpyAsync(d_ptr, h_ptr, ((size_t)rows + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    if (n > 0)
        TSG_CUDA(cudaMemcpyAsync(d_idx, h_idx, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    TSG_CUDA(cudaMemsetAsync(d_bits, 0, (size_t)rows * len * sizeof(unsigned), ctx->stream));
    k_tile_bitmaps<<<tsg_blocks((long long)rows * 32, 256), 256, 0, ctx->stream>>>(rows, len, d_ptr, d_idx, d_bits);
    TSG_LAUNCH_CHECK();
    TSG_CUDA(cudaMemcpyAsync(*out, d_bits, (size_t)rows * len * sizeof(unsigned), cudaMemcpyDeviceToHost,
                             ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    tsg_release(ctx, d_ptr);
    tsg_release(ctx, d_idx);
    tsg_release(ctx, d_bits);
    return TSG_OK;
}

extern "C" int tile_intersection_bitmaps(const SMatrix *A, const SMatrix *B, unsigned **bitmask_A,
                                         unsigned **bitmask_B, int *bitmask_len)
{
    if (!A || !B || !bitmask_A || !bitmask_B || !bitmask_len || !A->tile_ptr || !B->csc_tile_ptr ||
        (A->numtile > 0 && !A->tile_columnidx) || (B->numtile > 0 && !B->csc_tile_rowidx))
        return tsg_set_error(TSG_ERR_INVALID, "tile_intersection_bitmaps: A needs csr2tile_row_major's tiles, "
                                              "B csr2tile_col_major's");
    if (A->tilen != B->tilem)
        return tsg_set_error(TSG_ERR_INVALID, "tile_intersection_bitmaps: A has %d tile columns, B %d tile rows",
                             A->tilen, B->tilem);
    *bitmask_A = *bitmask_B = nullptr;
    const int len = (A->tilen + 31) / 32; // ceil(tilen_A / 32), as the reference's driver
    *bitmask_len = len;
    tsg_context *ctx = tsg_dropin_context();
    int st = bitmaps_of(ctx, A->tilem, len, A->tile_ptr, A->tile_columnidx, bitmask_A);
    if (st == TSG_OK)
        st = bitmaps_of(ctx, B->tilen, len, B->csc_tile_ptr, B->csc_tile_rowidx, bitmask_B);
    if (st != TSG_OK)
    {
        free(*bitmask_A);
        free(*bitmask_B);
        *bitmask_A = *bitmask_B = nullptr;
    }
    return st;
}

#define DROPIN_REPEAT 5

extern "C" void tilespgemm(SMatrix *matrixA, SMatrix *matrixB, SMatrix *matrixC,
                           unsigned int *blk_intersec_bitmask_A, unsigned int *blk_intersec_bitmask_B,
                           int blk_intersec_bitmask_len, double densityA, double densityB,
                           unsigned long long int nnzCub, unsigned long long int *nnzC_computed,
                           double *compression_rate, double *time_tile, double *gflops_tile, char *filename,
                           double *time_step1, double *time_step2, double *time_step3, double *time_malloc)
{
    (void)blk_intersec_bitmask_A;
    (void)blk_intersec_bitmask_B;
    (void)blk_intersec_bitmask_len;
    (void)densityA;
    (void)densityB;
    (void)filename;
    tsg_context *ctx = tsg_dropin_context();
    tsg_tiled A, B, C;
    dropin_check(tsg_tiled_upload_rowmajor(ctx, matrixA, &A), "upload A");
    dropin_check(tsg_tiled_upload_colmajor(ctx, matrixB, &B), "upload B");
    cudaStreamSynchronize(ctx->stream);
    double tmin = 1e300;
    tsg_spgemm_info info;
    memset(&C, 0, sizeof(C));
    for (int ri = 0; ri < DROPIN_REPEAT; ri++)
    {
        if (ri > 0)
            tsg_tiled_free(ctx, &C);
        ctx->timing = 1;
        cudaStreamSynchronize(ctx->stream);
        dropin_check(tsg_spgemm(ctx, &A, &B, &C, &info), "tilespgemm");
        cudaStreamSynchronize(ctx->stream);
        ctx->timing = 0;
        if (ri == 0)
        {
            if (time_step1)
                *time_step1 = info.ms_step1;
            if (time_step2)
                *time_step2 = info.ms_step2;
            if (time_step3)
                *time_step3 = info.ms_step3;
            if (time_malloc)
                *time_malloc = 0.0;
            printf("step1 ----Calculate the number and tile-column index of tiles of matrixC---\n");
            printf("step1 ---------------------- Runtime is  %.2f ms-------------------------\n", info.ms_step1);
            printf("\nstep2 --------Calculate the number of nonzeros of each tile of matrixC-----\n");
            printf("step2 ---------------------- Runtime is  %.2f ms-------------------------\n", info.ms_step2);
        }
        printf("Tiny: %d, Sml: %d, Lrg: %d, Dns: %d, Ful: %d\n", info.bins[0], 0, info.bins[1], info.bins[2],
               info.bins[3]);
        if (ri == 0)
        {
            printf("\nstep3 ---------Calculate the val&col of nonzeros of matrixC-------------\n");
            printf("step3 ---------------------- Runtime is  %.2f ms------------------------\n", info.ms_step3);
            printf("\n-----------------------Malloc uses %.2f ms-------------------------------\n", 0.0);
        }
        if (info.ms_total < tmin)
            tmin = info.ms_total;
    }
    if (nnzC_computed)
        *nnzC_computed = (unsigned long long)C.nnz;
    if (compression_rate)
        *compression_rate = C.nnz ? (double)nnzCub / (double)C.nnz : 0.0;
    if (time_tile)
        *time_tile = tmin;
    double gflops = tmin > 0 ? 2.0 * (double)nnzCub / (tmin * 1e6) : 0.0;
    if (gflops_tile)
        *gflops_tile = gflops;
    printf("Non-empty tiles of C = %i\n", C.numtile);
    printf("nnzC = %i\n", C.nnz);
    printf("CUDA  TileSpGEMM runtime is %4.2f ms, gflops = %4.2f\n", tmin, gflops);
    dropin_check(tsg_tiled_download(ctx, &C, 0, matrixC), "download C");
    tsg_tiled_free(ctx, &A);
    tsg_tiled_free(ctx, &B);
    tsg_tiled_free(ctx, &C);
    cudaStreamSynchronize(ctx->stream);
}

extern "C" int tsg_csr_host_to_tiled(tsg_context *ctx, int m, int n, int nnz, const int *h_rowptr,
                                     const int *h_colidx, const double *h_val, int flags, tsg_tiled *out)
{
    if (!ctx || !out || !h_rowptr)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    int *rp, *ci;
    double *v;
    TSG_TRY(h2d(ctx, &rp, h_rowptr, (size_t)m + 1));
    TSG_TRY(h2d(ctx, &ci, h_colidx, (size_t)nnz));
    TSG_TRY(h2d(ctx, &v, h_val, (size_t)nnz));
    const int st = tsg_csr_to_tiled(ctx, m, n, nnz, rp, ci, v, flags, out);
    tsg_release(ctx, rp);
    tsg_release(ctx, ci);
    tsg_release(ctx, v);
    return st;
}

extern "C" int tsg_tiled_to_csr_host(tsg_context *ctx, const tsg_tiled *C, int flags, int **rowptr, int **colidx,
                                     double **val)
{
    if (!ctx || !C || !rowptr || !colidx || !val)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    int *rp, *ci;
    double *v;
    TSG_TRY(tsg_alloc(ctx, &rp, (size_t)C->m + 1));
    TSG_TRY(tsg_alloc(ctx, &ci, (size_t)C->nnz));
    TSG_TRY(tsg_alloc(ctx, &v, (size_t)C->nnz));
    TSG_TRY(tsg_tiled_to_csr(ctx, C, rp, ci, v));
    if (flags & TSG_HOST_PINNED_OUTPUT)
    {
        TSG_TRY(d2h_pinned(ctx, rowptr, rp, (size_t)C->m + 1));
        TSG_TRY(d2h_pinned(ctx, colidx, ci, (size_t)C->nnz));
        TSG_TRY(d2h_pinned(ctx, val, v, (size_t)C->nnz));
    }
    else
    {
        TSG_TRY(d2h(ctx, rowptr, rp, (size_t)C->m + 1));
        TSG_TRY(d2h(ctx, colidx, ci, (size_t)C->nnz));
        TSG_TRY(d2h(ctx, val, v, (size_t)C->nnz));
    }
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    tsg_release(ctx, rp);
    tsg_release(ctx, ci);
    tsg_release(ctx, v);
    return TSG_OK;
}

// ---------------------------------------------------------------------------
// Two-phase end-to-end call (caller-owned output buffers).
// ---------------------------------------------------------------------------
struct tsg_result
{
    tsg_context *ctx;
    int m, nnz;
    int *rp, *ci;
    double *v;
};

extern "C" int tsg_spgemm_csr_host_start(tsg_context *ctx, int m, int k, int n, int nnzA, const int *a_rowptr,
                                         const int *a_colidx, const double *a_val, int nnzB, const int *b_rowptr,
                                         const int *b_colidx, const double *b_val, tsg_result **res, int *nnzC,
                                         tsg_spgemm_info *info)
{
    if (!ctx || !res || !nnzC || !a_rowptr || !b_rowptr)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    *res = nullptr;
    const bool alias =
        (a_rowptr == b_rowptr && a_colidx == b_colidx && a_val == b_val && m == k && k == n && nnzA == nnzB);
    tsg_tiled A, B, C;
    memset(&A, 0, sizeof(A));
    memset(&B, 0, sizeof(B));
    memset(&C, 0, sizeof(C));
    int st = alias ? tsg_csr_host_to_tiled(ctx, m, k, nnzA, a_rowptr, a_colidx, a_val, TSG_TILED_CSC_VIEW, &A)
                   : tsg_csr_host_to_tiled(ctx, m, k, nnzA, a_rowptr, a_colidx, a_val, TSG_TILED_PACKED_COL, &A);
    if (st == TSG_OK && !alias)
        st = tsg_csr_host_to_tiled(ctx, k, n, nnzB, b_rowptr, b_colidx, b_val, TSG_TILED_CSC_VIEW, &B);
    if (st == TSG_OK)
        st = tsg_spgemm(ctx, &A, alias ? &A : &B, &C, info);
    tsg_result *r = nullptr;
    if (st == TSG_OK)
    {
        r = (tsg_result *)calloc(1, sizeof(tsg_result));
        r->ctx = ctx;
        r->m = m;
        r->nnz = C.nnz;
        st = tsg_alloc(ctx, &r->rp, (size_t)m + 1);
        if (st == TSG_OK)
            st = tsg_alloc(ctx, &r->ci, (size_t)C.nnz);
        if (st == TSG_OK)
            st = tsg_alloc(ctx, &r->v, (size_t)C.nnz);
        if (st == TSG_OK)
            st = tsg_tiled_to_csr(ctx, &C, r->rp, r->ci, r->v);
    }
    tsg_tiled_free(ctx, &A);
    tsg_tiled_free(ctx, &B);
    tsg_tiled_free(ctx, &C);
    if (st != TSG_OK)
    {
        if (r)
            tsg_result_free(r);
        return st;
    }
    *nnzC = r->nnz;
    *res = r;
    return TSG_OK;
}

int tsg_copy_stream(tsg_context *ctx)
{
    if (ctx->copy_stream)
        return TSG_OK;
    TSG_CUDA(cudaEventCreateWithFlags(&ctx->copy_ev, cudaEventDisableTiming));
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess)
    {
        cudaEventDestroy(ctx->copy_ev);
        ctx->copy_stream = nullptr;
        return tsg_set_error(TSG_ERR_CUDA, "copy stream creation failed: %s", cudaGetErrorString(e));
    }
    return TSG_OK;
}

extern "C" int tsg_spgemm_csr_host_into(tsg_context *ctx, int m, int k, int n, int nnzA, const int *a_rowptr,
                                        const int *a_colidx, const double *a_val, int nnzB, const int *b_rowptr,
                                        const int *b_colidx, const double *b_val, int *c_rowptr, int *c_colidx,
                                        double *c_val, long long nnz_cap, int *nnzC, tsg_spgemm_info *info)
{
    if (!ctx || !nnzC || !a_rowptr || !b_rowptr || !c_rowptr || (nnz_cap > 0 && (!c_colidx || !c_val)) ||
        nnz_cap < 0)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    *nnzC = 0;
    const bool alias =
        (a_rowptr == b_rowptr && a_colidx == b_colidx && a_val == b_val && m == k && k == n && nnzA == nnzB);
    tsg_tiled A, B;
    memset(&A, 0, sizeof(A));
    memset(&B, 0, sizeof(B));
    int st = alias ? tsg_csr_host_to_tiled(ctx, m, k, nnzA, a_rowptr, a_colidx, a_val, TSG_TILED_CSC_VIEW, &A)
                   : tsg_csr_host_to_tiled(ctx, m, k, nnzA, a_rowptr, a_colidx, a_val, TSG_TILED_PACKED_COL, &A);
    if (st == TSG_OK && !alias)
        st = tsg_csr_host_to_tiled(ctx, k, n, nnzB, b_rowptr, b_colidx, b_val, TSG_TILED_CSC_VIEW, &B);
    if (st == TSG_OK)
        st = tsg_spgemm_to_host(ctx, &A, alias ? &A : &B, c_rowptr, c_colidx, c_val, nnz_cap, nnzC, info);
    tsg_tiled_free(ctx, &A);
    tsg_tiled_free(ctx, &B);
    return st;
}

extern "C" int tsg_result_copy(tsg_result *r, int *rowptr, int *colidx, double *val)
{
    if (!r || !rowptr)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    tsg_context *ctx = r->ctx;
    TSG_CUDA(cudaMemcpyAsync(rowptr, r->rp, ((size_t)r->m + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if (r->nnz)
    {
        TSG_CUDA(cudaMemcpyAsync(colidx, r->ci, (size_t)r->nnz * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        TSG_CUDA(cudaMemcpyAsync(val, r->v, (size_t)r->nnz * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    return TSG_OK;
}

extern "C" int tsg_result_free(tsg_result *r)
{
    if (!r)
        return TSG_OK;
    tsg_context *ctx = r->ctx;
    tsg_release(ctx, r->rp);
    tsg_release(ctx, r->ci);
    tsg_release(ctx, r->v);
    free(r);
    return TSG_OK;
}
