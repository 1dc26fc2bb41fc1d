// GPU format conversion: CSR -> 16x16 tiles, the column view of B, the
// column-major (reference B layout) gather, and tiles -> CSR.
//
// CSR -> tiles restates src/csr2tile.h:6-259 (row-major, packed (row<<4)|col
// bytes) and :261-478 (column-major B, plain bytes) of the reference, and
// tiles -> CSR restates src/tile2csr.h:8-137.  Rows must be sorted by
// strictly increasing column (checked by tsg_check_csr): the tile columns of
// one tile row are then the merge of 16 sorted lists, which a half-warp walks
// with one lane per row, so every tile row is converted in one pass with no
// scratch memory and the output comes out already sorted.
#include <limits.h>

#include "tsg_internal.h"

#define HW_MASK(tid) (0xFFFFu << ((tid) & 16))

// ---------------------------------------------------------------------------
// Pass 1: number of non-empty tiles in each tile row (half-warp per row).
// ---------------------------------------------------------------------------
__global__ void k_tile_count(int m, int tilem, const int *__restrict__ rowptr,
                             const int *__restrict__ col, int *__restrict__ tile_cnt)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int tr = (int)(gid >> 4);
    const int lane = threadIdx.x & 15;
    const unsigned hmask = HW_MASK(threadIdx.x);
    if (tr >= tilem)
        return;
    const int r = tr * TSG_BS + lane;
    int p = 0, e = 0;
    if (r < m)
    {
        p = rowptr[r];
        e = rowptr[r + 1];
    }
    int cur = p < e ? (col[p] >> 4) : INT_MAX;
    int cnt = 0;
    while (true)
    {
        const int jm = __reduce_min_sync(hmask, cur);
        if (jm == INT_MAX)
            break;
        cnt++;
        if (cur == jm)
        {
            do
            {
                ++p;
            } while (p < e && (col[p] >> 4) == jm);
            cur = p < e ? (col[p] >> 4) : INT_MAX;
        }
    }
    if (lane == 0)
        tile_cnt[tr] = cnt;
}

// ---------------------------------------------------------------------------
// Pass 2: tile columns, per-row offsets, masks and the in-tile entries.
// ---------------------------------------------------------------------------
__global__ void k_tile_fill(int m, int tilem, const int *__restrict__ rowptr,
                            const int *__restrict__ col, const double *__restrict__ val,
                            const int *__restrict__ tile_ptr, int packed,
                            int *__restrict__ tile_columnidx, int *__restrict__ tile_rowidx,
                            int *__restrict__ tile_nnz, unsigned char *__restrict__ tPtr,
                            unsigned char *__restrict__ tCol, double *__restrict__ tVal,
                            unsigned short *__restrict__ tMask)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int tr = (int)(gid >> 4);
    const int lane = threadIdx.x & 15;
    const unsigned hmask = HW_MASK(threadIdx.x);
    if (tr >= tilem)
        return;
    const int r = tr * TSG_BS + lane;
    int p = 0, e = 0;
    if (r < m)
    {
        p = rowptr[r];
        e = rowptr[r + 1];
    }
    // value offset of the tile row's first tile: the row's first CSR entry
    int run = __shfl_sync(hmask, p, 0, 16);
    int t = tile_ptr[tr];
    int cur = p < e ? (col[p] >> 4) : INT_MAX;
    while (true)
    {
        const int jm = __reduce_min_sync(hmask, cur);
        if (jm == INT_MAX)
            break;
        int c = 0;
        unsigned mk = 0;
        if (cur == jm)
        {
            int q = p;
            int cc;
            while (q < e && ((cc = col[q]) >> 4) == jm)
            {
                mk |= 0x8000u >> (cc & 15);
                q++;
            }
            c = q - p;
        }
        int incl = c;
#pragma unroll
        for (int d = 1; d < 16; d <<= 1)
        {
            int o = __shfl_up_sync(hmask, incl, d, 16);
            if (lane >= d)
                incl += o;
        }
        const int excl = incl - c;
        const int total = __shfl_sync(hmask, incl, 15, 16);
        tPtr[(long long)t * TSG_BS + lane] = (unsigned char)excl;
        tMask[(long long)t * TSG_BS + lane] = (unsigned short)mk;
        if (lane == 0)
        {
            tile_columnidx[t] = jm;
            tile_rowidx[t] = tr;
            tile_nnz[t] = run;
        }
        const int dst = run + excl;
        for (int i = 0; i < c; i++)
        {
            const int cc = col[p + i] & 15;
            tCol[dst + i] = (unsigned char)(packed ? ((lane << 4) | cc) : cc);
            tVal[dst + i] = val[p + i];
        }
        p += c;
        cur = p < e ? (col[p] >> 4) : INT_MAX;
        run += total;
        t++;
    }
    if (tr == tilem - 1 && lane == 0)
        tile_nnz[t] = run; // tile_nnz[numtile] = nnz
}

int tsg_tiled_alloc_arrays(tsg_context *ctx, tsg_tiled *t, int with_csc)
{
    const size_t T = (size_t)t->numtile;
    TSG_TRY(tsg_alloc(ctx, &t->tile_columnidx, T));
    TSG_TRY(tsg_alloc(ctx, &t->tile_rowidx, T));
    TSG_TRY(tsg_alloc(ctx, &t->tile_nnz, T + 1));
    TSG_TRY(tsg_alloc(ctx, &t->tile_csr_Ptr, T * TSG_BS));
    TSG_TRY(tsg_alloc(ctx, &t->mask, T * TSG_BS));
    TSG_TRY(tsg_alloc(ctx, &t->tile_csr_Col, (size_t)t->nnz));
    TSG_TRY(tsg_alloc(ctx, &t->tile_csr_Value, (size_t)t->nnz));
    if (with_csc)
    {
        TSG_TRY(tsg_alloc(ctx, &t->csc_tile_ptr, (size_t)t->tilen + 1));
        TSG_TRY(tsg_alloc(ctx, &t->csc_tile_rowidx, T));
        TSG_TRY(tsg_alloc(ctx, &t->csc_tile_pos, T));
    }
    return TSG_OK;
}

extern "C" int tsg_csr_to_tiled(tsg_context *ctx, int m, int n, int nnz, const int *d_rowptr,
                                const int *d_colidx, const double *d_val, int flags, tsg_tiled *out)
{
    if (!ctx || !out)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    memset(out, 0, sizeof(*out));
    TSG_TRY(tsg_check_csr(ctx, m, n, nnz, d_rowptr, d_colidx));
    out->m = m;
    out->n = n;
    out->nnz = nnz;
    out->tilem = (m + TSG_BS - 1) / TSG_BS;
    out->tilen = (n + TSG_BS - 1) / TSG_BS;
    out->col_packed = (flags & TSG_TILED_PACKED_COL) ? 1 : 0;
    const int tilem = out->tilem;
    TSG_TRY(tsg_alloc(ctx, &out->tile_ptr, (size_t)tilem + 1));
    long long T = 0;
    if (tilem > 0)
    {
        k_tile_count<<<tsg_blocks((long long)tilem * 16, 256), 256, 0, ctx->stream>>>(
            m, tilem, d_rowptr, d_colidx, out->tile_ptr);
        TSG_LAUNCH_CHECK();
        TSG_TRY(tsg_scan_counts(ctx, out->tile_ptr, out->tile_ptr, tilem, &T));
    }
    else
    {
        TSG_CUDA(cudaMemsetAsync(out->tile_ptr, 0, sizeof(int), ctx->stream));
    }
    out->numtile = (int)T;
    TSG_TRY(tsg_tiled_alloc_arrays(ctx, out, (flags & TSG_TILED_CSC_VIEW) ? 1 : 0));
    if (tilem > 0)
    {
        k_tile_fill<<<tsg_blocks((long long)tilem * 16, 256), 256, 0, ctx->stream>>>(
            m, tilem, d_rowptr, d_colidx, d_val, out->tile_ptr, out->col_packed, out->tile_columnidx,
            out->tile_rowidx, out->tile_nnz, out->tile_csr_Ptr, out->tile_csr_Col, out->tile_csr_Value,
            out->mask);
        TSG_LAUNCH_CHECK();
    }
    else
    {
        TSG_CUDA(cudaMemsetAsync(out->tile_nnz, 0, sizeof(int), ctx->stream));
    }
    if (flags & TSG_TILED_CSC_VIEW)
        TSG_TRY(tsg_build_csc_view(ctx, out));
    return TSG_OK;
}

// ---------------------------------------------------------------------------
// Column view: tiles sorted stably by tile column (row order kept inside a
// column), giving csc_tile_ptr / csc_tile_rowidx / csc_tile_pos.
// ---------------------------------------------------------------------------
__global__ void k_csc_keys(int T, const int *__restrict__ tile_col, unsigned int *__restrict__ keys,
                           int *__restrict__ vals, int *__restrict__ hist)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
    {
        int j = tile_col[t];
        keys[t] = (unsigned int)j;
        vals[t] = t;
        atomicAdd(&hist[j], 1);
    }
}

__global__ void k_csc_rows(int T, const int *__restrict__ pos, const int *__restrict__ tile_row,
                           int *__restrict__ csc_row)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < T; q += gridDim.x * blockDim.x)
        csc_row[q] = tile_row[pos[q]];
}

static int bits_for(long long v)
{
    int b = 1;
    while (b < 63 && (1LL << b) <= v)
        b++;
    return b;
}

// transposed masks: mask_t[t][c] has bit (15-r) when mask[t][r] has bit (15-c)
__global__ void k_mask_transpose(int T, const unsigned short *__restrict__ mask, unsigned short *__restrict__ mask_t)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int t = (int)(gid >> 4), c = threadIdx.x & 15;
    if (t >= T)
        return;
    const uint4 *mb = reinterpret_cast<const uint4 *>(mask + (long long)t * TSG_BS);
    const uint4 q0 = mb[0], q1 = mb[1];
    const unsigned w[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
    unsigned out = 0;
#pragma unroll
    for (int r = 0; r < 16; r++)
    {
        const unsigned row = (r & 1) ? (w[r >> 1] >> 16) : (w[r >> 1] & 0xFFFFu);
        out |= ((row >> (15 - c)) & 1u) << (15 - r);
    }
    mask_t[(long long)t * TSG_BS + c] = (unsigned short)out;
}

int tsg_build_mask_t(tsg_context *ctx, tsg_tiled *mat)
{
    const int T = mat->numtile;
    if (!mat->mask_t)
        TSG_TRY(tsg_alloc(ctx, &mat->mask_t, (size_t)T * TSG_BS));
    if (T > 0)
    {
        k_mask_transpose<<<tsg_blocks((long long)T * 16, 256), 256, 0, ctx->stream>>>(T, mat->mask, mat->mask_t);
        TSG_LAUNCH_CHECK();
    }
    return TSG_OK;
}

// Row view (scalar CSR of the matrix), from its tiles.
int tsg_build_row_view(tsg_context *ctx, tsg_tiled *mat)
{
    if (!mat->row_ptr)
    {
        TSG_TRY(tsg_alloc(ctx, &mat->row_ptr, (size_t)mat->m + 1));
        TSG_TRY(tsg_alloc(ctx, &mat->row_col, (size_t)mat->nnz));
        TSG_TRY(tsg_alloc(ctx, &mat->row_val, (size_t)mat->nnz));
    }
    return tsg_tiled_to_csr(ctx, mat, mat->row_ptr, mat->row_col, mat->row_val);
}

int tsg_build_csc_view(tsg_context *ctx, tsg_tiled *mat)
{
    TSG_TRY(tsg_build_mask_t(ctx, mat));
    TSG_TRY(tsg_build_row_view(ctx, mat));
    const int T = mat->numtile, tilen = mat->tilen;
    if (!mat->csc_tile_ptr)
    {
        TSG_TRY(tsg_alloc(ctx, &mat->csc_tile_ptr, (size_t)tilen + 1));
        TSG_TRY(tsg_alloc(ctx, &mat->csc_tile_rowidx, (size_t)T));
        TSG_TRY(tsg_alloc(ctx, &mat->csc_tile_pos, (size_t)T));
    }
    TSG_CUDA(cudaMemsetAsync(mat->csc_tile_ptr, 0, ((size_t)tilen + 1) * sizeof(int), ctx->stream));
    if (T == 0)
        return TSG_OK;
    unsigned int *keys;
    TSG_TRY(tsg_alloc(ctx, &keys, (size_t)T));
    unsigned grid = tsg_blocks(T, 256);
    k_csc_keys<<<grid, 256, 0, ctx->stream>>>(T, mat->tile_columnidx, keys, mat->csc_tile_pos, mat->csc_tile_ptr);
    TSG_LAUNCH_CHECK();
    TSG_TRY(tsg_scan_counts(ctx, mat->csc_tile_ptr, mat->csc_tile_ptr, tilen, nullptr));
    TSG_TRY(tsg_sort_pairs_u32(ctx, keys, mat->csc_tile_pos, T, bits_for(tilen)));
    k_csc_rows<<<grid, 256, 0, ctx->stream>>>(T, mat->csc_tile_pos, mat->tile_rowidx, mat->csc_tile_rowidx);
    TSG_LAUNCH_CHECK();
    tsg_release(ctx, keys);
    return TSG_OK;
}

// ---------------------------------------------------------------------------
// Column-major gather (the reference B layout): tile data reordered by the
// column view, Col bytes unpacked to plain columns.
// ---------------------------------------------------------------------------
__global__ void k_cm_counts(int T, const int *__restrict__ pos, const int *__restrict__ tnnz,
                            int *__restrict__ cnt)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < T; q += gridDim.x * blockDim.x)
    {
        int t = pos ? pos[q] : q;
        cnt[q] = tnnz[t + 1] - tnnz[t];
    }
}

// Half-warp per output tile q.
__global__ void k_cm_gather(int T, const int *__restrict__ pos, const int *__restrict__ tnnz_src,
                            const unsigned char *__restrict__ Ptr_src, const unsigned short *__restrict__ mask_src,
                            const unsigned char *__restrict__ Col_src, const double *__restrict__ Val_src,
                            const int *__restrict__ tnnz_dst, unsigned char *__restrict__ Ptr_dst,
                            unsigned short *__restrict__ mask_dst, unsigned char *__restrict__ Col_dst,
                            double *__restrict__ Val_dst)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int q = (int)(gid >> 4);
    const int lane = threadIdx.x & 15;
    if (q >= T)
        return;
    const int t = pos ? pos[q] : q;
    Ptr_dst[(long long)q * TSG_BS + lane] = Ptr_src[(long long)t * TSG_BS + lane];
    mask_dst[(long long)q * TSG_BS + lane] = mask_src[(long long)t * TSG_BS + lane];
    const int s = tnnz_src[t], n = tnnz_src[t + 1] - s, d = tnnz_dst[q];
    for (int i = lane; i < n; i += 16)
    {
        Col_dst[d + i] = Col_src[s + i] & 15;
        Val_dst[d + i] = Val_src[s + i];
    }
}

// ---------------------------------------------------------------------------
// Tiles -> CSR (src/tile2csr.h:8-137).  Half-warp per tile row, lane = row.
// Row r of a tile spans [Ptr[r], Ptr[r+1]); the last real row of the tile
// row ends at the tile nnz.
// ---------------------------------------------------------------------------
__global__ void k_t2c_rowlen(int m, int tilem, const int *__restrict__ tile_ptr,
                             const int *__restrict__ tnnz, const unsigned char *__restrict__ Ptr,
                             int *__restrict__ rowlen)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int tr = (int)(gid >> 4);
    const int lane = threadIdx.x & 15;
    if (tr >= tilem)
        return;
    const int rows = tr == tilem - 1 ? m - (tilem - 1) * TSG_BS : TSG_BS;
    if (lane >= rows)
        return;
    int sum = 0;
    for (int t = tile_ptr[tr]; t < tile_ptr[tr + 1]; t++)
    {
        const int s = Ptr[(long long)t * TSG_BS + lane];
        const int e = lane == rows - 1 ? tnnz[t + 1] - tnnz[t] : Ptr[(long long)t * TSG_BS + lane + 1];
        sum += e - s;
    }
    rowlen[tr * TSG_BS + lane] = sum;
}

__global__ void k_t2c_fill(int m, int tilem, const int *__restrict__ tile_ptr,
                           const int *__restrict__ tile_col, const int *__restrict__ tnnz,
                           const unsigned char *__restrict__ Ptr, const unsigned char *__restrict__ Col,
                           const double *__restrict__ Val, const int *__restrict__ rowptr,
                           int *__restrict__ ccol, double *__restrict__ cval)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int tr = (int)(gid >> 4);
    const int lane = threadIdx.x & 15;
    if (tr >= tilem)
        return;
    const int rows = tr == tilem - 1 ? m - (tilem - 1) * TSG_BS : TSG_BS;
    if (lane >= rows)
        return;
    int off = rowptr[tr * TSG_BS + lane];
    for (int t = tile_ptr[tr]; t < tile_ptr[tr + 1]; t++)
    {
        const int s = Ptr[(long long)t * TSG_BS + lane];
        const int e = lane == rows - 1 ? tnnz[t + 1] - tnnz[t] : Ptr[(long long)t * TSG_BS + lane + 1];
        const int base = tnnz[t];
        const int cb = tile_col[t] * TSG_BS;
        for (int q = s; q < e; q++)
        {
            ccol[off] = cb + Col[base + q];
            cval[off] = Val[base + q];
            off++;
        }
    }
}

extern "C" int tsg_tiled_to_csr(tsg_context *ctx, const tsg_tiled *C, int *d_rowptr, int *d_colidx,
                                double *d_val)
{
    if (!ctx || !C || !d_rowptr)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    const int m = C->m, tilem = C->tilem;
    if (m == 0)
    {
        TSG_CUDA(cudaMemsetAsync(d_rowptr, 0, sizeof(int), ctx->stream));
        return TSG_OK;
    }
    k_t2c_rowlen<<<tsg_blocks((long long)tilem * 16, 256), 256, 0, ctx->stream>>>(
        m, tilem, C->tile_ptr, C->tile_nnz, C->tile_csr_Ptr, d_rowptr);
    TSG_LAUNCH_CHECK();
    TSG_TRY(tsg_scan_counts(ctx, d_rowptr, d_rowptr, m, nullptr));
    k_t2c_fill<<<tsg_blocks((long long)tilem * 16, 256), 256, 0, ctx->stream>>>(
        m, tilem, C->tile_ptr, C->tile_columnidx, C->tile_nnz, C->tile_csr_Ptr, C->tile_csr_Col,
        C->tile_csr_Value, d_rowptr, d_colidx, d_val);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}

// Column-major download helper used by tsg_tiled_download (tsg_api.cu).
int tsg_gather_colmajor(tsg_context *ctx, const tsg_tiled *src, int *tnnz_cm, unsigned char *Ptr_cm,
                        unsigned short *mask_cm, unsigned char *Col_cm, double *Val_cm)
{
    const int T = src->numtile;
    if (T == 0)
    {
        TSG_CUDA(cudaMemsetAsync(tnnz_cm, 0, sizeof(int), ctx->stream));
        return TSG_OK;
    }
    unsigned grid = tsg_blocks(T, 256);
    k_cm_counts<<<grid, 256, 0, ctx->stream>>>(T, src->csc_tile_pos, src->tile_nnz, tnnz_cm);
    TSG_LAUNCH_CHECK();
    TSG_TRY(tsg_scan_counts(ctx, tnnz_cm, tnnz_cm, T, nullptr));
    k_cm_gather<<<tsg_blocks((long long)T * 16, 256), 256, 0, ctx->stream>>>(
        T, src->csc_tile_pos, src->tile_nnz, src->tile_csr_Ptr, src->mask, src->tile_csr_Col,
        src->tile_csr_Value, tnnz_cm, Ptr_cm, mask_cm, Col_cm, Val_cm);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}

// ---------------------------------------------------------------------------
// Column-major tile data (the reference's B layout) -> the library's layout:
// row-major tile data plus the column view (csc_tile_pos[q] = row-major
// index of column-major tile q).
// ---------------------------------------------------------------------------
// warp per tile column: row-major index of every tile of the column
__global__ void k_cm_rowpos(int tilen, const int *__restrict__ cptr, const int *__restrict__ crow,
                            const int *__restrict__ tile_ptr, const int *__restrict__ tile_col, int *__restrict__ pos)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= tilen)
        return;
    const int j = (int)w;
    for (int q = cptr[j] + lane; q < cptr[j + 1]; q += 32)
    {
        const int R = crow[q];
        int lo = tile_ptr[R], n = tile_ptr[R + 1] - lo;
        while (n > 0)
        {
            const int h = n >> 1;
            if (tile_col[lo + h] < j)
            {
                lo += h + 1;
                n -= h + 1;
            }
            else
                n = h;
        }
        pos[q] = lo;
    }
}

__global__ void k_cm_rm_counts(int T, const int *__restrict__ pos, const int *__restrict__ tnnz_cm, int *__restrict__ cnt)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < T; q += gridDim.x * blockDim.x)
        cnt[pos[q]] = tnnz_cm[q + 1] - tnnz_cm[q];
}

// half-warp per column-major tile q, scattered to row-major slot pos[q]
__global__ void k_cm_rm_scatter(int T, const int *__restrict__ pos, const int *__restrict__ tnnz_cm,
                                const unsigned char *__restrict__ Ptr_cm, const unsigned short *__restrict__ mask_cm,
                                const unsigned char *__restrict__ Col_cm, const double *__restrict__ Val_cm,
                                const int *__restrict__ tnnz_rm, unsigned char *__restrict__ Ptr_rm,
                                unsigned short *__restrict__ mask_rm, unsigned char *__restrict__ Col_rm,
                                double *__restrict__ Val_rm)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int q = (int)(gid >> 4);
    const int lane = threadIdx.x & 15;
    if (q >= T)
        return;
    const int p = pos[q];
    Ptr_rm[(long long)p * TSG_BS + lane] = Ptr_cm[(long long)q * TSG_BS + lane];
    mask_rm[(long long)p * TSG_BS + lane] = mask_cm[(long long)q * TSG_BS + lane];
    const int s = tnnz_cm[q], n = tnnz_cm[q + 1] - s, d = tnnz_rm[p];
    for (int i = lane; i < n; i += 16)
    {
        Col_rm[d + i] = Col_cm[s + i];
        Val_rm[d + i] = Val_cm[s + i];
    }
}

__global__ void k_rowidx_from_ptr(int tilem, const int *__restrict__ tile_ptr, int *__restrict__ rowidx)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= tilem)
        return;
    for (int t = tile_ptr[w] + lane; t < tile_ptr[w + 1]; t += 32)
        rowidx[t] = (int)w;
}

// mat holds column-major data (tile_nnz, Ptr, mask, Col, Value in csc order),
// row-major tile_ptr / tile_columnidx and csc_tile_ptr / csc_tile_rowidx.
int tsg_colmajor_data_to_rowmajor(tsg_context *ctx, tsg_tiled *mat)
{
    const int T = mat->numtile;
    cudaStream_t st = ctx->stream;
    TSG_TRY(tsg_alloc(ctx, &mat->csc_tile_pos, (size_t)T));
    int *tnnz, *rowidx;
    unsigned char *Ptr, *Col;
    unsigned short *mask;
    double *Val;
    TSG_TRY(tsg_alloc(ctx, &tnnz, (size_t)T + 1));
    TSG_TRY(tsg_alloc(ctx, &rowidx, (size_t)T));
    TSG_TRY(tsg_alloc(ctx, &Ptr, (size_t)T * TSG_BS));
    TSG_TRY(tsg_alloc(ctx, &mask, (size_t)T * TSG_BS));
    TSG_TRY(tsg_alloc(ctx, &Col, (size_t)mat->nnz));
    TSG_TRY(tsg_alloc(ctx, &Val, (size_t)mat->nnz));
    if (T > 0)
    {
        k_cm_rowpos<<<tsg_blocks((long long)mat->tilen * 32, 256), 256, 0, st>>>(
            mat->tilen, mat->csc_tile_ptr, mat->csc_tile_rowidx, mat->tile_ptr, mat->tile_columnidx, mat->csc_tile_pos);
        TSG_LAUNCH_CHECK();
        k_cm_rm_counts<<<tsg_blocks(T, 256), 256, 0, st>>>(T, mat->csc_tile_pos, mat->tile_nnz, tnnz);
        TSG_LAUNCH_CHECK();
        TSG_TRY(tsg_scan_counts(ctx, tnnz, tnnz, T, nullptr));
        k_cm_rm_scatter<<<tsg_blocks((long long)T * 16, 256), 256, 0, st>>>(
            T, mat->csc_tile_pos, mat->tile_nnz, mat->tile_csr_Ptr, mat->mask, mat->tile_csr_Col, mat->tile_csr_Value,
            tnnz, Ptr, mask, Col, Val);
        TSG_LAUNCH_CHECK();
        k_rowidx_from_ptr<<<tsg_blocks((long long)mat->tilem * 32, 256), 256, 0, st>>>(mat->tilem, mat->tile_ptr, rowidx);
        TSG_LAUNCH_CHECK();
    }
    else
        TSG_CUDA(cudaMemsetAsync(tnnz, 0, sizeof(int), st));
    tsg_release(ctx, mat->tile_nnz);
    tsg_release(ctx, mat->tile_rowidx);
    tsg_release(ctx, mat->tile_csr_Ptr);
    tsg_release(ctx, mat->mask);
    tsg_release(ctx, mat->tile_csr_Col);
    tsg_release(ctx, mat->tile_csr_Value);
    mat->tile_nnz = tnnz;
    mat->tile_rowidx = rowidx;
    mat->tile_csr_Ptr = Ptr;
    mat->mask = mask;
    mat->tile_csr_Col = Col;
    mat->tile_csr_Value = Val;
    TSG_TRY(tsg_build_mask_t(ctx, mat));
    return tsg_build_row_view(ctx, mat);
}
