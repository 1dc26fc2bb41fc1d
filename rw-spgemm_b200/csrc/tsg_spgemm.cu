// Tiled SpGEMM C = A*B on 16x16 tiles, FP64, for sm_100a: one product.
//
// The per-item device code lives in tsg_device.cuh (shared with the batched
// persistent kernel of tsg_batch.cu); this file holds the one-product kernels
// and the host orchestration of tsg_spgemm:
//   step 1  count (warp per A tile row) -> scan -> emit sorted C tile columns
//   step 2  masks / row offsets / nnz per C tile -> scan of tile nnz
//   step 3  values and column bytes
// Steps 2 and 3 run in one of two work schedules with bit-identical results:
// the tile schedule (half-warp per C tile, A-row x B-column intersection, as
// the reference decomposes the work) or the row-segment schedule (half-warp
// per run of C tiles in one tile row, tile-level Gustavson, no intersection).
#include <algorithm>

#include "tsg_device.cuh"
#include "tsg_staged.cuh"

#define S1_WARPS 8

template <bool EMIT>
__global__ void __launch_bounds__(S1_WARPS * 32) k_step1(ProdView P, int *__restrict__ C_cnt,
                                                         unsigned long long *__restrict__ pairs)
{
    __shared__ unsigned int s_bm[S1_WARPS][S1_WORDS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * S1_WARPS + warp;
    if (i >= P.tilemA)
        return;
    const int cnt = step1_row<EMIT>(P, i, s_bm[warp], lane, pairs);
    if (!EMIT && lane == 0)
        C_cnt[i] = cnt;
}

// step 1's count pass summed over the block into one device word
__global__ void __launch_bounds__(S1_WARPS * 32) k_step1_total(ProdView P, unsigned long long *__restrict__ total)
{
    __shared__ unsigned int s_bm[S1_WARPS][S1_WORDS];
    __shared__ int s_cnt[S1_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * S1_WARPS + warp;
    const int cnt = i < P.tilemA ? step1_row<false>(P, i, s_bm[warp], lane, nullptr) : 0;
    if (lane == 0)
        s_cnt[warp] = cnt;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        unsigned long long sum = 0;
        for (int w = 0; w < S1_WARPS; w++)
            sum += (unsigned long long)s_cnt[w];
        if (sum)
            atomicAdd(total, sum);
    }
}

// fused step-1 emit + step 2 (warp per A tile row); wide rows are emitted by
// step1_row and flagged for the wide-row step 2 (1, or 2 when hypersparse)
__global__ void __launch_bounds__(256) k_step12(ProdView P, int *__restrict__ wide, int *__restrict__ bins)
{
    __shared__ S12Smem sm[8];
    __shared__ int s_bins[4];
    if (threadIdx.x < 4)
        s_bins[threadIdx.x] = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * 8 + warp;
    if (i < P.tilemA)
    {
        const int done = step12_row(P, i, sm[warp], lane, s_bins);
        int kind = 0;
        if (!done)
        {
            static_assert(sizeof(S12Smem) >= S1_WORDS * sizeof(unsigned), "bitmap scratch");
            __syncwarp();
            step1_row<true>(P, i, reinterpret_cast<unsigned *>(&sm[warp]), lane, nullptr);
            __syncwarp(); // the row's C columns, emitted by all lanes
            kind = wide_kind(P, i, lane);
        }
        if (lane == 0)
        {
            wide[i] = kind;
            if (kind)
                atomicAdd(&wide[P.tilemA], 1); // count of wide rows
            if (kind == 2)
                atomicAdd(&wide[P.tilemA + 1], 1); // count of hypersparse rows
        }
    }
    __syncthreads();
    if (threadIdx.x < 4 && s_bins[threadIdx.x])
        atomicAdd(&bins[threadIdx.x], s_bins[threadIdx.x]);
}

// step 2 (tile schedule) for the C tiles of rows k_step12 left to it
__global__ void __launch_bounds__(256) k_step2_wide(ProdView P, const int *__restrict__ wide, int *__restrict__ bins)
{
    __shared__ int s_bins[4];
    if (threadIdx.x < 4)
        s_bins[threadIdx.x] = 0;
    __syncthreads();
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    if (t < P.numC && wide[P.C_row[t]])
        step2_tile(P, (int)t, TSG_HW_MASK(threadIdx.x), threadIdx.x & 15, s_bins);
    __syncthreads();
    if (threadIdx.x < 4 && s_bins[threadIdx.x])
        atomicAdd(&bins[threadIdx.x], s_bins[threadIdx.x]);
}

// scalar step 2 for the wide rows k_step12 left: CTAs take blocks of C tiles
// from a device counter and run the wide rows' parts
__global__ void __launch_bounds__(SPA_THREADS) k_step2_spa(ProdView P, const int *__restrict__ wide,
                                                           unsigned *__restrict__ ctr, int *__restrict__ bins)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    Spa2Smem &S = *reinterpret_cast<Spa2Smem *>(s_raw);
    __shared__ int s_bins[4];
    __shared__ int s_blk;
    if (wide[P.tilemA] == 0) // no wide row (k_step12 counted them)
        return;
    if (threadIdx.x < 4)
        s_bins[threadIdx.x] = 0;
    unsigned nxt = 0; // thread 0: the next block, claimed one block ahead
    if (threadIdx.x == 0)
        nxt = atomicAdd(ctr, 1u);
    for (;;)
    {
        __syncthreads();
        if (threadIdx.x == 0)
        {
            s_blk = (int)nxt;
            nxt = atomicAdd(ctr, 1u);
        }
        __syncthreads();
        const long long tb = (long long)s_blk * SPA_BLK;
        if (tb >= P.numC)
            break;
        if (threadIdx.x == 0)
            spa_skip_hyper(P, wide, (int)tb, ctr, 0);
        step2_spa_block(P, S, (int)tb, (int)min((long long)P.numC, tb + SPA_BLK), wide, s_bins);
    }
    __syncthreads();
    if (threadIdx.x < 4 && s_bins[threadIdx.x])
        atomicAdd(&bins[threadIdx.x], s_bins[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_step2(ProdView P, int *__restrict__ bins)
{
    __shared__ int s_bins[4];
    if (threadIdx.x < 4)
        s_bins[threadIdx.x] = 0;
    __syncthreads();
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    if (t < P.numC)
        step2_tile(P, (int)t, TSG_HW_MASK(threadIdx.x), threadIdx.x & 15, s_bins);
    __syncthreads();
    if (threadIdx.x < 4 && s_bins[threadIdx.x])
        atomicAdd(&bins[threadIdx.x], s_bins[threadIdx.x]);
}

#define S3_THREADS 256
#define S3_HW (S3_THREADS / 16)

__global__ void __launch_bounds__(S3_THREADS) k_step3(ProdView P)
{
    __shared__ double s_acc[S3_HW][TSG_BS * S3T_STRIDE];
    const int hw = threadIdx.x >> 4, lane = threadIdx.x & 15;
    const unsigned hmask = TSG_HW_MASK(threadIdx.x);
    double *acc = s_acc[hw];
    for (int q = lane; q < TSG_BS * S3T_STRIDE; q += 16)
        acc[q] = 0.0;
    __syncwarp(hmask);
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    if (t < P.numC)
        step3_tile(P, (int)t, hmask, lane, acc);
}

__global__ void __launch_bounds__(256) k_step3_elems(ProdView P)
{
    __shared__ int2 s_pairs[8][S3E_PAIRS];
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t < P.numC)
        step3_elems_tile(P, (int)t, s_pairs[threadIdx.x >> 5]);
}

template <int W>
__global__ void __launch_bounds__(128) k_step2_rows(ProdView P, int *__restrict__ bins)
{
    __shared__ S2RowsSmem<W> sm[8];
    __shared__ int s_bins[4];
    if (threadIdx.x < 4)
        s_bins[threadIdx.x] = 0;
    __syncthreads();
    const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    step2_rows_item<W>(P, item, TSG_HW_MASK(threadIdx.x), threadIdx.x & 15, sm[threadIdx.x >> 4], s_bins);
    __syncthreads();
    if (threadIdx.x < 4 && s_bins[threadIdx.x])
        atomicAdd(&bins[threadIdx.x], s_bins[threadIdx.x]);
}

template <int W, int CAP>
__global__ void __launch_bounds__(128) k_step3_rows(ProdView P)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    S3RowsSmem<W, CAP> *sm = reinterpret_cast<S3RowsSmem<W, CAP> *>(s_raw);
    const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    step3_rows_item<W, CAP>(P, item, TSG_HW_MASK(threadIdx.x), threadIdx.x & 15, sm[threadIdx.x >> 4]);
}

// persistent: CTAs take blocks of C tiles from a device counter; kind (may
// be null) marks the hypersparse rows (2), each done whole.  RANGED: only
// the tile rows [row0, row1) are done -- the blocks holding their tiles, each
// clamped to those tiles (a separate instantiation keeps the whole-product
// form's registers).
template <bool FLAT, bool RANGED, int BLK>
__global__ void __launch_bounds__(SPA_THREADS, 3) k_step3_spa(ProdView P, const int *__restrict__ kind, int row0,
                                                              int row1, unsigned *__restrict__ ctr)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    SpaSmem &S = *reinterpret_cast<SpaSmem *>(s_raw);
    __shared__ int s_blk;
    unsigned nxt = 0; // thread 0: the next block, claimed one block ahead
    if (threadIdx.x == 0)
        nxt = atomicAdd(ctr, 1u);
    const int t_beg = RANGED ? P.C_ptr[row0] : 0, t_end = RANGED ? P.C_ptr[row1] : P.numC;
    const long long blk0 = t_beg / BLK;
    for (;;)
    {
        __syncthreads();
        if (threadIdx.x == 0)
        {
            s_blk = (int)nxt;
            nxt = atomicAdd(ctr, 1u);
        }
        __syncthreads();
        const long long tb = (blk0 + s_blk) * BLK;
        if (tb >= t_end)
            break;
        if (threadIdx.x == 0)
            spa_skip_hyper<BLK>(P, kind, (int)tb, ctr, -blk0);
        // the block, clamped to the tiles of rows [row0, row1)
        step3_spa_block<FLAT, BLK>(P, S, max((int)tb, t_beg), (int)min((long long)t_end, tb + BLK), kind);
    }
}

// The tile rows the staged numeric step left (left[I] != 0: its stage would
// not fit, or the row is hypersparse), by the SPA kernel; nothing unless it
// left some (left[tilemA]).
template <bool RANGED>
__global__ void __launch_bounds__(SPA_THREADS, 2) k_step3_rest(ProdView P, const int *__restrict__ kind,
                                                               const int *__restrict__ left, int row0, int row1,
                                                               unsigned *__restrict__ ctr)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    SpaSmem &S = *reinterpret_cast<SpaSmem *>(s_raw);
    __shared__ int s_blk;
    if (left[P.tilemA] == 0)
        return;
    unsigned nxt = 0;
    if (threadIdx.x == 0)
        nxt = atomicAdd(ctr, 1u);
    const int t_beg = RANGED ? P.C_ptr[row0] : 0, t_end = RANGED ? P.C_ptr[row1] : P.numC;
    const long long blk0 = t_beg / SPA_BLK;
    for (;;)
    {
        __syncthreads();
        if (threadIdx.x == 0)
        {
            s_blk = (int)nxt;
            nxt = atomicAdd(ctr, 1u);
        }
        __syncthreads();
        const long long tb = (blk0 + s_blk) * SPA_BLK;
        if (tb >= t_end)
            break;
        if (threadIdx.x == 0)
            spa_skip_hyper(P, kind, (int)tb, ctr, -blk0);
        step3_spa_block<false>(P, S, max((int)tb, t_beg), (int)min((long long)t_end, tb + SPA_BLK), kind, left);
    }
}

// ---------------------------------------------------------------------------
// Host orchestration.
// ---------------------------------------------------------------------------
static int validate_operands(const tsg_tiled *A, const tsg_tiled *B)
{
    if (!A || !B)
        return tsg_set_error(TSG_ERR_INVALID, "null operand");
    if (A->n != B->m)
        return tsg_set_error(TSG_ERR_INVALID, "inner dimensions differ (A is %dx%d, B is %dx%d)", A->m,
                             A->n, B->m, B->n);
    if (!B->csc_tile_ptr || !B->csc_tile_rowidx)
        return tsg_set_error(TSG_ERR_INVALID, "B has no column view (build it with TSG_TILED_CSC_VIEW)");
    if (!A->tile_ptr || !B->tile_ptr)
        return tsg_set_error(TSG_ERR_INVALID, "operand without tile structure");
    return TSG_OK;
}

static float ev_ms(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

static ProdView make_view(const tsg_tiled *A, const tsg_tiled *B, tsg_tiled *C)
{
    ProdView P;
    P.A_ptr = A->tile_ptr;
    P.A_col = A->tile_columnidx;
    P.A_tnnz = A->tile_nnz;
    P.A_Ptr = A->tile_csr_Ptr;
    P.A_Colb = A->tile_csr_Col;
    P.A_Val = A->tile_csr_Value;
    P.A_mask = A->mask;
    P.tilemA = A->tilem;
    P.B_ptr = B->tile_ptr;
    P.B_col = B->tile_columnidx;
    P.B_cptr = B->csc_tile_ptr;
    P.B_crow = B->csc_tile_rowidx;
    P.B_cpos = B->csc_tile_pos;
    P.B_tnnz = B->tile_nnz;
    P.B_Ptr = B->tile_csr_Ptr;
    P.B_Colb = B->tile_csr_Col;
    P.B_Val = B->tile_csr_Value;
    P.B_mask = B->mask;
    P.B_maskT = B->mask_t;
    P.B_rptr = B->row_ptr;
    P.B_rcol = B->row_col;
    P.B_rval = B->row_val;
    P.browB = B->m > 0 ? (int)(B->nnz / B->m) : 0;
    P.tilenB = B->tilen;
    P.C_ptr = C->tile_ptr;
    P.C_col = C->tile_columnidx;
    P.C_row = C->tile_rowidx;
    P.C_tnnz = C->tile_nnz;
    P.C_mask = C->mask;
    P.C_Ptr = C->tile_csr_Ptr;
    P.C_Colb = C->tile_csr_Col;
    P.C_Val = C->tile_csr_Value;
    P.numC = C->numtile;
    // the staged numeric step copies ranges rounded out to 16-byte
    // boundaries: library allocations only (tsg_alloc's slack), 16-byte aligned
    const void *bases[] = {P.A_mask, P.A_Ptr, P.A_tnnz, P.A_col, P.A_Val, P.B_rcol, P.B_rval,
                           P.C_mask, P.C_Ptr, P.C_tnnz, P.C_col};
    bool aligned = true;
    for (const void *p : bases)
        aligned = aligned && ((uintptr_t)p & 15) == 0;
    P.padded = !A->_alloc && !B->_alloc && !C->_alloc && aligned;
    P.status = nullptr;
    return P;
}

template <int W, int CAP>
static int launch_step3_rows(tsg_context *ctx, const ProdView &P)
{
    const size_t smem = 8 * sizeof(S3RowsSmem<W, CAP>);
    TSG_CUDA(cudaFuncSetAttribute(k_step3_rows<W, CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long items = ((long long)P.numC + W - 1) / W;
    k_step3_rows<W, CAP><<<tsg_blocks(items * 16, 128), 128, smem, ctx->stream>>>(P);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}

template <int W>
static int launch_step2_rows(tsg_context *ctx, const ProdView &P, int *d_bins)
{
    const long long items = ((long long)P.numC + W - 1) / W;
    k_step2_rows<W><<<tsg_blocks(items * 16, 128), 128, 0, ctx->stream>>>(P, d_bins);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}

static int launch_step2(tsg_context *ctx, const ProdView &P, int *d_bins)
{
    if (ctx->sched == TSG_SCHED_ROWS)
    {
        if (ctx->seg_tiles == 32)
            return launch_step2_rows<32>(ctx, P, d_bins);
        if (ctx->seg_tiles == 16)
            return launch_step2_rows<16>(ctx, P, d_bins);
        return launch_step2_rows<8>(ctx, P, d_bins);
    }
    k_step2<<<tsg_blocks((long long)P.numC * 16, 256), 256, 0, ctx->stream>>>(P, d_bins);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}

// persistent grid of a SPA kernel: resident CTAs on every SM
template <typename K>
static int spa_grid(tsg_context *ctx, K kern, int smem, unsigned *grid)
{
    TSG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    TSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SPA_THREADS, smem));
    *grid = (unsigned)(ctx->num_sms * (per_sm > 0 ? per_sm : 1));
    return TSG_OK;
}

// step 2 for the rows k_step12 declined, through B's row view
static int launch_step2_spa(tsg_context *ctx, const ProdView &P, const int *d_wide, int *d_bins)
{
    unsigned *ctr = nullptr, grid = 0;
    const int smem = (int)sizeof(Spa2Smem);
    TSG_TRY(spa_grid(ctx, k_step2_spa, smem, &grid));
    TSG_TRY(tsg_alloc(ctx, &ctr, 1));
    TSG_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned), ctx->stream));
    k_step2_spa<<<grid, SPA_THREADS, smem, ctx->stream>>>(P, d_wide, ctr, d_bins);
    TSG_LAUNCH_CHECK();
    tsg_release(ctx, ctr);
    return TSG_OK;
}

template <bool FLAT, bool RANGED, int BLK = SPA_BLK>
static int launch_step3_spa(tsg_context *ctx, const ProdView &P0, const int *d_kind, int row0, int row1)
{
    ProdView P = P0;
    P.status = ctx->d_status;
    unsigned *ctr = nullptr, grid = 0;
    const int smem = (int)sizeof(SpaSmem);
    TSG_TRY(spa_grid(ctx, k_step3_spa<FLAT, RANGED, BLK>, smem, &grid));
    TSG_TRY(tsg_alloc(ctx, &ctr, 1));
    TSG_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned), ctx->stream));
    k_step3_spa<FLAT, RANGED, BLK><<<grid, SPA_THREADS, smem, ctx->stream>>>(P, d_kind, row0, row1, ctr);
    TSG_LAUNCH_CHECK();
    tsg_release(ctx, ctr);
    return TSG_OK;
}

// the staged numeric step for tile rows [row0, row1), then the SPA kernel
// for the rows it left
template <bool RANGED>
static int launch_step3_stg(tsg_context *ctx, const ProdView &P0, const int *d_kind, int row0, int row1)
{
    ProdView P = P0;
    P.status = ctx->d_status;
    unsigned *ctr = nullptr, grid = 0;
    int *left = nullptr;
    const int smem = (int)sizeof(StgSmem);
    TSG_CUDA(cudaFuncSetAttribute(k_step3_stg<RANGED>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    TSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step3_stg<RANGED>, STG_THREADS, smem));
    if (per_sm < 1)
        return tsg_set_error(TSG_ERR_CUDA, "the staged numeric step does not fit an SM");
    TSG_TRY(tsg_alloc(ctx, &ctr, 2));
    TSG_TRY(tsg_alloc(ctx, &left, (size_t)P.tilemA + 1));
    TSG_CUDA(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned), ctx->stream));
    TSG_CUDA(cudaMemsetAsync(left, 0, ((size_t)P.tilemA + 1) * sizeof(int), ctx->stream));
    k_step3_stg<RANGED><<<ctx->num_sms * per_sm, STG_THREADS, smem, ctx->stream>>>(P, d_kind, row0, row1, ctr, left,
                                                                                 ctx->d_status);
    TSG_LAUNCH_CHECK();
    const int rsmem = (int)sizeof(SpaSmem);
    TSG_TRY(spa_grid(ctx, k_step3_rest<RANGED>, rsmem, &grid));
    k_step3_rest<RANGED><<<grid, SPA_THREADS, rsmem, ctx->stream>>>(P, d_kind, left, row0, row1, ctr + 1);
    TSG_LAUNCH_CHECK();
    tsg_release(ctx, ctr);
    tsg_release(ctx, left);
    return TSG_OK;
}

// step 3 by the SPA kernel: the default schedule, except for products whose
// C tiles are dense on average (>= ctx->spa_dense values, SPA_DENSE unless
// set) and B without a row view (borrowed foreign buffers), which take the
// tile kernel
static bool step3_by_spa(const tsg_context *ctx, const ProdView &P, long long nnzC)
{
    return ctx->sched == TSG_SCHED_SPA && P.B_rptr && nnzC < (long long)ctx->spa_dense * P.numC;
}

// the SPA numeric step for tile rows [row0, row1)
static int launch_step3_spa_rows(tsg_context *ctx, const ProdView &P, long long nnzC, const int *d_kind, int row0,
                                 int row1)
{
    const bool flat = spa_wants_flat(P.browB, P.numC, nnzC, P.tilemA);
    const bool whole = row0 == 0 && row1 == P.tilemA;
    ctx->last_step3 = flat ? TSG_STEP3_FLAT : P.padded ? TSG_STEP3_STAGED : TSG_STEP3_SPA;
    if (flat && nnzC >= (long long)SPA_BLK_NARROW_VALUES * P.numC)
        return whole ? launch_step3_spa<true, false, SPA_BLK_NARROW>(ctx, P, d_kind, 0, 0)
                     : launch_step3_spa<true, true, SPA_BLK_NARROW>(ctx, P, d_kind, row0, row1);
    if (flat)
        return whole ? launch_step3_spa<true, false>(ctx, P, d_kind, 0, 0)
                     : launch_step3_spa<true, true>(ctx, P, d_kind, row0, row1);
    if (P.padded)
        return whole ? launch_step3_stg<false>(ctx, P, d_kind, 0, 0) : launch_step3_stg<true>(ctx, P, d_kind, row0, row1);
    // operands viewing a batch arena: not padded for the bulk copies' rounding
    return whole ? launch_step3_spa<false, false>(ctx, P, d_kind, 0, 0)
                 : launch_step3_spa<false, true>(ctx, P, d_kind, row0, row1);
}

// d_kind: the row kinds of the fused step 1/2 pass (0 narrow, 1 wide,
// 2 hypersparse), or null
static int launch_step3(tsg_context *ctx, const ProdView &P, long long nnzC, const int *d_kind)
{
    if (step3_by_spa(ctx, P, nnzC))
        return launch_step3_spa_rows(ctx, P, nnzC, d_kind, 0, P.tilemA);
    if (ctx->sched == TSG_SCHED_ROWS)
    {
        const int W = ctx->seg_tiles, cap = ctx->acc_cap;
        ctx->last_step3 = TSG_STEP3_ROWS;
#define TSG_DISPATCH3(w, c)                    \
    if (W == w && cap == c)                    \
        return launch_step3_rows<w, c>(ctx, P);
        TSG_ROW_CONFIGS(TSG_DISPATCH3)
#undef TSG_DISPATCH3
        return tsg_set_error(TSG_ERR_INVALID, "unsupported row schedule (%d, %d)", W, cap);
    }
    if (ctx->sched == TSG_SCHED_ELEMS)
    {
        if (!P.B_maskT)
            return tsg_set_error(TSG_ERR_INVALID, "element schedule needs B's column masks (mask_t)");
        ctx->last_step3 = TSG_STEP3_ELEMS;
        k_step3_elems<<<tsg_blocks((long long)P.numC * 32, 256), 256, 0, ctx->stream>>>(P);
        TSG_LAUNCH_CHECK();
        return TSG_OK;
    }
    ctx->last_step3 = TSG_STEP3_TILES;
    k_step3<<<tsg_blocks((long long)P.numC * 16, S3_THREADS), S3_THREADS, 0, ctx->stream>>>(P);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}

// What steps 1-2 leave for step 3 and the statistics.
struct SpgemmRun
{
    unsigned long long *d_pairs;
    int *d_bins;
    int *d_wide; // row kinds of the fused pass, or null
    long long numC, nnzC;
};

// Steps 1 and 2 of C = A*B: on return C's tile structure, masks, row offsets
// and tile value offsets are final, nnz(C) is known on the host and C's value
// arrays are allocated.  Records ev[0..2] when timing.
static int spgemm_structure(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B, tsg_tiled *C, SpgemmRun &R)
{
    memset(&R, 0, sizeof(R));
    memset(C, 0, sizeof(*C));
    C->m = A->m;
    C->n = B->n;
    C->tilem = A->tilem;
    C->tilen = B->tilen;
    C->col_packed = 0;
    const int tilem = C->tilem;
    cudaStream_t st = ctx->stream;
    const int timing = ctx->timing;
    if (timing)
        TSG_CUDA(cudaEventRecord(ctx->ev[0], st));

    // step 1: structure
    TSG_TRY(tsg_alloc(ctx, &R.d_pairs, 1));
    TSG_TRY(tsg_alloc(ctx, &R.d_bins, 4));
    TSG_CUDA(cudaMemsetAsync(R.d_pairs, 0, sizeof(unsigned long long), st));
    TSG_CUDA(cudaMemsetAsync(R.d_bins, 0, 4 * sizeof(int), st));
    TSG_TRY(tsg_alloc(ctx, &C->tile_ptr, (size_t)tilem + 1));
    long long numC = 0;
    if (tilem > 0)
    {
        ProdView P = make_view(A, B, C);
        k_step1<false><<<tsg_blocks(tilem, S1_WARPS), S1_WARPS * 32, 0, st>>>(P, C->tile_ptr, R.d_pairs);
        TSG_LAUNCH_CHECK();
        TSG_TRY(tsg_scan_counts(ctx, C->tile_ptr, C->tile_ptr, tilem, &numC));
    }
    else
        TSG_CUDA(cudaMemsetAsync(C->tile_ptr, 0, sizeof(int), st));
    C->numtile = (int)numC;
    R.numC = numC;
    TSG_TRY(tsg_alloc(ctx, &C->tile_columnidx, (size_t)numC));
    TSG_TRY(tsg_alloc(ctx, &C->tile_rowidx, (size_t)numC));
    TSG_TRY(tsg_alloc(ctx, &C->mask, (size_t)numC * TSG_BS));
    TSG_TRY(tsg_alloc(ctx, &C->tile_csr_Ptr, (size_t)numC * TSG_BS));
    TSG_TRY(tsg_alloc(ctx, &C->tile_nnz, (size_t)numC + 1));
    long long nnzC = 0;
    const bool fused = ctx->fuse12 && ctx->sched != TSG_SCHED_ROWS;
    if (numC > 0)
    {
        ProdView P = make_view(A, B, C);
        if (fused)
        {
            TSG_TRY(tsg_alloc(ctx, &R.d_wide, (size_t)tilem + 2));
            TSG_CUDA(cudaMemsetAsync(R.d_wide + tilem, 0, 2 * sizeof(int), st));
            k_step12<<<tsg_blocks(tilem, 8), 256, 0, st>>>(P, R.d_wide, R.d_bins);
            TSG_LAUNCH_CHECK();
        }
        else
        {
            k_step1<true><<<tsg_blocks(tilem, S1_WARPS), S1_WARPS * 32, 0, st>>>(P, nullptr, nullptr);
            TSG_LAUNCH_CHECK();
        }
    }
    if (timing)
        TSG_CUDA(cudaEventRecord(ctx->ev[1], st));

    // step 2: symbolic (rows the fused kernel left, or all tiles)
    if (numC > 0)
    {
        ProdView P = make_view(A, B, C);
        if (fused && P.B_rptr)
            TSG_TRY(launch_step2_spa(ctx, P, R.d_wide, R.d_bins));
        else if (fused)
        {
            k_step2_wide<<<tsg_blocks(numC * 16, 256), 256, 0, st>>>(P, R.d_wide, R.d_bins);
            TSG_LAUNCH_CHECK();
        }
        else
            TSG_TRY(launch_step2(ctx, P, R.d_bins));
        TSG_TRY(tsg_scan_counts(ctx, C->tile_nnz, C->tile_nnz, numC, &nnzC));
    }
    else
        TSG_CUDA(cudaMemsetAsync(C->tile_nnz, 0, sizeof(int), st));
    C->nnz = (int)nnzC;
    if (timing)
        TSG_CUDA(cudaEventRecord(ctx->ev[2], st));

    R.nnzC = nnzC;
    // C's value arrays
    TSG_TRY(tsg_alloc(ctx, &C->tile_csr_Col, (size_t)nnzC));
    TSG_TRY(tsg_alloc(ctx, &C->tile_csr_Value, (size_t)nnzC));
    return TSG_OK;
}

// Statistics of a product (tile pairs, bins, step times from ev[0..3]) and
// the release of the steps' scratch.
static int spgemm_finish(tsg_context *ctx, SpgemmRun &R, tsg_spgemm_info *info)
{
    cudaStream_t st = ctx->stream;
    tsg_release(ctx, R.d_wide);
    R.d_wide = nullptr;
    {
        const int dev = tsg_take_device_status(ctx);
        if (dev != TSG_OK)
        {
            tsg_release(ctx, R.d_pairs);
            tsg_release(ctx, R.d_bins);
            return dev;
        }
    }
    if (info)
    {
        memset(info, 0, sizeof(*info));
        info->numtile_C = R.numC;
        info->nnz_C = R.nnzC;
        long long *h = ctx->h_pinned;
        TSG_CUDA(cudaMemcpyAsync(h, R.d_pairs, sizeof(long long), cudaMemcpyDeviceToHost, st));
        TSG_CUDA(cudaMemcpyAsync(h + 1, R.d_bins, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
        TSG_CUDA(cudaStreamSynchronize(st));
        info->tile_pairs = h[0];
        memcpy(info->bins, h + 1, 4 * sizeof(int));
        info->step3_kernel = R.nnzC > 0 ? ctx->last_step3 : TSG_STEP3_NONE;
        if (ctx->timing)
        {
            info->ms_step1 = ev_ms(ctx->ev[0], ctx->ev[1]);
            info->ms_step2 = ev_ms(ctx->ev[1], ctx->ev[2]);
            info->ms_step3 = ev_ms(ctx->ev[2], ctx->ev[3]);
            info->ms_total = ev_ms(ctx->ev[0], ctx->ev[3]);
        }
    }
    tsg_release(ctx, R.d_pairs);
    tsg_release(ctx, R.d_bins);
    return TSG_OK;
}

extern "C" int tsg_spgemm(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B, tsg_tiled *C,
                          tsg_spgemm_info *info)
{
    if (!ctx || !C)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    TSG_TRY(validate_operands(A, B));
    SpgemmRun R;
    TSG_TRY(spgemm_structure(ctx, A, B, C, R));
    // step 3: numeric
    if (R.nnzC > 0)
        TSG_TRY(launch_step3(ctx, make_view(A, B, C), R.nnzC, R.d_wide));
    if (ctx->timing)
        TSG_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
    return spgemm_finish(ctx, R, info);
}

__global__ void k_t2c_rowlen(int m, int tilem, const int *__restrict__ tile_ptr, const int *__restrict__ tnnz,
                             const unsigned char *__restrict__ Ptr, int *__restrict__ rowlen);
__global__ void k_t2c_fill(int m, int tilem, const int *__restrict__ tile_ptr, const int *__restrict__ tile_col,
                           const int *__restrict__ tnnz, const unsigned char *__restrict__ Ptr,
                           const unsigned char *__restrict__ Col, const double *__restrict__ Val,
                           const int *__restrict__ rowptr, int *__restrict__ ccol, double *__restrict__ cval);

// C = A*B straight into host CSR buffers, the copy overlapping the numeric
// step.  After step 2 the row pointer of C is final: it is computed and
// copied first, so the host knows where every tile row's entries go.  Then
// the tile rows of C are taken in chunks of about equal nonzeros: a chunk's
// numeric step (the SPA kernel over its rows) and its CSR fill run on the
// context's stream while the previous chunks' column indices and values are
// copied out on the copy stream.  Products whose step 3 is not the SPA
// kernel run it whole first; their fill and copy are still chunked.
int tsg_spgemm_to_host(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B, int *h_rowptr, int *h_colidx,
                       double *h_val, long long nnz_cap, int *nnzC_out, tsg_spgemm_info *info)
{
    TSG_TRY(validate_operands(A, B));
    tsg_tiled C;
    SpgemmRun R;
    int status = spgemm_structure(ctx, A, B, &C, R);
    int *d_rp = nullptr, *d_ci = nullptr;
    double *d_v = nullptr;
    cudaStream_t st = ctx->stream;
    const int m = C.m, tilem = C.tilem;
    if (status == TSG_OK)
    {
        *nnzC_out = R.nnzC > INT_MAX ? INT_MAX : (int)R.nnzC; // the scan rejects more than 32-bit offsets
        if (R.nnzC > nnz_cap)
            status = tsg_set_error(TSG_ERR_OVERFLOW, "C has %lld nonzeros; the output buffers hold %lld", R.nnzC,
                                   nnz_cap);
    }
    if (status == TSG_OK)
        status = tsg_alloc(ctx, &d_rp, (size_t)m + 1);
    if (status == TSG_OK)
        status = tsg_alloc(ctx, &d_ci, (size_t)R.nnzC);
    if (status == TSG_OK)
        status = tsg_alloc(ctx, &d_v, (size_t)R.nnzC);
    if (status == TSG_OK)
        status = ([&]() -> int {
            // row pointer, to the host first
            if (m > 0)
            {
                k_t2c_rowlen<<<tsg_blocks((long long)tilem * 16, 256), 256, 0, st>>>(m, tilem, C.tile_ptr, C.tile_nnz,
                                                                                   C.tile_csr_Ptr, d_rp);
                TSG_LAUNCH_CHECK();
                TSG_TRY(tsg_scan_counts(ctx, d_rp, d_rp, m, nullptr));
            }
            else
                TSG_CUDA(cudaMemsetAsync(d_rp, 0, sizeof(int), st));
            TSG_CUDA(cudaMemcpyAsync(h_rowptr, d_rp, ((size_t)m + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
            TSG_CUDA(cudaStreamSynchronize(st));
            if (R.nnzC == 0 || tilem == 0)
                return TSG_OK;
            TSG_TRY(tsg_copy_stream(ctx));
            const ProdView P = make_view(A, B, &C);
            const bool spa = step3_by_spa(ctx, P, R.nnzC);
            if (!spa)
                TSG_TRY(launch_step3(ctx, P, R.nnzC, R.d_wide));
            // chunks of about equal nonzeros (>= TSG_CHUNK_NNZ each, at most TSG_MAX_CHUNKS)
            const long long nch = std::max(1LL, std::min((long long)TSG_MAX_CHUNKS, R.nnzC / TSG_CHUNK_NNZ));
            int r0 = 0;
            for (long long c = 1; c <= nch; c++)
            {
                int r1 = tilem;
                if (c < nch)
                {
                    // first tile row whose entries start at or after c / nch of C's
                    const long long want = R.nnzC * c / nch;
                    int lo = r0 + 1, hi = tilem;
                    while (lo < hi)
                    {
                        const int mid = (lo + hi) >> 1;
                        if ((long long)h_rowptr[(long long)mid * TSG_BS] >= want)
                            hi = mid;
                        else
                            lo = mid + 1;
                    }
                    r1 = lo;
                }
                if (r1 <= r0)
                    continue;
                if (spa)
                    TSG_TRY(launch_step3_spa_rows(ctx, P, R.nnzC, R.d_wide, r0, r1));
                const int rows = std::min(m, r1 * TSG_BS) - r0 * TSG_BS;
                k_t2c_fill<<<tsg_blocks((long long)(r1 - r0) * 16, 256), 256, 0, st>>>(
                    rows, r1 - r0, C.tile_ptr + r0, C.tile_columnidx, C.tile_nnz, C.tile_csr_Ptr, C.tile_csr_Col,
                    C.tile_csr_Value, d_rp + (long long)r0 * TSG_BS, d_ci, d_v);
                TSG_LAUNCH_CHECK();
                TSG_CUDA(cudaEventRecord(ctx->copy_ev, st));
                TSG_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->copy_ev, 0));
                const long long e0 = h_rowptr[(long long)r0 * TSG_BS], e1 = h_rowptr[r1 * TSG_BS < m ? r1 * TSG_BS : m];
                if (e1 > e0)
                {
                    TSG_CUDA(cudaMemcpyAsync(h_colidx + e0, d_ci + e0, (size_t)(e1 - e0) * sizeof(int),
                                             cudaMemcpyDeviceToHost, ctx->copy_stream));
                    TSG_CUDA(cudaMemcpyAsync(h_val + e0, d_v + e0, (size_t)(e1 - e0) * sizeof(double),
                                             cudaMemcpyDeviceToHost, ctx->copy_stream));
                }
                r0 = r1;
            }
            return TSG_OK;
        })();
    // the copies end before the buffers are released on the context's stream
    if (ctx->copy_stream)
        cudaStreamSynchronize(ctx->copy_stream);
    if (status == TSG_OK && ctx->timing)
        status = cudaEventRecord(ctx->ev[3], st) == cudaSuccess ? TSG_OK
                                                                 : tsg_set_error(TSG_ERR_CUDA, "cudaEventRecord");
    tsg_release(ctx, d_rp);
    tsg_release(ctx, d_ci);
    tsg_release(ctx, d_v);
    if (status == TSG_OK)
        status = spgemm_finish(ctx, R, info);
    else
    {
        tsg_release(ctx, R.d_wide);
        tsg_release(ctx, R.d_pairs);
        tsg_release(ctx, R.d_bins);
    }
    tsg_tiled_free(ctx, &C);
    if (status == TSG_OK)
        TSG_CUDA(cudaStreamSynchronize(st));
    return status;
}

// Number of C tiles of A*B (step 1's count pass only) added to the device
// word *total, without synchronising; A and B need their row-major tile
// structure.
int tsg_count_c_tiles_async(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B, unsigned long long *total)
{
    if (A->tilem == 0)
        return TSG_OK;
    tsg_tiled Cdummy;
    memset(&Cdummy, 0, sizeof(Cdummy));
    k_step1_total<<<tsg_blocks(A->tilem, S1_WARPS), S1_WARPS * 32, 0, ctx->stream>>>(make_view(A, B, &Cdummy), total);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}
