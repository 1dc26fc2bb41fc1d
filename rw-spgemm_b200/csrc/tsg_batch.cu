// Batched tiled SpGEMM: many independent products C_p = A_p * B_p of uneven
// size in ONE persistent, cooperatively launched kernel, captured once in a
// CUDA graph and replayed by tsg_batch_run.
//
// The kernel runs seven phases separated by a grid barrier; in each phase the
// work of all products is one flattened index space (product found by binary
// search over a prefix array), so small products do not leave the GPU idle:
//   1 step-1 counts (warp per A tile row)        2 per-product scan of them
//   3 item prefix over products (block 0)        4 step-1 emit
//   5 step 2 (half-warp per item)                6 per-product scan of tile nnz
//   7 step 3 (half-warp per item)
// An item is one C tile (tile schedule) or seg_tiles C tiles (row schedule);
// the per-item code is tsg_device.cuh's, identical to the one-product path.
//
// Memory: one arena per batch, sized at creation from per-product upper
// bounds computed on the device (C tiles <= matched tile pairs, C nonzeros <=
// scalar products), so a run needs no host round trip.  The grid barrier is
// bounded in time (%globaltimer): a wait longer than the batch's limit --
// BATCH_WAIT_FLOOR_NS plus BATCH_WAIT_NS_PER_PRODUCT per scalar product of
// the whole batch, or tsg_batch_set_wait_limit's -- sets TSG_ERR_TIMEOUT in
// the error word that tsg_batch_sync reports, and every block leaves.
#include <cooperative_groups.h>
#include <stdlib.h>

#include <vector>

#include "tsg_device.cuh"

int tsg_count_c_tiles_async(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B, unsigned long long *total);

struct BatchProd
{
    ProdView P;
    int *wide; // per A tile row: 1 when step 2 runs per tile (fused pass declined), 2 hypersparse
    long long capT, capN;
    int tilemA;
    int status; // 0 ok, 1 tile capacity, 2 value capacity
    int numC, nnzC;
};

struct tsg_batch
{
    tsg_context *ctx;
    int count;
    tsg_batch_params params;
    std::vector<BatchProd> host;    // descriptors (host copy)
    std::vector<long long> rowoff;  // prefix of tilemA over products
    BatchProd *d_prod;
    long long *d_rowoff;
    long long *d_itemoff;
    unsigned *d_bar; // [0] arrivals, [1] generation, [2] / [3] next tile block (SPA steps 3 / 2),
                     // [4..5] the barrier's wait limit in ns (64-bit)
    int *d_err;
    int *d_bins;
    void *arena;
    size_t arena_bytes;
    int grid, block;
    size_t smem;
    int grid3; // persistent grid of k_batch_spa3 (SPA schedule)
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    int graph_ok;
    std::vector<int> m, n, tilen; // per product C dimensions
    long long launches;
    unsigned long long wait_ns; // the grid barrier's wait limit
    unsigned bar_init[8];       // host image of d_bar at creation (zeros, the wait limit at [4])
    int dense;                  // SPA schedule: values per C tile from which a product takes the tile kernel
};

#define BATCH_THREADS 128
// a barrier wait gives up after this floor plus a share of the batch's work
// (a B200 does well over 10 scalar products per ns, so the bound is loose)
#define BATCH_WAIT_FLOOR_NS 2000000000ULL
#define BATCH_WAIT_NS_PER_PRODUCT 10ULL

__device__ __forceinline__ unsigned long long batch_clock_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// bounded grid barrier (all blocks co-resident: cooperative launch)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err)
{
    __syncthreads();
    if (threadIdx.x == 0)
    {
        volatile unsigned *vgen = bar + 1;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u) + 1u;
        if (arrived == gridDim.x)
        {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        }
        else
        {
            const unsigned long long limit = *(volatile unsigned long long *)(bar + 4);
            const unsigned long long t0 = batch_clock_ns();
            while (*vgen == gen)
            {
                if (*(volatile int *)err || batch_clock_ns() - t0 > limit)
                {
                    atomicCAS(err, 0, TSG_ERR_TIMEOUT);
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *)err == 0;
}

__device__ __forceinline__ int find_product(const long long *__restrict__ off, int count, long long x)
{
    int lo = 0, hi = count - 1; // largest p with off[p] <= x
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// The same for x at or after off[p] (a CTA's claims from a counter only grow):
// usually x is still in product p.
__device__ __forceinline__ int find_product_from(const long long *__restrict__ off, int count, long long x, int p)
{
    return off[p + 1] > x ? p : find_product(off, count, x);
}

// Block-wide exclusive scan of a[0..n) in place, a[n] = total (NT threads;
// s_tmp holds NT / 32 partial sums).
template <int NT>
__device__ long long block_scan_inplace(int *a, int n, long long *s_tmp)
{
    long long run = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n; base += NT)
    {
        const int i = base + threadIdx.x;
        const long long v = i < n ? a[i] : 0;
        long long incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const long long o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
            if (lane >= d)
                incl += o;
        }
        if (lane == 31)
            s_tmp[warp] = incl;
        __syncthreads();
        long long woff = 0;
        for (int w = 0; w < warp; w++)
            woff += s_tmp[w];
        long long tot = 0;
#pragma unroll
        for (int w = 0; w < NT / 32; w++)
            tot += s_tmp[w];
        if (i < n)
            a[i] = (int)(run + woff + incl - v);
        run += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        a[n] = (int)run;
    __syncthreads();
    return run;
}

// Block-wide sum of a[0..n) (NT threads).
template <int NT>
__device__ long long block_sum(const int *a, int n, long long *s_tmp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long v = 0;
    for (int i = threadIdx.x; i < n; i += NT)
        v += a[i];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
        v += __shfl_xor_sync(TSG_FULL_MASK, v, d);
    if (lane == 0)
        s_tmp[warp] = v;
    __syncthreads();
    long long tot = 0;
#pragma unroll
    for (int w = 0; w < NT / 32; w++)
        tot += s_tmp[w];
    __syncthreads();
    return tot;
}

// Block-wide exclusive scan of a[0..n) in place, offset by off (NT threads).
template <int NT>
__device__ void block_scan_offset(int *a, int n, long long off, long long *s_tmp)
{
    long long run = off;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n; base += NT)
    {
        const int i = base + threadIdx.x;
        const long long v = i < n ? a[i] : 0;
        long long incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const long long o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
            if (lane >= d)
                incl += o;
        }
        if (lane == 31)
            s_tmp[warp] = incl;
        __syncthreads();
        long long woff = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < NT / 32; w++)
        {
            woff += w < warp ? s_tmp[w] : 0;
            tot += s_tmp[w];
        }
        if (i < n)
            a[i] = (int)(run + woff + incl - v);
        run += tot;
        __syncthreads();
    }
}

// Exclusive scan of v[0..n) in place (long long) by one block; returns the total.
template <int NT>
__device__ long long block_scan_ll(long long *v, int n, long long *s_tmp)
{
    long long run = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n; base += NT)
    {
        const int i = base + threadIdx.x;
        const long long x = i < n ? v[i] : 0;
        long long incl = x;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const long long o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
            if (lane >= d)
                incl += o;
        }
        if (lane == 31)
            s_tmp[warp] = incl;
        __syncthreads();
        long long woff = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < NT / 32; w++)
        {
            woff += w < warp ? s_tmp[w] : 0;
            tot += s_tmp[w];
        }
        if (i < n)
            v[i] = run + woff + incl - x;
        run += tot;
        __syncthreads();
    }
    return run;
}

#define SCAN_CHUNK 4096 // C tiles per chunk of the tile-count scan

// GPU global timer (ns); block 0 stamps the end of each phase into
// stamp[1..6] and every block raises stamp[7] as it leaves.
__device__ __forceinline__ unsigned long long gtimer() { return batch_clock_ns(); }

#define BATCH_STAMP(k)                                                  \
    if (blockIdx.x == 0 && threadIdx.x == 0)                           \
        stamp[k] = gtimer();

template <int SCHED, int W, int CAP, int NT>
__global__ void __launch_bounds__(NT)
    k_batch(BatchProd *prods, int count, const long long *__restrict__ rowoff, long long *itemoff, unsigned *bar,
            int *err, int *bins)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ long long s_tmp[NT / 32 + 1];
    __shared__ int s_row;
    __shared__ int s_bins[4];
    const int lane32 = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 15, hw = threadIdx.x >> 4;
    const unsigned hmask = TSG_HW_MASK(threadIdx.x);
    const long long nwarps = (long long)gridDim.x * (NT / 32);
    const long long nhw = (long long)gridDim.x * (NT / 16);
    const long long total_rows = rowoff[count];
    unsigned long long *stamp = reinterpret_cast<unsigned long long *>(itemoff + 2 * ((long long)count + 1));
    BATCH_STAMP(0)

    // phase 1: step-1 counts
    {
        unsigned *bm = reinterpret_cast<unsigned *>(s_raw) + warp * S1_WORDS;
        for (long long w = (long long)blockIdx.x * (NT / 32) + warp; w < total_rows; w += nwarps)
        {
            const int p = find_product(rowoff, count, w);
            const ProdView &P = prods[p].P;
            const int i = (int)(w - rowoff[p]);
            const int cnt = step1_row<false>(P, i, bm, lane32, nullptr);
            if (lane32 == 0)
                P.C_ptr[i] = cnt;
        }
    }
    if (!grid_barrier(bar, err))
        return;
    BATCH_STAMP(1)
    // phase 2: per-product scan of C tile counts
    for (int p = blockIdx.x; p < count; p += gridDim.x)
    {
        BatchProd &bp = prods[p];
        const long long tot = block_scan_inplace<NT>(bp.P.C_ptr, bp.tilemA, s_tmp);
        if (threadIdx.x == 0)
        {
            if (tot > bp.capT)
            {
                bp.status = 1;
                bp.numC = 0;
            }
            else
            {
                bp.status = 0;
                bp.numC = (int)tot;
            }
            bp.P.numC = bp.numC;
        }
    }
    if (!grid_barrier(bar, err))
        return;
    BATCH_STAMP(2)
    // phase 3: item prefix over products (block 0)
    if (blockIdx.x == 0)
    {
        if (threadIdx.x == 0)
        {
            long long run = 0;
            for (int p = 0; p < count; p++)
            {
                itemoff[p] = run;
                const long long nc = prods[p].numC;
                run += SCHED == 1 ? (nc + W - 1) / W : nc;
            }
            itemoff[count] = run;
            // SPA: blocks of SPA_BLK C tiles per product, prefix after itemoff
            long long *blkoff = itemoff + count + 1;
            run = 0;
            for (int p = 0; p < count; p++)
            {
                blkoff[p] = run;
                run += ((long long)prods[p].numC + SPA_BLK - 1) / SPA_BLK;
            }
            blkoff[count] = run;
            // tile-count scan chunks per product, prefix after the stamps
            long long *chunkoff = itemoff + 2 * ((long long)count + 1) + 8;
            run = 0;
            for (int p = 0; p < count; p++)
            {
                chunkoff[p] = run;
                run += ((long long)prods[p].numC + SCAN_CHUNK - 1) / SCAN_CHUNK;
            }
            chunkoff[count] = run;
            bar[2] = 0;
            bar[3] = 0;
        }
        if (threadIdx.x < 4)
            bins[threadIdx.x] = 0;
    }
    if (!grid_barrier(bar, err))
        return;
    BATCH_STAMP(3)
    // phase 4: step-1 emit (fused with step 2 for narrow rows unless the
    // row schedule runs its own step 2)
    if (threadIdx.x < 4)
        s_bins[threadIdx.x] = 0;
    __syncthreads();
    {
        unsigned *bm = reinterpret_cast<unsigned *>(s_raw) + warp * S1_WORDS;
        S12Smem *s12 = reinterpret_cast<S12Smem *>(s_raw) + warp;
        for (long long w = (long long)blockIdx.x * (NT / 32) + warp; w < total_rows; w += nwarps)
        {
            const int p = find_product(rowoff, count, w);
            if (prods[p].status)
                continue;
            const int i = (int)(w - rowoff[p]);
            if (SCHED == 1)
                step1_row<true>(prods[p].P, i, bm, lane32, nullptr);
            else
            {
                const int done = step12_row(prods[p].P, i, *s12, lane32, s_bins);
                int kind = 0;
                if (!done)
                {
                    __syncwarp();
                    step1_row<true>(prods[p].P, i, reinterpret_cast<unsigned *>(s12), lane32, nullptr);
                    __syncwarp(); // the row's C columns, emitted by all lanes
                    kind = SCHED == 3 ? wide_kind(prods[p].P, i, lane32) : 1;
                }
                if (lane32 == 0)
                    prods[p].wide[i] = kind;
                __syncwarp();
            }
        }
    }
    if (!grid_barrier(bar, err))
        return;
    BATCH_STAMP(4)
    // phase 5: step 2 (all tiles for the row schedule, tiles of wide rows otherwise)
    if (SCHED == 3)
    {
        // wide rows through B's row view; CTAs take blocks of C tiles
        Spa2Smem &S2 = *reinterpret_cast<Spa2Smem *>(s_raw);
        const long long *blkoff = itemoff + count + 1;
        unsigned nxt = 0; // thread 0: the next block, claimed one block ahead
        if (threadIdx.x == 0)
            nxt = atomicAdd(&bar[3], 1u);
        int p = 0;
        for (;;)
        {
            __syncthreads();
            if (threadIdx.x == 0)
            {
                s_row = (int)nxt;
                nxt = atomicAdd(&bar[3], 1u);
            }
            __syncthreads();
            const long long blk = s_row;
            if (blk >= blkoff[count])
                break;
            p = find_product_from(blkoff, count, blk, p);
            if (prods[p].status)
                continue;
            const ProdView &P = prods[p].P;
            const long long tb = (blk - blkoff[p]) * SPA_BLK;
            if (threadIdx.x == 0)
                spa_skip_hyper(P, prods[p].wide, (int)tb, &bar[3], blkoff[p]);
            step2_spa_block(P, S2, (int)tb, (int)min((long long)P.numC, tb + SPA_BLK), prods[p].wide, s_bins);
        }
    }
    else
    {
        const long long total_items = itemoff[count];
        for (long long h = (long long)blockIdx.x * (NT / 16) + hw; h < total_items; h += nhw)
        {
            const int p = find_product(itemoff, count, h);
            const ProdView &P = prods[p].P;
            const long long item = h - itemoff[p];
            if (SCHED == 1)
                step2_rows_item<W>(P, item, hmask, lane, reinterpret_cast<S2RowsSmem<W> *>(s_raw)[hw], s_bins);
            else if (prods[p].wide[P.C_row[item]])
                step2_tile(P, (int)item, hmask, lane, s_bins);
        }
    }
    __syncthreads();
    if (threadIdx.x < 4 && s_bins[threadIdx.x])
        atomicAdd(&bins[threadIdx.x], s_bins[threadIdx.x]);
    if (!grid_barrier(bar, err))
        return;
    BATCH_STAMP(5)
    // phase 6: per-product exclusive scan of the tile counts, in chunks of
    // SCAN_CHUNK tiles spread over all blocks: chunk sums, a scan of each
    // product's chunk sums, then every chunk scanned with its offset
    {
        const long long *chunkoff = itemoff + 2 * ((long long)count + 1) + 8;
        long long *csum = const_cast<long long *>(chunkoff) + count + 1;
        const long long nch = chunkoff[count];
        for (long long c = blockIdx.x; c < nch; c += gridDim.x)
        {
            const int p = find_product(chunkoff, count, c);
            const BatchProd &bp = prods[p];
            const long long t0 = (c - chunkoff[p]) * SCAN_CHUNK;
            const int n = (int)min((long long)SCAN_CHUNK, (long long)bp.numC - t0);
            const long long tot = bp.status ? 0 : block_sum<NT>(bp.P.C_tnnz + t0, n, s_tmp);
            if (threadIdx.x == 0)
                csum[c] = tot;
        }
        if (!grid_barrier(bar, err))
            return;
        for (int p = blockIdx.x; p < count; p += gridDim.x)
        {
            BatchProd &bp = prods[p];
            const long long tot =
                block_scan_ll<NT>(csum + chunkoff[p], (int)(chunkoff[p + 1] - chunkoff[p]), s_tmp);
            if (threadIdx.x == 0 && !bp.status)
            {
                if (tot > bp.capN)
                {
                    bp.status = 2;
                    bp.nnzC = 0;
                }
                else
                    bp.nnzC = (int)tot;
                bp.P.C_tnnz[bp.numC] = (int)(tot > bp.capN ? 0 : tot);
            }
        }
        if (!grid_barrier(bar, err))
            return;
        for (long long c = blockIdx.x; c < nch; c += gridDim.x)
        {
            const int p = find_product(chunkoff, count, c);
            const BatchProd &bp = prods[p];
            if (bp.status)
                continue;
            const long long t0 = (c - chunkoff[p]) * SCAN_CHUNK;
            const int n = (int)min((long long)SCAN_CHUNK, (long long)bp.numC - t0);
            block_scan_offset<NT>(bp.P.C_tnnz + t0, n, csum[c], s_tmp);
        }
    }
    if (!grid_barrier(bar, err))
        return;
    BATCH_STAMP(6)
    // phase 7: step 3 (the SPA schedule runs it as two kernels after this one:
    // k_batch_spa3 and k_batch_dense3, each at its own occupancy)
    if (SCHED == 3)
        return;
    if (SCHED == 2)
    {
        int2 *pairs = reinterpret_cast<int2 *>(s_raw) + warp * S3E_PAIRS;
        const long long total_items = itemoff[count];
        for (long long w = (long long)blockIdx.x * (NT / 32) + warp; w < total_items; w += nwarps)
        {
            const int p = find_product(itemoff, count, w);
            if (prods[p].status)
                continue;
            step3_elems_tile(prods[p].P, (int)(w - itemoff[p]), pairs);
        }
    }
    else
    {
        double *tacc = reinterpret_cast<double *>(s_raw) + hw * (TSG_BS * S3T_STRIDE);
        if (!SCHED)
        {
            for (int q = lane; q < TSG_BS * S3T_STRIDE; q += 16)
                tacc[q] = 0.0;
            __syncwarp(hmask);
        }
        const long long total_items = itemoff[count];
        for (long long h = (long long)blockIdx.x * (NT / 16) + hw; h < total_items; h += nhw)
        {
            const int p = find_product(itemoff, count, h);
            if (prods[p].status)
                continue;
            const ProdView &P = prods[p].P;
            const long long item = h - itemoff[p];
            if (SCHED == 1)
                step3_rows_item<W, CAP>(P, item, hmask, lane, reinterpret_cast<S3RowsSmem<W, CAP> *>(s_raw)[hw]);
            else
                step3_tile(P, (int)item, hmask, lane, tacc);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)
        atomicMax(&stamp[7], gtimer());
}

// Step 3 of the SPA schedule over a batch, after k_batch: products with
// sparse C tiles, CTAs taking blocks of SPA_BLK C tiles (all products) from a
// device counter.  Raises stamp[7] on exit.  Does nothing when k_batch left
// with an error (its later phases did not run).
__global__ void __launch_bounds__(SPA_THREADS, 3)
    k_batch_spa3(BatchProd *prods, int count, const long long *__restrict__ itemoff, unsigned *bar, const int *err,
                 int dense)
{
    if (*(volatile const int *)err)
        return;
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ int s_blk;
    SpaSmem &S = *reinterpret_cast<SpaSmem *>(s_raw);
    const long long *blkoff = itemoff + count + 1;
    unsigned nxt = 0; // thread 0: the next block, claimed one block ahead
    if (threadIdx.x == 0)
        nxt = atomicAdd(&bar[2], 1u);
    int p = 0;
    for (;;)
    {
        __syncthreads();
        if (threadIdx.x == 0)
        {
            s_blk = (int)nxt;
            nxt = atomicAdd(&bar[2], 1u);
        }
        __syncthreads();
        const long long blk = s_blk;
        if (blk >= blkoff[count])
            break;
        p = find_product_from(blkoff, count, blk, p);
        if (prods[p].status || prods[p].nnzC >= (long long)dense * prods[p].numC)
            continue;
        const ProdView &P = prods[p].P;
        const long long tb = (blk - blkoff[p]) * SPA_BLK;
        if (threadIdx.x == 0)
            spa_skip_hyper(P, prods[p].wide, (int)tb, &bar[2], blkoff[p]);
        step3_spa_block<true>(P, S, (int)tb, (int)min((long long)P.numC, tb + SPA_BLK), prods[p].wide);
    }
    __syncthreads();
    if (threadIdx.x == 0)
        atomicMax(reinterpret_cast<unsigned long long *>(const_cast<long long *>(itemoff)) + 2 * ((long long)count + 1) +
                      7,
                  gtimer());
}

// ... and products with dense C tiles (>= `dense` values per tile on
// average): the tile kernel, a half-warp per C tile.
#define DENSE3_THREADS 256
__global__ void __launch_bounds__(DENSE3_THREADS)
    k_batch_dense3(BatchProd *prods, int count, const long long *__restrict__ itemoff, const int *err, int dense)
{
    if (*(volatile const int *)err)
        return;
    __shared__ double s_acc[DENSE3_THREADS / 16][TSG_BS * S3T_STRIDE];
    const int lane = threadIdx.x & 15, hw = threadIdx.x >> 4;
    const unsigned hmask = TSG_HW_MASK(threadIdx.x);
    double *tacc = s_acc[hw];
    for (int q = lane; q < TSG_BS * S3T_STRIDE; q += 16)
        tacc[q] = 0.0;
    __syncwarp(hmask);
    const long long total_items = itemoff[count];
    const long long nhw = (long long)gridDim.x * (DENSE3_THREADS / 16);
    for (long long h = (long long)blockIdx.x * (DENSE3_THREADS / 16) + hw; h < total_items; h += nhw)
    {
        const int p = find_product(itemoff, count, h);
        if (prods[p].status || prods[p].nnzC < (long long)dense * prods[p].numC)
            continue;
        step3_tile(prods[p].P, (int)(h - itemoff[p]), hmask, lane, tacc);
    }
    __syncthreads();
    if (threadIdx.x == 0)
        atomicMax(reinterpret_cast<unsigned long long *>(const_cast<long long *>(itemoff)) + 2 * ((long long)count + 1) +
                      7,
                  gtimer());
}

// ---------------------------------------------------------------------------
// upper bounds: matched tile pairs and scalar products per product
// ---------------------------------------------------------------------------
// half-warp per B tile row: element row lengths of B from the tile masks
__global__ void k_brow_len(int tilem, int m, const int *__restrict__ tile_ptr, const unsigned short *__restrict__ mask,
                           int *__restrict__ rowlen)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int tr = (int)(gid >> 4), lane = threadIdx.x & 15;
    if (tr >= tilem)
        return;
    int s = 0;
    for (int t = tile_ptr[tr]; t < tile_ptr[tr + 1]; t++)
        s += __popc((unsigned)mask[(long long)t * TSG_BS + lane]);
    if (tr * TSG_BS + lane < m)
        rowlen[tr * TSG_BS + lane] = s;
}

// half-warp per A tile: tile pairs and scalar products it generates
__global__ void k_bounds(int T, const int *__restrict__ A_col, const unsigned short *__restrict__ A_mask,
                         const int *__restrict__ B_ptr, const int *__restrict__ browlen, int mB,
                         unsigned long long *__restrict__ out)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int t = (int)(gid >> 4), lane = threadIdx.x & 15;
    unsigned long long prods = 0, pairs = 0;
    if (t < T)
    {
        const int k = A_col[t];
        unsigned ma = A_mask[(long long)t * TSG_BS + lane];
        while (ma)
        {
            const int bit = 31 - __clz(ma);
            const int row = k * TSG_BS + (15 - bit);
            if (row < mB)
                prods += (unsigned long long)browlen[row];
            ma ^= 1u << bit;
        }
        if (lane == 0)
            pairs = (unsigned long long)(B_ptr[k + 1] - B_ptr[k]);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
    {
        prods += __shfl_xor_sync(TSG_FULL_MASK, prods, d);
        pairs += __shfl_xor_sync(TSG_FULL_MASK, pairs, d);
    }
    if ((threadIdx.x & 31) == 0 && (prods || pairs))
    {
        atomicAdd(out, prods);
        atomicAdd(out + 1, pairs);
    }
}

extern "C" int tsg_product_bounds_many(tsg_context *ctx, int count, const tsg_tiled *A, const tsg_tiled *B,
                                       long long *products, long long *tile_pairs, long long *c_tiles)
{
    if (!ctx || count < 0 || (count && (!A || !B || !products || !tile_pairs)))
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    if (count == 0)
        return TSG_OK;
    int maxm = 0;
    for (int p = 0; p < count; p++)
        maxm = B[p].m > maxm ? B[p].m : maxm;
    int *rowlen;
    unsigned long long *d;
    TSG_TRY(tsg_alloc(ctx, &rowlen, (size_t)maxm + 1));
    TSG_TRY(tsg_alloc(ctx, &d, (size_t)count * 3));
    TSG_CUDA(cudaMemsetAsync(d, 0, (size_t)count * 3 * sizeof(unsigned long long), ctx->stream));
    int st = TSG_OK;
    for (int p = 0; p < count && st == TSG_OK; p++)
    {
        // k_brow_len writes every row of B below m: the buffer is reused in
        // stream order without clearing
        if (B[p].tilem > 0)
        {
            k_brow_len<<<tsg_blocks((long long)B[p].tilem * 16, 256), 256, 0, ctx->stream>>>(
                B[p].tilem, B[p].m, B[p].tile_ptr, B[p].mask, rowlen);
            TSG_LAUNCH_CHECK();
        }
        if (A[p].numtile > 0)
        {
            k_bounds<<<tsg_blocks((long long)A[p].numtile * 16, 256), 256, 0, ctx->stream>>>(
                A[p].numtile, A[p].tile_columnidx, A[p].mask, B[p].tile_ptr, rowlen, B[p].m, d + 3 * p);
            TSG_LAUNCH_CHECK();
        }
        if (c_tiles)
            st = tsg_count_c_tiles_async(ctx, &A[p], &B[p], d + 3 * p + 2);
    }
    if (st == TSG_OK)
    {
        std::vector<unsigned long long> h((size_t)count * 3);
        TSG_CUDA(cudaMemcpyAsync(h.data(), d, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 ctx->stream));
        TSG_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int p = 0; p < count; p++)
        {
            products[p] = (long long)h[3 * p];
            tile_pairs[p] = (long long)h[3 * p + 1];
            if (c_tiles)
                c_tiles[p] = (long long)h[3 * p + 2];
        }
    }
    tsg_release(ctx, rowlen);
    tsg_release(ctx, d);
    return st;
}

extern "C" int tsg_product_bounds(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B, long long *products,
                                  long long *tile_pairs)
{
    if (!ctx || !A || !B || !products || !tile_pairs)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    return tsg_product_bounds_many(ctx, 1, A, B, products, tile_pairs, nullptr);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef void (*batch_kernel_t)(BatchProd *, int, const long long *, long long *, unsigned *, int *, int *);

// Kernel, dynamic shared memory and block size of a batch schedule.
static batch_kernel_t pick_kernel(const tsg_batch_params &p, size_t *smem, int *threads)
{
    *threads = BATCH_THREADS;
    const size_t s1a = (size_t)(BATCH_THREADS / 32) * S1_WORDS * 4;
    const size_t s12 = (size_t)(BATCH_THREADS / 32) * sizeof(S12Smem);
    const size_t s1 = s1a > s12 ? s1a : s12;
    if (p.schedule == TSG_SCHED_SPA)
    {
        *threads = SPA_THREADS;
        const size_t t1a = (size_t)(SPA_THREADS / 32) * S1_WORDS * 4;
        const size_t t12 = (size_t)(SPA_THREADS / 32) * sizeof(S12Smem);
        const size_t t1 = t1a > t12 ? t1a : t12;
        *smem = t1 > sizeof(Spa2Smem) ? t1 : sizeof(Spa2Smem);
        return k_batch<3, 8, 256, SPA_THREADS>;
    }
    if (p.schedule == TSG_SCHED_ELEMS)
    {
        const size_t s3 = (size_t)(BATCH_THREADS / 32) * S3E_PAIRS * sizeof(int2);
        *smem = s1 > s3 ? s1 : s3;
        return k_batch<2, 8, 256, BATCH_THREADS>;
    }
    if (p.schedule == TSG_SCHED_TILES)
    {
        const size_t s3 = (size_t)(BATCH_THREADS / 16) * TSG_BS * S3T_STRIDE * 8;
        *smem = s1 > s3 ? s1 : s3;
        return k_batch<0, 8, 256, BATCH_THREADS>;
    }
#define TSG_PICK(w, c)                                                                          \
    if (p.seg_tiles == w && p.acc_cap == c)                                                     \
    {                                                                                           \
        size_t s2 = (size_t)(BATCH_THREADS / 16) * sizeof(S2RowsSmem<w>);                       \
        size_t s3 = (size_t)(BATCH_THREADS / 16) * sizeof(S3RowsSmem<w, c>);                    \
        size_t mx = s1 > s2 ? s1 : s2;                                                          \
        *smem = mx > s3 ? mx : s3;                                                              \
        return k_batch<1, w, c, BATCH_THREADS>;                                                 \
    }
    TSG_ROW_CONFIGS(TSG_PICK)
#undef TSG_PICK
    return nullptr;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static int record_run(tsg_batch *b, cudaStream_t st)
{
    size_t smem;
    int threads;
    batch_kernel_t kern = pick_kernel(b->params, &smem, &threads);
    TSG_CUDA(cudaMemsetAsync(b->d_err, 0, sizeof(int), st));
    TSG_CUDA(cudaMemsetAsync(b->d_bar, 0, sizeof(unsigned), st));
    // phase stamps (after the two item prefixes): [7] is a running maximum
    TSG_CUDA(cudaMemsetAsync(b->d_itemoff + 2 * ((size_t)b->count + 1), 0, 8 * sizeof(long long), st));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)b->grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = b->smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TSG_CUDA(cudaLaunchKernelEx(&cfg, kern, b->d_prod, b->count, (const long long *)b->d_rowoff, b->d_itemoff,
                                b->d_bar, b->d_err, b->d_bins));
    if (b->params.schedule == TSG_SCHED_SPA)
    {
        k_batch_spa3<<<b->grid3, SPA_THREADS, sizeof(SpaSmem), st>>>(b->d_prod, b->count, b->d_itemoff, b->d_bar,
                                                                     b->d_err, b->dense);
        TSG_CUDA(cudaGetLastError());
        k_batch_dense3<<<b->ctx->num_sms * 8, DENSE3_THREADS, 0, st>>>(b->d_prod, b->count, b->d_itemoff, b->d_err,
                                                                        b->dense);
        TSG_CUDA(cudaGetLastError());
    }
    return TSG_OK;
}

// products / c_tiles: the bounds of every product when the caller has them
// (tsg_product_bounds_many), else null and computed here
static int batch_create(tsg_context *ctx, int count, const tsg_tiled *A, const tsg_tiled *B,
                        const tsg_batch_params *params, const long long *products, const long long *c_tiles,
                        tsg_batch **out)
{
    if (!ctx || !out || count <= 0 || !A || !B)
        return tsg_set_error(TSG_ERR_INVALID, "bad batch arguments");
    *out = nullptr;
    tsg_batch_params prm;
    if (params)
        prm = *params;
    else
    {
        prm.schedule = TSG_SCHED_ROWS;
        prm.seg_tiles = 16;
        prm.acc_cap = 1024;
        prm.use_graph = 1;
        prm.dense_threshold = 0;
    }
    if (prm.dense_threshold < 0 || prm.dense_threshold > 257)
        return tsg_set_error(TSG_ERR_INVALID, "dense threshold %d outside [0, 257]", prm.dense_threshold);
    size_t smem;
    int threads;
    batch_kernel_t kern = pick_kernel(prm, &smem, &threads);
    if (!kern)
        return tsg_set_error(TSG_ERR_INVALID, "unsupported batch schedule (%d, %d, %d)", prm.schedule, prm.seg_tiles,
                             prm.acc_cap);
    for (int p = 0; p < count; p++)
    {
        if (A[p].n != B[p].m || !B[p].csc_tile_ptr)
            return tsg_set_error(TSG_ERR_INVALID, "product %d: inner dimensions differ or B lacks its column view", p);
        if (prm.schedule == TSG_SCHED_ELEMS && !B[p].mask_t)
            return tsg_set_error(TSG_ERR_INVALID, "product %d: element schedule needs B's column masks", p);
        if (prm.schedule == TSG_SCHED_SPA && !B[p].row_ptr)
            return tsg_set_error(TSG_ERR_INVALID, "product %d: SPA schedule needs B's row view", p);
    }
    tsg_batch *b = new tsg_batch();
    b->ctx = ctx;
    b->count = count;
    b->params = prm;
    b->dense = prm.dense_threshold ? prm.dense_threshold : SPA_DENSE;
    b->host.resize(count);
    b->rowoff.resize(count + 1);
    b->m.resize(count);
    b->n.resize(count);
    b->tilen.resize(count);
    b->launches = 0;
    // bounds and arena layout
    size_t bytes = 0;
    std::vector<size_t> off(count);
    long long run = 0, chunk_cap = 0, total_prods = 0;
    // scalar products and the exact C tile count (step 1's count pass) of
    // every product, one synchronisation for the whole batch
    std::vector<long long> v_prods(count), v_pairs(count), v_tiles(count);
    if (products && c_tiles)
        for (int p = 0; p < count; p++)
        {
            if (products[p] < 0 || c_tiles[p] < 0)
            {
                delete b;
                return tsg_set_error(TSG_ERR_INVALID, "product %d: negative bound", p);
            }
            v_prods[p] = products[p];
            v_tiles[p] = c_tiles[p];
        }
    else
    {
        int st = tsg_product_bounds_many(ctx, count, A, B, v_prods.data(), v_pairs.data(), v_tiles.data());
        if (st != TSG_OK)
        {
            delete b;
            return st;
        }
    }
    for (int p = 0; p < count; p++)
    {
        const long long prods = v_prods[p], capT = v_tiles[p];
        total_prods += prods;
        long long capN = prods < 256 * capT ? prods : 256 * capT;
        if (capN > 2147483647LL || capT > 2147483647LL / 16)
        {
            delete b;
            return tsg_set_error(TSG_ERR_OVERFLOW, "product %d exceeds 32-bit offsets", p);
        }
        BatchProd &h = b->host[p];
        memset(&h, 0, sizeof(h));
        h.capT = capT;
        h.capN = capN;
        chunk_cap += (capT + SCAN_CHUNK - 1) / SCAN_CHUNK;
        h.tilemA = A[p].tilem;
        b->rowoff[p] = run;
        run += A[p].tilem;
        b->m[p] = A[p].m;
        b->n[p] = B[p].n;
        b->tilen[p] = B[p].tilen;
        off[p] = bytes;
        bytes += align256(((size_t)A[p].tilem + 1) * 4) + align256((size_t)A[p].tilem * 4) + 2 * align256((size_t)capT * 4) +
                 align256(((size_t)capT + 1) * 4) +
                 align256((size_t)capT * 32) + align256((size_t)capT * 16) + align256((size_t)capN) +
                 align256((size_t)capN * 8);
    }
    b->rowoff[count] = run;
    b->arena_bytes = bytes;
    int st = TSG_OK;
    if ((st = tsg_alloc(ctx, (char **)&b->arena, bytes ? bytes : 256)) != TSG_OK)
    {
        delete b;
        return st;
    }
    for (int p = 0; p < count; p++)
    {
        BatchProd &h = b->host[p];
        char *q = (char *)b->arena + off[p];
        auto take = [&](size_t nbytes) {
            char *r = q;
            q += align256(nbytes);
            return r;
        };
        ProdView &P = h.P;
        P.A_ptr = A[p].tile_ptr;
        P.A_col = A[p].tile_columnidx;
        P.A_tnnz = A[p].tile_nnz;
        P.A_Ptr = A[p].tile_csr_Ptr;
        P.A_Colb = A[p].tile_csr_Col;
        P.A_Val = A[p].tile_csr_Value;
        P.A_mask = A[p].mask;
        P.tilemA = A[p].tilem;
        P.B_ptr = B[p].tile_ptr;
        P.B_col = B[p].tile_columnidx;
        P.B_cptr = B[p].csc_tile_ptr;
        P.B_crow = B[p].csc_tile_rowidx;
        P.B_cpos = B[p].csc_tile_pos;
        P.B_tnnz = B[p].tile_nnz;
        P.B_Ptr = B[p].tile_csr_Ptr;
        P.B_Colb = B[p].tile_csr_Col;
        P.B_Val = B[p].tile_csr_Value;
        P.B_mask = B[p].mask;
        P.B_maskT = B[p].mask_t;
        P.B_rptr = B[p].row_ptr;
        P.B_rcol = B[p].row_col;
        P.B_rval = B[p].row_val;
        P.browB = B[p].m > 0 ? (int)(B[p].nnz / B[p].m) : 0;
        P.tilenB = B[p].tilen;
        P.C_ptr = (int *)take(((size_t)A[p].tilem + 1) * 4);
        h.wide = (int *)take((size_t)A[p].tilem * 4);
        P.C_col = (int *)take((size_t)h.capT * 4);
        P.C_row = (int *)take((size_t)h.capT * 4);
        P.C_tnnz = (int *)take(((size_t)h.capT + 1) * 4);
        P.C_mask = (unsigned short *)take((size_t)h.capT * 32);
        P.C_Ptr = (unsigned char *)take((size_t)h.capT * 16);
        P.C_Colb = (unsigned char *)take((size_t)h.capN);
        P.C_Val = (double *)take((size_t)h.capN * 8);
        P.numC = 0;
        P.padded = 0;
        P.status = nullptr; // the batch's error word, set once it is allocated
    }
    if ((st = tsg_alloc(ctx, &b->d_prod, (size_t)count)) != TSG_OK || (st = tsg_alloc(ctx, &b->d_rowoff, (size_t)count + 1)) ||
        (st = tsg_alloc(ctx, &b->d_itemoff, 3 * ((size_t)count + 1) + 8 + (size_t)chunk_cap)) || (st = tsg_alloc(ctx, &b->d_bar, 8)) ||
        (st = tsg_alloc(ctx, &b->d_err, 1)) || (st = tsg_alloc(ctx, &b->d_bins, 4)))
    {
        tsg_batch_destroy(b);
        return st;
    }
    cudaStream_t s = ctx->stream;
    // an in-kernel error (a numeric accumulator overflow) goes to the batch's error word
    for (BatchProd &h : b->host)
        h.P.status = b->d_err;
    // copies only (no memset kernels): creating a batch never waits for SMs
    // held by another stream's persistent kernel
    b->wait_ns = BATCH_WAIT_FLOOR_NS + BATCH_WAIT_NS_PER_PRODUCT * (unsigned long long)total_prods;
    memset(b->bar_init, 0, sizeof(b->bar_init));
    memcpy(&b->bar_init[4], &b->wait_ns, sizeof(unsigned long long));
    cudaMemcpyAsync(b->d_prod, b->host.data(), sizeof(BatchProd) * count, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b->d_rowoff, b->rowoff.data(), sizeof(long long) * (count + 1), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b->d_bar, b->bar_init, sizeof(b->bar_init), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b->d_err, &b->bar_init[0], sizeof(int), cudaMemcpyHostToDevice, s);
    // co-resident grid
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    {
        tsg_batch_destroy(b);
        return tsg_set_error(TSG_ERR_CUDA, "cannot reserve %zu bytes of shared memory", smem);
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (per_sm < 1)
    {
        tsg_batch_destroy(b);
        return tsg_set_error(TSG_ERR_CUDA, "batch kernel cannot be resident");
    }
    b->grid = per_sm * ctx->num_sms;
    b->grid3 = 0;
    if (prm.schedule == TSG_SCHED_SPA)
    {
        int per3 = 0;
        if (cudaFuncSetAttribute(k_batch_spa3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SpaSmem)) !=
                cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per3, k_batch_spa3, SPA_THREADS, sizeof(SpaSmem)) !=
                cudaSuccess ||
            per3 < 1)
        {
            tsg_batch_destroy(b);
            return tsg_set_error(TSG_ERR_CUDA, "batch numeric kernel cannot be resident");
        }
        b->grid3 = per3 * ctx->num_sms;
    }
    b->block = threads;
    b->smem = smem;
    b->graph_ok = 0;
    if (prm.use_graph)
    {
        cudaStream_t cs;
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess)
        {
            cudaStreamSynchronize(s);
            if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess)
            {
                int rs = record_run(b, cs);
                cudaGraph_t g = nullptr;
                cudaError_t e = cudaStreamEndCapture(cs, &g);
                if (rs == TSG_OK && e == cudaSuccess && g &&
                    cudaGraphInstantiate(&b->exec, g, 0) == cudaSuccess)
                {
                    b->graph = g;
                    b->graph_ok = 1;
                }
                else if (g)
                    cudaGraphDestroy(g);
            }
            cudaGetLastError(); // a failed capture falls back to direct launches
            cudaStreamDestroy(cs);
        }
    }
    TSG_CUDA(cudaStreamSynchronize(s));
    *out = b;
    return TSG_OK;
}

extern "C" int tsg_batch_create(tsg_context *ctx, int count, const tsg_tiled *A, const tsg_tiled *B,
                                const tsg_batch_params *params, tsg_batch **out)
{
    return batch_create(ctx, count, A, B, params, nullptr, nullptr, out);
}

extern "C" int tsg_batch_create_bounded(tsg_context *ctx, int count, const tsg_tiled *A, const tsg_tiled *B,
                                        const tsg_batch_params *params, const long long *products,
                                        const long long *c_tiles, tsg_batch **out)
{
    if (!products || !c_tiles)
        return tsg_set_error(TSG_ERR_INVALID, "null bounds");
    return batch_create(ctx, count, A, B, params, products, c_tiles, out);
}

extern "C" int tsg_batch_run(tsg_batch *b)
{
    if (!b)
        return tsg_set_error(TSG_ERR_INVALID, "null batch");
    tsg_context *ctx = b->ctx;
    if (b->graph_ok)
        TSG_CUDA(cudaGraphLaunch(b->exec, ctx->stream));
    else
        TSG_TRY(record_run(b, ctx->stream));
    ctx->launches++;
    b->launches++;
    return TSG_OK;
}

extern "C" int tsg_batch_sync(tsg_batch *b, long long *total_tiles, long long *total_nnz)
{
    if (!b)
        return tsg_set_error(TSG_ERR_INVALID, "null batch");
    tsg_context *ctx = b->ctx;
    int err = 0;
    TSG_CUDA(cudaMemcpyAsync(b->host.data(), b->d_prod, sizeof(BatchProd) * b->count, cudaMemcpyDeviceToHost,
                             ctx->stream));
    TSG_CUDA(cudaMemcpyAsync(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (err == TSG_ERR_OVERFLOW)
        return tsg_set_error(TSG_ERR_OVERFLOW, "a numeric accumulator of the batch overflowed");
    if (err)
        return tsg_set_error(TSG_ERR_TIMEOUT, "batch grid barrier gave up waiting (bound %.3f s)", b->wait_ns * 1e-9);
    long long tt = 0, tn = 0;
    for (int p = 0; p < b->count; p++)
    {
        if (b->host[p].status)
            return tsg_set_error(TSG_ERR_OVERFLOW, "product %d exceeded its bound (%d)", p, b->host[p].status);
        tt += b->host[p].numC;
        tn += b->host[p].nnzC;
    }
    if (total_tiles)
        *total_tiles = tt;
    if (total_nnz)
        *total_nnz = tn;
    return TSG_OK;
}

extern "C" int tsg_batch_set_wait_limit(tsg_batch *b, double seconds)
{
    if (!b || !(seconds >= 0.0) || seconds > 1e6)
        return tsg_set_error(TSG_ERR_INVALID, "bad batch wait limit");
    tsg_context *ctx = b->ctx;
    b->wait_ns = (unsigned long long)(seconds * 1e9);
    TSG_CUDA(cudaMemcpyAsync(b->d_bar + 4, &b->wait_ns, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                             ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    return TSG_OK;
}

extern "C" int tsg_batch_product(tsg_batch *b, int p, tsg_tiled *C)
{
    if (!b || !C || p < 0 || p >= b->count)
        return tsg_set_error(TSG_ERR_INVALID, "bad batch product index");
    const BatchProd &h = b->host[p];
    memset(C, 0, sizeof(*C));
    C->m = b->m[p];
    C->n = b->n[p];
    C->tilem = h.tilemA;
    C->tilen = b->tilen[p];
    C->numtile = h.numC;
    C->nnz = h.nnzC;
    C->tile_ptr = h.P.C_ptr;
    C->tile_columnidx = h.P.C_col;
    C->tile_rowidx = h.P.C_row;
    C->tile_nnz = h.P.C_tnnz;
    C->mask = h.P.C_mask;
    C->tile_csr_Ptr = h.P.C_Ptr;
    C->tile_csr_Col = h.P.C_Colb;
    C->tile_csr_Value = h.P.C_Val;
    C->_alloc = (void *)b; // borrowed view into the batch arena
    return TSG_OK;
}

extern "C" int tsg_batch_phase_ms(tsg_batch *b, double *ms)
{
    if (!b || !ms)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    unsigned long long t[8];
    tsg_context *ctx = b->ctx;
    TSG_CUDA(cudaMemcpyAsync(t, b->d_itemoff + 2 * ((size_t)b->count + 1), sizeof(t), cudaMemcpyDeviceToHost,
                             ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 7; k++)
        ms[k] = t[k + 1] >= t[k] ? (double)(t[k + 1] - t[k]) * 1e-6 : 0.0;
    return TSG_OK;
}

extern "C" int tsg_batch_info(tsg_batch *b, int *graph, int *grid, size_t *arena_bytes, long long *launches)
{
    if (!b)
        return tsg_set_error(TSG_ERR_INVALID, "null batch");
    if (graph)
        *graph = b->graph_ok;
    if (grid)
        *grid = b->grid;
    if (arena_bytes)
        *arena_bytes = b->arena_bytes;
    if (launches)
        *launches = b->launches;
    return TSG_OK;
}

extern "C" int tsg_batch_destroy(tsg_batch *b)
{
    if (!b)
        return TSG_OK;
    tsg_context *ctx = b->ctx;
    cudaStreamSynchronize(ctx->stream);
    if (b->graph_ok)
    {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
    }
    tsg_release(ctx, b->d_prod);
    tsg_release(ctx, b->d_rowoff);
    tsg_release(ctx, b->d_itemoff);
    tsg_release(ctx, b->d_bar);
    tsg_release(ctx, b->d_err);
    tsg_release(ctx, b->d_bins);
    char *a = (char *)b->arena;
    tsg_release(ctx, a);
    cudaStreamSynchronize(ctx->stream);
    delete b;
    return TSG_OK;
}
