// Tiled SpGEMM C = A*B on 16x16 tiles, FP64, for sm_100a.
//
// Restates the three steps of the reference's tilespgemm()
// (src/tilespgemm-cuda.h:2610-3221):
//   step 1  tile structure of C        (reference :257-369, :2766-2848)
//   step 2  per-tile bitmask symbolic   (reference :371-755, :2866-2989)
//   step 3  numeric                     (reference :1505-2608, :3006-3118)
// with the same outputs (tile_ptr, sorted tile columns, 16-bit row masks,
// uint8 row offsets, tile nnz scan, plain column bytes, FP64 values).
//
// Design (B200):
//  * step 1: one warp per A tile row ORs the tile-column lists of the B tile
//    rows it touches into a shared-memory bitmap restricted to the row's
//    column window; popcount gives the count, an ordered bit walk emits the
//    sorted C tile columns.
//  * step 2/3: one half-warp per C tile.  The A tile row and the B tile
//    column are intersected 16 elements at a time with lanes holding the
//    chunks in registers (shuffle binary search + ballot), so matches come
//    out in ascending k with no scratch memory.  Step 2 multiplies 16x16
//    boolean tiles: lane r ORs the B mask rows selected by A's row-r mask
//    (the whole B mask is one 32-byte broadcast load).  Step 3 gives lane r
//    ownership of C row r: it accumulates a*b for its A row entries against
//    the selected B rows into a padded shared-memory row, in k-ascending,
//    A-entry order, with separately rounded multiply and add -- the order and
//    rounding of the reference's CPU oracle (src/spgemm-cpu.h:330), so
//    results are deterministic and bit-identical run to run, with no FP64
//    atomics.  The compressed tile is then written with coalesced stores,
//    columns recovered from the mask with __fns.
#include <limits.h>

#include "tsg_internal.h"

#define FULL_MASK 0xffffffffu
#define HW_MASK(tid) (0xFFFFu << ((tid) & 16))

// ---------------------------------------------------------------------------
// Step 1
// ---------------------------------------------------------------------------
#define S1_WARPS 8
#define S1_WORDS 1024

template <bool EMIT>
__global__ void __launch_bounds__(S1_WARPS * 32)
    k_step1(int tilemA, const int *__restrict__ A_ptr, const int *__restrict__ A_col,
            const int *__restrict__ B_ptr, const int *__restrict__ B_col, int *__restrict__ C_cnt,
            const int *__restrict__ C_ptr, int *__restrict__ C_col, int *__restrict__ C_row,
            unsigned long long *__restrict__ pairs)
{
    __shared__ unsigned int s_bm[S1_WARPS][S1_WORDS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * S1_WARPS + warp;
    if (i >= tilemA)
        return;
    unsigned int *bm = s_bm[warp];
    const int a0 = A_ptr[i], a1 = A_ptr[i + 1];
    int lo = INT_MAX, hi = -1;
    unsigned long long np = 0;
    for (int pa = a0 + lane; pa < a1; pa += 32)
    {
        const int k = A_col[pa];
        const int b0 = B_ptr[k], b1 = B_ptr[k + 1];
        if (b1 > b0)
        {
            lo = min(lo, B_col[b0]);
            hi = max(hi, B_col[b1 - 1]);
            np += (unsigned long long)(b1 - b0);
        }
    }
    lo = __reduce_min_sync(FULL_MASK, lo);
    hi = __reduce_max_sync(FULL_MASK, hi);
    if (!EMIT && pairs)
    {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1)
            np += __shfl_xor_sync(FULL_MASK, np, d);
        if (lane == 0 && np)
            atomicAdd(pairs, np);
    }
    int out = 0;
    const int cbase = EMIT ? C_ptr[i] : 0;
    if (hi >= 0)
    {
        for (int c0 = lo & ~31; c0 <= hi; c0 += S1_WORDS * 32)
        {
            const int c1 = min(hi + 1, c0 + S1_WORDS * 32);
            const int nw = (c1 - c0 + 31) >> 5;
            for (int w = lane; w < nw; w += 32)
                bm[w] = 0;
            __syncwarp();
            for (int pa = a0; pa < a1; pa++)
            {
                const int k = A_col[pa];
                const int b0 = B_ptr[k], b1 = B_ptr[k + 1];
                for (int pb = b0 + lane; pb < b1; pb += 32)
                {
                    const int j = B_col[pb];
                    if (j >= c0 && j < c1)
                        atomicOr(&bm[(j - c0) >> 5], 1u << ((j - c0) & 31));
                }
            }
            __syncwarp();
            for (int wb = 0; wb < nw; wb += 32)
            {
                const int w = wb + lane;
                unsigned bits = w < nw ? bm[w] : 0u;
                const int cnt = __popc(bits);
                if (EMIT)
                {
                    int incl = cnt;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1)
                    {
                        int o = __shfl_up_sync(FULL_MASK, incl, d);
                        if (lane >= d)
                            incl += o;
                    }
                    int pos = cbase + out + incl - cnt;
                    while (bits)
                    {
                        const int b = __ffs(bits) - 1;
                        bits &= bits - 1;
                        C_col[pos] = c0 + (w << 5) + b;
                        C_row[pos] = i;
                        pos++;
                    }
                    out += __shfl_sync(FULL_MASK, incl, 31);
                }
                else
                {
                    out += __reduce_add_sync(FULL_MASK, cnt);
                }
            }
            __syncwarp();
        }
    }
    if (!EMIT && lane == 0)
        C_cnt[i] = out;
}

// ---------------------------------------------------------------------------
// Tile-list intersection for one C tile (half-warp).  Calls f(x, posA, posB)
// for every matched k in ascending order; uniform across the half-warp.
// ---------------------------------------------------------------------------
template <typename F>
__device__ __forceinline__ void intersect_tiles(unsigned hmask, int lane, const int *__restrict__ a_list,
                                                int abase, int la, const int *__restrict__ b_list,
                                                const int *__restrict__ b_pos, int bbase, int lb, F f)
{
    int ia = 0, ib = 0;
    while (ia < la && ib < lb)
    {
        const int va = ia + lane < la ? a_list[abase + ia + lane] : INT_MAX;
        const int vb = ib + lane < lb ? b_list[bbase + ib + lane] : INT_MAX;
        int pos = 0;
#pragma unroll
        for (int s = 8; s >= 1; s >>= 1)
        {
            const int v = __shfl_sync(hmask, vb, pos + s - 1, 16);
            if (v < va)
                pos += s;
        }
        const int cand = __shfl_sync(hmask, vb, pos, 16);
        const bool found = (cand == va) && (va != INT_MAX);
        unsigned bal = __ballot_sync(hmask, found);
        bal = (bal >> (threadIdx.x & 16)) & 0xFFFFu;
        while (bal)
        {
            const int x = __ffs(bal) - 1;
            bal &= bal - 1;
            const int y = __shfl_sync(hmask, pos, x, 16);
            const int q = bbase + ib + y;
            const int posB = b_pos ? b_pos[q] : q;
            f(abase + ia + x, posB);
        }
        const int amax = __shfl_sync(hmask, va, 15, 16);
        const int bmax = __shfl_sync(hmask, vb, 15, 16);
        if (amax <= bmax)
            ia += 16;
        if (bmax <= amax)
            ib += 16;
    }
}

// Row r of the boolean product: OR of B's mask rows c for every column c set
// in A's row mask (bit 15-c).  q0/q1 hold B's 16 row masks (rows 2w, 2w+1 in
// the low / high half of word w).
__device__ __forceinline__ unsigned bool_row(unsigned ma, uint4 q0, uint4 q1)
{
    unsigned r = 0;
    const unsigned w[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
    for (int c = 0; c < 16; c++)
    {
        const unsigned row = (c & 1) ? (w[c >> 1] >> 16) : (w[c >> 1] & 0xFFFFu);
        r |= ((ma >> (15 - c)) & 1u) ? row : 0u;
    }
    return r;
}

// ---------------------------------------------------------------------------
// Step 2: masks, row offsets and nnz of every C tile (half-warp per tile).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_step2(int numC, const int *__restrict__ C_row, const int *__restrict__ C_col,
            const int *__restrict__ A_ptr, const int *__restrict__ A_col,
            const unsigned short *__restrict__ A_mask, const int *__restrict__ B_cptr,
            const int *__restrict__ B_crow, const int *__restrict__ B_cpos,
            const unsigned short *__restrict__ B_mask, unsigned short *__restrict__ C_mask,
            unsigned char *__restrict__ C_Ptr, int *__restrict__ C_cnt, int *__restrict__ bins)
{
    __shared__ int s_bins[4];
    if (threadIdx.x < 4)
        s_bins[threadIdx.x] = 0;
    __syncthreads();
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int t = (int)(gid >> 4);
    const int lane = threadIdx.x & 15;
    const unsigned hmask = HW_MASK(threadIdx.x);
    if (t < numC)
    {
        const int i = C_row[t], j = C_col[t];
        const int abase = A_ptr[i], la = A_ptr[i + 1] - abase;
        const int bbase = B_cptr[j], lb = B_cptr[j + 1] - bbase;
        unsigned acc = 0;
        intersect_tiles(hmask, lane, A_col, abase, la, B_crow, B_cpos, bbase, lb, [&](int posA, int posB) {
            const unsigned ma = A_mask[(long long)posA * TSG_BS + lane];
            const uint4 *mb = reinterpret_cast<const uint4 *>(B_mask + (long long)posB * TSG_BS);
            const uint4 q0 = __ldg(mb), q1 = __ldg(mb + 1);
            acc |= bool_row(ma, q0, q1);
        });
        const int cnt = __popc(acc);
        int incl = cnt;
#pragma unroll
        for (int d = 1; d < 16; d <<= 1)
        {
            const int o = __shfl_up_sync(hmask, incl, d, 16);
            if (lane >= d)
                incl += o;
        }
        const int total = __shfl_sync(hmask, incl, 15, 16);
        C_mask[(long long)t * TSG_BS + lane] = (unsigned short)acc;
        C_Ptr[(long long)t * TSG_BS + lane] = (unsigned char)(incl - cnt);
        if (lane == 0)
        {
            C_cnt[t] = total;
            if (total > 0)
            {
                const int b = total <= 32 ? 0 : total <= 224 ? 1 : total < 256 ? 2 : 3;
                atomicAdd(&s_bins[b], 1);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < 4 && s_bins[threadIdx.x])
        atomicAdd(&bins[threadIdx.x], s_bins[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// Step 3: numeric (half-warp per C tile, lane r owns C row r).
// ---------------------------------------------------------------------------
#define S3_THREADS 256
#define S3_HW (S3_THREADS / 16)
#define S3_STRIDE 17

__global__ void __launch_bounds__(S3_THREADS)
    k_step3(int numC, const int *__restrict__ C_row, const int *__restrict__ C_col,
            const int *__restrict__ A_ptr, const int *__restrict__ A_col, const int *__restrict__ A_tnnz,
            const unsigned char *__restrict__ A_Ptr, const unsigned char *__restrict__ A_Colb,
            const double *__restrict__ A_Val, const int *__restrict__ B_cptr, const int *__restrict__ B_crow,
            const int *__restrict__ B_cpos, const int *__restrict__ B_tnnz,
            const unsigned char *__restrict__ B_Ptr, const unsigned char *__restrict__ B_Colb,
            const double *__restrict__ B_Val, const int *__restrict__ C_tnnz,
            const unsigned short *__restrict__ C_mask, const unsigned char *__restrict__ C_Ptr,
            unsigned char *__restrict__ C_Colb, double *__restrict__ C_Val)
{
    __shared__ double s_acc[S3_HW][TSG_BS * S3_STRIDE];
    const int hw = threadIdx.x >> 4;
    double *acc = s_acc[hw];
    const int lane = threadIdx.x & 15;
    const unsigned hmask = HW_MASK(threadIdx.x);
    for (int q = lane; q < TSG_BS * S3_STRIDE; q += 16)
        acc[q] = 0.0;
    __syncwarp(hmask);
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int t = (int)(gid >> 4);
    if (t >= numC)
        return;
    const int cb = C_tnnz[t], cn = C_tnnz[t + 1] - cb;
    if (cn == 0)
        return;
    const int i = C_row[t], j = C_col[t];
    const int abase = A_ptr[i], la = A_ptr[i + 1] - abase;
    const int bbase = B_cptr[j], lb = B_cptr[j + 1] - bbase;
    double *myrow = acc + lane * S3_STRIDE;
    intersect_tiles(hmask, lane, A_col, abase, la, B_crow, B_cpos, bbase, lb, [&](int posA, int posB) {
        const int a0 = A_tnnz[posA], na = A_tnnz[posA + 1] - a0;
        const int sa = A_Ptr[(long long)posA * TSG_BS + lane];
        const int ea = lane == TSG_BS - 1 ? na : A_Ptr[(long long)posA * TSG_BS + lane + 1];
        const int b0 = B_tnnz[posB], nb = B_tnnz[posB + 1] - b0;
        const unsigned char *bp = B_Ptr + (long long)posB * TSG_BS;
        for (int x = sa; x < ea; x++)
        {
            const int ca = A_Colb[a0 + x] & 15;
            const double a = A_Val[a0 + x];
            const int sb = bp[ca];
            const int eb = ca == TSG_BS - 1 ? nb : bp[ca + 1];
            for (int y = sb; y < eb; y++)
            {
                const int c = B_Colb[b0 + y] & 15;
                myrow[c] = __dadd_rn(myrow[c], __dmul_rn(a, B_Val[b0 + y]));
            }
        }
    });
    __syncwarp(hmask);
    const int excl = C_Ptr[(long long)t * TSG_BS + lane];
    const unsigned mrev = __brev((unsigned)C_mask[(long long)t * TSG_BS + lane]) >> 16;
    // every lane runs the same trip count so the shuffles see all 16 lanes
    for (int pb = 0; pb < cn; pb += 16)
    {
        const int p = pb + lane;
        int r = 0;
#pragma unroll
        for (int s = 8; s >= 1; s >>= 1)
        {
            const int v = __shfl_sync(hmask, excl, r + s, 16);
            if (v <= p)
                r += s;
        }
        const unsigned mr = __shfl_sync(hmask, mrev, r, 16);
        const int rank = p - __shfl_sync(hmask, excl, r, 16);
        if (p < cn)
        {
            const int c = (int)__fns(mr, 0, rank + 1) & 15;
            double *cell = acc + r * S3_STRIDE + c;
            C_Colb[cb + p] = (unsigned char)c;
            C_Val[cb + p] = *cell;
            *cell = 0.0;
        }
    }
}

// ---------------------------------------------------------------------------
// Row-segment schedule (tile-level Gustavson) for steps 2 and 3.
//
// A work item is W consecutive C tiles (global order), cut at tile-row
// boundaries into segments.  For a segment of C tile row i the half-warp walks
// A's tile row i in k order and, for each A tile (i,k), the tiles of B's tile
// row k whose columns fall in the segment's column range (binary search for
// the first, then a merge against the segment's sorted C columns) -- every
// (A tile, B tile) pair of the segment is visited exactly once and no
// intersection is searched.  Lane r owns row r of every C tile of the
// segment.  Step 2 ORs boolean tile products into per-tile row masks; step 3
// accumulates a*b into a compact FP64 buffer holding exactly the segment's
// nonzeros (slot = tile offset + row offset + popcount of the row mask left
// of the column), in k-ascending then A-entry order with separately rounded
// multiply and add -- the oracle's order -- and streams the buffer out with
// contiguous stores.  A segment whose nonzeros exceed CAP is processed in
// tile sub-chunks of at most CAP values.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lower_bound_int(const int *__restrict__ a, int n, int key)
{
    int lo = 0;
    while (n > 0)
    {
        const int h = n >> 1;
        if (a[lo + h] < key)
        {
            lo += h + 1;
            n -= h + 1;
        }
        else
            n = h;
    }
    return lo;
}

template <int W>
__global__ void __launch_bounds__(128)
    k_step2_rows(int numC, const int *__restrict__ C_row, const int *__restrict__ C_col,
                 const int *__restrict__ C_ptr, const int *__restrict__ A_ptr, const int *__restrict__ A_col,
                 const unsigned short *__restrict__ A_mask, const int *__restrict__ B_ptr,
                 const int *__restrict__ B_col, const unsigned short *__restrict__ B_mask,
                 unsigned short *__restrict__ C_mask, unsigned char *__restrict__ C_Ptr, int *__restrict__ C_cnt,
                 int *__restrict__ bins)
{
    __shared__ unsigned int s_m[8][W][16];
    __shared__ int s_col[8][W];
    __shared__ int s_bins[4];
    if (threadIdx.x < 4)
        s_bins[threadIdx.x] = 0;
    __syncthreads();
    const int hw = threadIdx.x >> 4, lane = threadIdx.x & 15;
    const unsigned hmask = HW_MASK(threadIdx.x);
    const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const long long tb = item * W;
    if (tb < numC)
    {
        const int t_end = (int)min((long long)numC, tb + W);
        int t = (int)tb;
        while (t < t_end)
        {
            const int i = C_row[t];
            const int seg_end = min(t_end, C_ptr[i + 1]);
            const int n = seg_end - t;
            if (lane < n)
                s_col[hw][lane] = C_col[t + lane];
            for (int jl = 0; jl < n; jl++)
                s_m[hw][jl][lane] = 0u;
            __syncwarp(hmask);
            const int jlo = s_col[hw][0], jhi = s_col[hw][n - 1];
            for (int pa = A_ptr[i]; pa < A_ptr[i + 1]; pa++)
            {
                const int k = A_col[pa];
                const unsigned ma = A_mask[(long long)pa * TSG_BS + lane];
                const int b0 = B_ptr[k], b1 = B_ptr[k + 1];
                int pb = b0 + lower_bound_int(B_col + b0, b1 - b0, jlo);
                int jl = 0;
                for (; pb < b1; pb++)
                {
                    const int j = B_col[pb];
                    if (j > jhi)
                        break;
                    while (jl < n - 1 && s_col[hw][jl] != j)
                        jl++;
                    const uint4 *mb = reinterpret_cast<const uint4 *>(B_mask + (long long)pb * TSG_BS);
                    const uint4 q0 = __ldg(mb), q1 = __ldg(mb + 1);
                    if (ma)
                        s_m[hw][jl][lane] |= bool_row(ma, q0, q1);
                }
            }
            __syncwarp(hmask);
            for (int jl = 0; jl < n; jl++)
            {
                const unsigned acc = s_m[hw][jl][lane];
                const int cnt = __popc(acc);
                int incl = cnt;
#pragma unroll
                for (int d = 1; d < 16; d <<= 1)
                {
                    const int o = __shfl_up_sync(hmask, incl, d, 16);
                    if (lane >= d)
                        incl += o;
                }
                const int total = __shfl_sync(hmask, incl, 15, 16);
                const long long tt = t + jl;
                C_mask[tt * TSG_BS + lane] = (unsigned short)acc;
                C_Ptr[tt * TSG_BS + lane] = (unsigned char)(incl - cnt);
                if (lane == 0)
                {
                    C_cnt[tt] = total;
                    if (total > 0)
                        atomicAdd(&s_bins[total <= 32 ? 0 : total <= 224 ? 1 : total < 256 ? 2 : 3], 1);
                }
            }
            __syncwarp(hmask);
            t = seg_end;
        }
    }
    __syncthreads();
    if (threadIdx.x < 4 && s_bins[threadIdx.x])
        atomicAdd(&bins[threadIdx.x], s_bins[threadIdx.x]);
}

template <int W, int CAP>
__global__ void __launch_bounds__(128)
    k_step3_rows(int numC, const int *__restrict__ C_row, const int *__restrict__ C_col,
                 const int *__restrict__ C_ptr, const int *__restrict__ C_tnnz,
                 const unsigned short *__restrict__ C_mask, const unsigned char *__restrict__ C_Ptr,
                 const int *__restrict__ A_ptr, const int *__restrict__ A_col, const int *__restrict__ A_tnnz,
                 const unsigned char *__restrict__ A_Ptr, const unsigned char *__restrict__ A_Colb,
                 const double *__restrict__ A_Val, const int *__restrict__ B_ptr, const int *__restrict__ B_col,
                 const int *__restrict__ B_tnnz, const unsigned char *__restrict__ B_Ptr,
                 const unsigned char *__restrict__ B_Colb, const double *__restrict__ B_Val,
                 unsigned char *__restrict__ C_Colb, double *__restrict__ C_Val)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    const int hw = threadIdx.x >> 4, lane = threadIdx.x & 15;
    const unsigned hmask = HW_MASK(threadIdx.x);
    // per half-warp: acc[CAP] doubles, base[W][16] ints, mask[W][16] u32, col[W] ints
    const size_t per_hw = (size_t)CAP * 8 + (size_t)W * 16 * 4 * 2 + (size_t)W * 4;
    double *acc = reinterpret_cast<double *>(s_raw + hw * per_hw);
    int *s_base = reinterpret_cast<int *>(acc + CAP);
    unsigned *s_mk = reinterpret_cast<unsigned *>(s_base + W * 16);
    int *s_col = reinterpret_cast<int *>(s_mk + W * 16);
    const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const long long tb = item * W;
    if (tb >= numC)
        return;
    const int t_end = (int)min((long long)numC, tb + W);
    int t = (int)tb;
    while (t < t_end)
    {
        const int i = C_row[t];
        const int seg_end = min(t_end, C_ptr[i + 1]);
        int s = t;
        while (s < seg_end)
        {
            const int base0 = C_tnnz[s];
            int e = s + 1;
            while (e < seg_end && C_tnnz[e + 1] - base0 <= CAP)
                e++;
            const int n = e - s, cn = C_tnnz[e] - base0;
            if (lane < n)
                s_col[lane] = C_col[s + lane];
            for (int jl = 0; jl < n; jl++)
            {
                const long long tt = (long long)(s + jl) * TSG_BS + lane;
                s_base[jl * 16 + lane] = C_tnnz[s + jl] - base0 + C_Ptr[tt];
                s_mk[jl * 16 + lane] = C_mask[tt];
            }
            for (int q = lane; q < cn; q += 16)
                acc[q] = 0.0;
            __syncwarp(hmask);
            const int jlo = s_col[0], jhi = s_col[n - 1];
            for (int pa = A_ptr[i]; pa < A_ptr[i + 1]; pa++)
            {
                const int k = A_col[pa];
                const int b0 = B_ptr[k], b1 = B_ptr[k + 1];
                const int pb0 = b0 + lower_bound_int(B_col + b0, b1 - b0, jlo);
                const int a0 = A_tnnz[pa], na = A_tnnz[pa + 1] - a0;
                const int xa0 = A_Ptr[(long long)pa * TSG_BS + lane];
                const int xa1 = lane == TSG_BS - 1 ? na : A_Ptr[(long long)pa * TSG_BS + lane + 1];
                if (xa0 >= xa1)
                    continue;
                int jl = 0;
                for (int pb = pb0; pb < b1; pb++)
                {
                    const int j = B_col[pb];
                    if (j > jhi)
                        break;
                    while (jl < n - 1 && s_col[jl] != j)
                        jl++;
                    const int rb = s_base[jl * 16 + lane];
                    const unsigned mk = s_mk[jl * 16 + lane];
                    const int bt0 = B_tnnz[pb], nb = B_tnnz[pb + 1] - bt0;
                    const unsigned char *bp = B_Ptr + (long long)pb * TSG_BS;
                    for (int x = xa0; x < xa1; x++)
                    {
                        const int ca = A_Colb[a0 + x] & 15;
                        const double a = A_Val[a0 + x];
                        const int yb0 = bp[ca];
                        const int yb1 = ca == TSG_BS - 1 ? nb : bp[ca + 1];
                        for (int y = yb0; y < yb1; y++)
                        {
                            const int c = B_Colb[bt0 + y] & 15;
                            const int slot = rb + __popc(mk >> (16 - c));
                            if (slot < CAP)
                                acc[slot] = __dadd_rn(acc[slot], __dmul_rn(a, B_Val[bt0 + y]));
                        }
                    }
                }
            }
            __syncwarp(hmask);
            for (int q = lane; q < cn; q += 16)
                C_Val[base0 + q] = acc[q];
            for (int jl = 0; jl < n; jl++)
            {
                unsigned mk = s_mk[jl * 16 + lane];
                int p = base0 + s_base[jl * 16 + lane];
                while (mk)
                {
                    const int bit = 31 - __clz(mk); // highest set bit = smallest column
                    C_Colb[p++] = (unsigned char)(15 - bit);
                    mk &= ~(1u << bit);
                }
            }
            __syncwarp(hmask);
            s = e;
        }
        t = seg_end;
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

template <int W, int CAP>
static int launch_step3_rows(tsg_context *ctx, long long numC, const tsg_tiled *A, const tsg_tiled *B, tsg_tiled *C)
{
    const size_t per_hw = (size_t)CAP * 8 + (size_t)W * 16 * 4 * 2 + (size_t)W * 4;
    const size_t smem = 8 * per_hw;
    TSG_CUDA(cudaFuncSetAttribute(k_step3_rows<W, CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long items = (numC + W - 1) / W;
    k_step3_rows<W, CAP><<<tsg_blocks(items * 16, 128), 128, smem, ctx->stream>>>(
        (int)numC, C->tile_rowidx, C->tile_columnidx, C->tile_ptr, C->tile_nnz, C->mask, C->tile_csr_Ptr,
        A->tile_ptr, A->tile_columnidx, A->tile_nnz, A->tile_csr_Ptr, A->tile_csr_Col, A->tile_csr_Value,
        B->tile_ptr, B->tile_columnidx, B->tile_nnz, B->tile_csr_Ptr, B->tile_csr_Col, B->tile_csr_Value,
        C->tile_csr_Col, C->tile_csr_Value);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}

template <int W>
static int launch_step2_rows(tsg_context *ctx, long long numC, const tsg_tiled *A, const tsg_tiled *B, tsg_tiled *C,
                             int *d_bins)
{
    const long long items = (numC + W - 1) / W;
    k_step2_rows<W><<<tsg_blocks(items * 16, 128), 128, 0, ctx->stream>>>(
        (int)numC, C->tile_rowidx, C->tile_columnidx, C->tile_ptr, A->tile_ptr, A->tile_columnidx, A->mask,
        B->tile_ptr, B->tile_columnidx, B->mask, C->mask, C->tile_csr_Ptr, C->tile_nnz, d_bins);
    TSG_LAUNCH_CHECK();
    return TSG_OK;
}

static int launch_step3_rows_any(tsg_context *ctx, long long numC, const tsg_tiled *A, const tsg_tiled *B, tsg_tiled *C)
{
    const int W = ctx->seg_tiles, cap = ctx->acc_cap;
    if (W == 8 && cap == 256)
        return launch_step3_rows<8, 256>(ctx, numC, A, B, C);
    if (W == 8 && cap == 512)
        return launch_step3_rows<8, 512>(ctx, numC, A, B, C);
    if (W == 8 && cap == 1024)
        return launch_step3_rows<8, 1024>(ctx, numC, A, B, C);
    if (W == 16 && cap == 512)
        return launch_step3_rows<16, 512>(ctx, numC, A, B, C);
    if (W == 16 && cap == 1024)
        return launch_step3_rows<16, 1024>(ctx, numC, A, B, C);
    if (W == 16 && cap == 2048)
        return launch_step3_rows<16, 2048>(ctx, numC, A, B, C);
    return tsg_set_error(TSG_ERR_INVALID, "unsupported row schedule (%d, %d)", W, cap);
}

extern "C" int tsg_spgemm(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B, tsg_tiled *C,
                          tsg_spgemm_info *info)
{
    if (!ctx || !C)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    TSG_TRY(validate_operands(A, B));
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
    unsigned long long *d_pairs;
    int *d_bins;
    TSG_TRY(tsg_alloc(ctx, &d_pairs, 1));
    TSG_TRY(tsg_alloc(ctx, &d_bins, 4));
    TSG_CUDA(cudaMemsetAsync(d_pairs, 0, sizeof(unsigned long long), st));
    TSG_CUDA(cudaMemsetAsync(d_bins, 0, 4 * sizeof(int), st));
    TSG_TRY(tsg_alloc(ctx, &C->tile_ptr, (size_t)tilem + 1));
    long long numC = 0;
    if (tilem > 0)
    {
        k_step1<false><<<tsg_blocks(tilem, S1_WARPS), S1_WARPS * 32, 0, st>>>(
            tilem, A->tile_ptr, A->tile_columnidx, B->tile_ptr, B->tile_columnidx, C->tile_ptr, nullptr,
            nullptr, nullptr, d_pairs);
        TSG_LAUNCH_CHECK();
        TSG_TRY(tsg_scan_counts(ctx, C->tile_ptr, C->tile_ptr, tilem, &numC));
    }
    else
        TSG_CUDA(cudaMemsetAsync(C->tile_ptr, 0, sizeof(int), st));
    C->numtile = (int)numC;
    TSG_TRY(tsg_alloc(ctx, &C->tile_columnidx, (size_t)numC));
    TSG_TRY(tsg_alloc(ctx, &C->tile_rowidx, (size_t)numC));
    if (numC > 0)
    {
        k_step1<true><<<tsg_blocks(tilem, S1_WARPS), S1_WARPS * 32, 0, st>>>(
            tilem, A->tile_ptr, A->tile_columnidx, B->tile_ptr, B->tile_columnidx, nullptr, C->tile_ptr,
            C->tile_columnidx, C->tile_rowidx, nullptr);
        TSG_LAUNCH_CHECK();
    }
    if (timing)
        TSG_CUDA(cudaEventRecord(ctx->ev[1], st));

    // step 2: symbolic
    TSG_TRY(tsg_alloc(ctx, &C->mask, (size_t)numC * TSG_BS));
    TSG_TRY(tsg_alloc(ctx, &C->tile_csr_Ptr, (size_t)numC * TSG_BS));
    TSG_TRY(tsg_alloc(ctx, &C->tile_nnz, (size_t)numC + 1));
    long long nnzC = 0;
    if (numC > 0)
    {
        if (ctx->sched == TSG_SCHED_ROWS)
        {
            if (ctx->seg_tiles == 16)
                TSG_TRY(launch_step2_rows<16>(ctx, numC, A, B, C, d_bins));
            else
                TSG_TRY(launch_step2_rows<8>(ctx, numC, A, B, C, d_bins));
        }
        else
        {
            k_step2<<<tsg_blocks(numC * 16, 256), 256, 0, st>>>(
                (int)numC, C->tile_rowidx, C->tile_columnidx, A->tile_ptr, A->tile_columnidx, A->mask,
                B->csc_tile_ptr, B->csc_tile_rowidx, B->csc_tile_pos, B->mask, C->mask, C->tile_csr_Ptr,
                C->tile_nnz, d_bins);
            TSG_LAUNCH_CHECK();
        }
        TSG_TRY(tsg_scan_counts(ctx, C->tile_nnz, C->tile_nnz, numC, &nnzC));
    }
    else
        TSG_CUDA(cudaMemsetAsync(C->tile_nnz, 0, sizeof(int), st));
    C->nnz = (int)nnzC;
    if (timing)
        TSG_CUDA(cudaEventRecord(ctx->ev[2], st));

    // step 3: numeric
    TSG_TRY(tsg_alloc(ctx, &C->tile_csr_Col, (size_t)nnzC));
    TSG_TRY(tsg_alloc(ctx, &C->tile_csr_Value, (size_t)nnzC));
    if (nnzC > 0 && ctx->sched == TSG_SCHED_ROWS)
        TSG_TRY(launch_step3_rows_any(ctx, numC, A, B, C));
    else if (nnzC > 0)
    {
        k_step3<<<tsg_blocks(numC * 16, S3_THREADS), S3_THREADS, 0, st>>>(
            (int)numC, C->tile_rowidx, C->tile_columnidx, A->tile_ptr, A->tile_columnidx, A->tile_nnz,
            A->tile_csr_Ptr, A->tile_csr_Col, A->tile_csr_Value, B->csc_tile_ptr, B->csc_tile_rowidx,
            B->csc_tile_pos, B->tile_nnz, B->tile_csr_Ptr, B->tile_csr_Col, B->tile_csr_Value, C->tile_nnz,
            C->mask, C->tile_csr_Ptr, C->tile_csr_Col, C->tile_csr_Value);
        TSG_LAUNCH_CHECK();
    }
    if (timing)
        TSG_CUDA(cudaEventRecord(ctx->ev[3], st));

    if (info)
    {
        memset(info, 0, sizeof(*info));
        info->numtile_C = numC;
        info->nnz_C = nnzC;
        long long *h = ctx->h_pinned;
        TSG_CUDA(cudaMemcpyAsync(h, d_pairs, sizeof(long long), cudaMemcpyDeviceToHost, st));
        TSG_CUDA(cudaMemcpyAsync(h + 1, d_bins, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
        TSG_CUDA(cudaStreamSynchronize(st));
        info->tile_pairs = h[0];
        memcpy(info->bins, h + 1, 4 * sizeof(int));
        if (timing)
        {
            info->ms_step1 = ev_ms(ctx->ev[0], ctx->ev[1]);
            info->ms_step2 = ev_ms(ctx->ev[1], ctx->ev[2]);
            info->ms_step3 = ev_ms(ctx->ev[2], ctx->ev[3]);
            info->ms_total = ev_ms(ctx->ev[0], ctx->ev[3]);
        }
    }
    tsg_release(ctx, d_pairs);
    tsg_release(ctx, d_bins);
    return TSG_OK;
}

// Number of C tiles of A*B (step 1's count pass only); A and B need their
// row-major tile structure.
int tsg_count_c_tiles(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B, long long *numC)
{
    *numC = 0;
    if (A->tilem == 0)
        return TSG_OK;
    int *cnt;
    TSG_TRY(tsg_alloc(ctx, &cnt, (size_t)A->tilem + 1));
    k_step1<false><<<tsg_blocks(A->tilem, S1_WARPS), S1_WARPS * 32, 0, ctx->stream>>>(
        A->tilem, A->tile_ptr, A->tile_columnidx, B->tile_ptr, B->tile_columnidx, cnt, nullptr, nullptr, nullptr,
        nullptr);
    TSG_LAUNCH_CHECK();
    TSG_TRY(tsg_scan_counts(ctx, cnt, cnt, A->tilem, numC));
    tsg_release(ctx, cnt);
    return TSG_OK;
}
