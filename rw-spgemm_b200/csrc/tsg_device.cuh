// Device-side building blocks of the tiled SpGEMM, shared by the
// one-product kernels (tsg_spgemm.cu) and the batched persistent kernel
// (tsg_batch.cu), so both compute with identical code and order.
//
// Restates the three steps of the reference's tilespgemm()
// (src/tilespgemm-cuda.h:2610-3221): step 1 tile structure of C (:257-369),
// step 2 per-tile bitmask symbolic (:371-755), step 3 numeric (:1505-2608).
// Every C entry is accumulated as 0.0 + p1 + p2 + ... in k-ascending, then
// A-entry order with separately rounded multiply and add: the order and
// rounding of the reference's CPU oracle (src/spgemm-cpu.h:330), so the
// results are bit-identical to it and deterministic -- no FP64 atomics.
#pragma once

#include <limits.h>

#include "tsg_internal.h"

#define TSG_FULL_MASK 0xffffffffu
#define TSG_HW_MASK(tid) (0xFFFFu << ((tid) & 16))

// Pointers of one product C = A*B.  A: row-major tiles; B: row-major tiles
// plus the column view; C: outputs.
struct ProdView
{
    const int *A_ptr, *A_col, *A_tnnz;
    const unsigned char *A_Ptr, *A_Colb;
    const double *A_Val;
    const unsigned short *A_mask;
    int tilemA;
    const int *B_ptr, *B_col, *B_cptr, *B_crow, *B_cpos, *B_tnnz;
    const unsigned char *B_Ptr, *B_Colb;
    const double *B_Val;
    const unsigned short *B_mask;
    const unsigned short *B_maskT;
    const int *B_rptr, *B_rcol; // row view of B (scalar CSR), may be null
    const double *B_rval;
    int browB; // mean entries per row of B (rounded down)
    int tilenB;
    int *C_ptr, *C_col, *C_row, *C_tnnz;
    unsigned short *C_mask;
    unsigned char *C_Ptr, *C_Colb;
    double *C_Val;
    int numC;
    int padded;  // every array allocated by tsg_alloc (16-byte aligned, 16 bytes of slack at the end)
    int *status; // device status word for errors found inside a kernel (or null)
};

// ---------------------------------------------------------------------------
// Step 1 (warp per A tile row): the tile-column lists of the B tile rows the
// A tile row touches are ORed into a shared-memory bitmap restricted to the
// row's column window (S1_WORDS words per pass); popcount gives the count,
// an ordered bit walk emits the sorted C tile columns.
// ---------------------------------------------------------------------------
#define S1_WORDS 1024

template <bool EMIT>
__device__ __forceinline__ int step1_row(const ProdView &P, int i, unsigned int *bm, int lane,
                                         unsigned long long *pairs)
{
    const int a0 = P.A_ptr[i], a1 = P.A_ptr[i + 1];
    int lo = INT_MAX, hi = -1;
    unsigned long long np = 0;
    for (int pa = a0 + lane; pa < a1; pa += 32)
    {
        const int k = P.A_col[pa];
        const int b0 = P.B_ptr[k], b1 = P.B_ptr[k + 1];
        if (b1 > b0)
        {
            lo = min(lo, P.B_col[b0]);
            hi = max(hi, P.B_col[b1 - 1]);
            np += (unsigned long long)(b1 - b0);
        }
    }
    lo = __reduce_min_sync(TSG_FULL_MASK, lo);
    hi = __reduce_max_sync(TSG_FULL_MASK, hi);
    if (!EMIT && pairs)
    {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1)
            np += __shfl_xor_sync(TSG_FULL_MASK, np, d);
        if (lane == 0 && np)
            atomicAdd(pairs, np);
    }
    int out = 0;
    const int cbase = EMIT ? P.C_ptr[i] : 0;
    if (hi >= 0)
    {
        for (int c0 = lo & ~31; c0 <= hi; c0 += S1_WORDS * 32)
        {
            const int c1 = min(hi + 1, c0 + S1_WORDS * 32);
            const int nw = (c1 - c0 + 31) >> 5;
            for (int w = lane; w < nw; w += 32)
                bm[w] = 0;
            __syncwarp();
            // A's tiles 32 at a time, a lane each; their B tile rows' tiles
            // are either flattened over the lanes (short rows) or walked one
            // A tile after another, a lane per B tile
            for (int g = a0; g < a1; g += 32)
            {
                const int cnt = min(32, a1 - g);
                int b0 = 0, len = 0;
                if (lane < cnt)
                {
                    const int k = P.A_col[g + lane];
                    b0 = P.B_ptr[k];
                    len = P.B_ptr[k + 1] - b0;
                }
                int incl = len;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1)
                {
                    const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
                    if (lane >= d)
                        incl += o;
                }
                const int total = __shfl_sync(TSG_FULL_MASK, incl, 31);
                const int pre = incl - len;
                if (total < 16 * cnt)
                {
                    for (int base = 0; base < total; base += 32)
                    {
                        const int item = base + lane;
                        // the A tile of this pair: the last one whose first pair is at or before it
                        int t = 0;
#pragma unroll
                        for (int sz = 16; sz > 0; sz >>= 1)
                        {
                            const int pc = __shfl_sync(TSG_FULL_MASK, pre, t + sz);
                            if (t + sz < cnt && pc <= item)
                                t += sz;
                        }
                        const int ob = __shfl_sync(TSG_FULL_MASK, b0, t);
                        const int op = __shfl_sync(TSG_FULL_MASK, pre, t);
                        if (item < total)
                        {
                            const int j = P.B_col[ob + item - op];
                            if (j >= c0 && j < c1)
                                atomicOr(&bm[(j - c0) >> 5], 1u << ((j - c0) & 31));
                        }
                    }
                }
                else
                {
                    for (int t = 0; t < cnt; t++)
                    {
                        const int tb = __shfl_sync(TSG_FULL_MASK, b0, t);
                        const int tl = __shfl_sync(TSG_FULL_MASK, len, t);
                        for (int pb = tb + lane; pb < tb + tl; pb += 32)
                        {
                            const int j = P.B_col[pb];
                            if (j >= c0 && j < c1)
                                atomicOr(&bm[(j - c0) >> 5], 1u << ((j - c0) & 31));
                        }
                    }
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
                        const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
                        if (lane >= d)
                            incl += o;
                    }
                    int pos = cbase + out + incl - cnt;
                    while (bits)
                    {
                        const int b = __ffs(bits) - 1;
                        bits &= bits - 1;
                        P.C_col[pos] = c0 + (w << 5) + b;
                        P.C_row[pos] = i;
                        pos++;
                    }
                    out += __shfl_sync(TSG_FULL_MASK, incl, 31);
                }
                else
                {
                    out += __reduce_add_sync(TSG_FULL_MASK, cnt);
                }
            }
            __syncwarp();
        }
    }
    return out;
}

// forward declarations of helpers defined below
__device__ __forceinline__ unsigned bool_row(unsigned ma, uint4 q0, uint4 q1);
__device__ __forceinline__ int hw_excl_scan(unsigned hmask, int lane, int cnt, int &total);
__device__ __forceinline__ int nnz_bin(int total);

// ---------------------------------------------------------------------------
// Fused step 1 (emit) + step 2 for one A tile row (warp).  The row's C tile
// columns come from the window bitmap as in step1_row; when the window fits
// one pass of S12_WORDS words and the row has at most S12_MAXT C tiles, the
// bitmap's word-prefix popcounts give each B tile's C slot in O(1), and the
// warp ORs the 16x16 boolean products of every (A tile, B tile) pair of the
// row into per-slot row masks in shared memory (two B tiles at a time, one
// per half-warp, lane = row), then writes masks, row offsets and tile counts.
// No intersection is searched.  Returns 1 if the row was completed, 0 if it
// needs the tile-schedule step 2 (C columns are emitted either way).
// ---------------------------------------------------------------------------
#define S12_WORDS 256
#define S12_MAXT 128

struct S12Smem
{
    unsigned bm[S12_WORDS];
    unsigned short pre[S12_WORDS];
    unsigned short acc[16][S12_MAXT + 2]; // [row][slot], padded: both access forms spread over banks
};

__device__ __forceinline__ int step12_row(const ProdView &P, int i, S12Smem &sm, int lane, int *s_bins)
{
    const int a0 = P.A_ptr[i], a1 = P.A_ptr[i + 1];
    int lo = INT_MAX, hi = -1;
    for (int pa = a0 + lane; pa < a1; pa += 32)
    {
        const int k = P.A_col[pa];
        const int b0 = P.B_ptr[k], b1 = P.B_ptr[k + 1];
        if (b1 > b0)
        {
            lo = min(lo, P.B_col[b0]);
            hi = max(hi, P.B_col[b1 - 1]);
        }
    }
    lo = __reduce_min_sync(TSG_FULL_MASK, lo);
    hi = __reduce_max_sync(TSG_FULL_MASK, hi);
    const int cbase = P.C_ptr[i];
    const int ntiles = P.C_ptr[i + 1] - cbase;
    if (hi < 0)
        return 1;
    const int c0 = lo & ~31;
    const int nw = (hi - c0 + 32) >> 5;
    if (nw > S12_WORDS || ntiles > S12_MAXT)
        return 0; // wide row: the caller emits it with step1_row and runs step 2 per tile
    for (int w = lane; w < nw; w += 32)
        sm.bm[w] = 0;
    __syncwarp();
    for (int pa = a0; pa < a1; pa++)
    {
        const int k = P.A_col[pa];
        const int b0 = P.B_ptr[k], b1 = P.B_ptr[k + 1];
        for (int pb = b0 + lane; pb < b1; pb += 32)
        {
            const int j = P.B_col[pb] - c0;
            atomicOr(&sm.bm[j >> 5], 1u << (j & 31));
        }
    }
    __syncwarp();
    // word prefix popcounts (exclusive) and the sorted C columns
    int run = 0;
    for (int wb = 0; wb < nw; wb += 32)
    {
        const int w = wb + lane;
        unsigned bits = w < nw ? sm.bm[w] : 0u;
        const int cnt = __popc(bits);
        int incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
            if (lane >= d)
                incl += o;
        }
        int pos = run + incl - cnt;
        if (w < nw)
            sm.pre[w] = (unsigned short)pos;
        while (bits)
        {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            P.C_col[cbase + pos] = c0 + (w << 5) + b;
            P.C_row[cbase + pos] = i;
            pos++;
        }
        run += __shfl_sync(TSG_FULL_MASK, incl, 31);
    }
    const int r = lane & 15, half = lane >> 4;
    for (int q = half; q < ntiles; q += 2)
        sm.acc[r][q] = 0;
    __syncwarp();
    // OR the boolean products of all (A tile, B tile) pairs of the row: unit
    // (row r, B tile) ORs the B rows its A row meets -- one 16-bit load per
    // set bit of a sparse A row, two 16-byte loads for a dense one
    for (int pa = a0; pa < a1; pa++)
    {
        const int k = P.A_col[pa];
        const int b0 = P.B_ptr[k], b1 = P.B_ptr[k + 1];
        if (b1 - b0 >= 8)
        {
            // lane per B tile; the A tile's row masks are the same for all
            // lanes, so the walk over its set bits does not diverge
            const uint4 *amq = reinterpret_cast<const uint4 *>(P.A_mask + (long long)pa * TSG_BS);
            const uint4 aq0 = __ldg(amq), aq1 = __ldg(amq + 1);
            const unsigned aw[8] = {aq0.x, aq0.y, aq0.z, aq0.w, aq1.x, aq1.y, aq1.z, aq1.w};
            // A tile with a dense row: B's masks as two 16-byte loads
            const bool adense = __popc(aq0.x) + __popc(aq0.y) + __popc(aq0.z) + __popc(aq0.w) + __popc(aq1.x) +
                                    __popc(aq1.y) + __popc(aq1.z) + __popc(aq1.w) > 64;
            for (int pb = b0 + lane; pb < b1; pb += 32)
            {
                const int j = P.B_col[pb] - c0;
                const int slot = sm.pre[j >> 5] + __popc(sm.bm[j >> 5] & ((1u << (j & 31)) - 1u));
                const unsigned short *mbk = P.B_mask + (long long)pb * TSG_BS;
                if (adense)
                {
                    const uint4 *mb = reinterpret_cast<const uint4 *>(mbk);
                    const uint4 q0 = __ldg(mb), q1 = __ldg(mb + 1);
#pragma unroll
                    for (int rr = 0; rr < 16; rr++)
                    {
                        const unsigned mrow = (rr & 1) ? (aw[rr >> 1] >> 16) : (aw[rr >> 1] & 0xFFFFu);
                        if (mrow)
                            sm.acc[rr][slot] |= (unsigned short)bool_row(mrow, q0, q1);
                    }
                    continue;
                }
#pragma unroll
                for (int rr = 0; rr < 16; rr++)
                {
                    const unsigned mrow = (rr & 1) ? (aw[rr >> 1] >> 16) : (aw[rr >> 1] & 0xFFFFu);
                    if (!mrow)
                        continue;
                    unsigned acc = 0, bits = mrow;
                    do
                    {
                        const int bit = 31 - __clz(bits);
                        bits ^= 1u << bit;
                        acc |= __ldg(mbk + (15 - bit));
                    } while (bits);
                    sm.acc[rr][slot] |= (unsigned short)acc;
                }
            }
            __syncwarp();
            continue;
        }
        const unsigned ma = P.A_mask[(long long)pa * TSG_BS + r];
        if (ma)
        {
            const bool dense_row = __popc(ma) > 4;
            for (int pb = b0 + half; pb < b1; pb += 2)
            {
                const int j = P.B_col[pb] - c0;
                const int slot = sm.pre[j >> 5] + __popc(sm.bm[j >> 5] & ((1u << (j & 31)) - 1u));
                const unsigned short *mbk = P.B_mask + (long long)pb * TSG_BS;
                unsigned acc = 0;
                if (dense_row)
                {
                    const uint4 *mb = reinterpret_cast<const uint4 *>(mbk);
                    acc = bool_row(ma, __ldg(mb), __ldg(mb + 1));
                }
                else
                {
                    unsigned bits = ma;
                    do
                    {
                        const int bit = 31 - __clz(bits);
                        bits ^= 1u << bit;
                        acc |= __ldg(mbk + (15 - bit));
                    } while (bits);
                }
                sm.acc[r][slot] |= (unsigned short)acc;
            }
        }
        __syncwarp();
    }
    // row offsets, masks and counts, one C tile per half-warp
    const unsigned hmask = TSG_HW_MASK(threadIdx.x);
    for (int q0 = 0; q0 < ntiles; q0 += 2)
    {
        const int q = q0 + half;
        const unsigned accm = q < ntiles ? sm.acc[r][q] : 0u;
        int total;
        const int excl = hw_excl_scan(hmask, r, __popc(accm), total);
        if (q < ntiles)
        {
            const long long t = cbase + q;
            P.C_mask[t * TSG_BS + r] = (unsigned short)accm;
            P.C_Ptr[t * TSG_BS + r] = (unsigned char)excl;
            if (r == 0)
            {
                P.C_tnnz[t] = total;
                if (total > 0 && s_bins)
                    atomicAdd(&s_bins[nnz_bin(total)], 1);
            }
        }
    }
    __syncwarp();
    return 1;
}

// ---------------------------------------------------------------------------
// Helpers
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

// Row r of a 16x16 boolean tile product: OR of B's row masks c for every
// column c set in A's row mask (bit 15-c).  q0/q1 hold B's 16 row masks
// (rows 2w and 2w+1 in the low and high halves of word w).
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

// Exclusive half-warp scan of cnt; returns the exclusive value, total via ref.
__device__ __forceinline__ int hw_excl_scan(unsigned hmask, int lane, int cnt, int &total)
{
    int incl = cnt;
#pragma unroll
    for (int d = 1; d < 16; d <<= 1)
    {
        const int o = __shfl_up_sync(hmask, incl, d, 16);
        if (lane >= d)
            incl += o;
    }
    total = __shfl_sync(hmask, incl, 15, 16);
    return incl - cnt;
}

__device__ __forceinline__ int nnz_bin(int total)
{
    return total <= 32 ? 0 : total <= 224 ? 1 : total < 256 ? 2 : 3;
}

// Writes row r's mask, offset and (lane 0) the tile count / bin of tile t.
__device__ __forceinline__ void step2_store(const ProdView &P, long long t, unsigned hmask, int lane, unsigned acc,
                                            int *s_bins)
{
    int total;
    const int excl = hw_excl_scan(hmask, lane, __popc(acc), total);
    P.C_mask[t * TSG_BS + lane] = (unsigned short)acc;
    P.C_Ptr[t * TSG_BS + lane] = (unsigned char)excl;
    if (lane == 0)
    {
        P.C_tnnz[t] = total;
        if (total > 0 && s_bins)
            atomicAdd(&s_bins[nnz_bin(total)], 1);
    }
}

// ---------------------------------------------------------------------------
// Tile schedule: half-warp per C tile, A's tile row intersected with B's tile
// column 16 elements at a time, the chunks held in lanes' registers (shuffle
// binary search + ballot); f(posA, posB) is called for every matched k in
// ascending order, uniformly across the half-warp.
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

__device__ __forceinline__ void step2_tile(const ProdView &P, int t, unsigned hmask, int lane, int *s_bins)
{
    const int i = P.C_row[t], j = P.C_col[t];
    const int abase = P.A_ptr[i], la = P.A_ptr[i + 1] - abase;
    const int bbase = P.B_cptr[j], lb = P.B_cptr[j + 1] - bbase;
    unsigned acc = 0;
    intersect_tiles(hmask, lane, P.A_col, abase, la, P.B_crow, P.B_cpos, bbase, lb, [&](int posA, int posB) {
        const unsigned ma = P.A_mask[(long long)posA * TSG_BS + lane];
        const unsigned short *mbk = P.B_mask + (long long)posB * TSG_BS;
        if (__popc(ma) > 4)
        {
            const uint4 *mb = reinterpret_cast<const uint4 *>(mbk);
            acc |= bool_row(ma, __ldg(mb), __ldg(mb + 1));
        }
        else
        {
            unsigned bits = ma;
            while (bits)
            {
                const int bit = 31 - __clz(bits);
                bits ^= 1u << bit;
                acc |= __ldg(mbk + (15 - bit));
            }
        }
    });
    step2_store(P, t, hmask, lane, acc, s_bins);
}

#define S3T_STRIDE 17

// acc: 16 x S3T_STRIDE doubles of this half-warp, all zero on entry and on exit
__device__ __forceinline__ void step3_tile(const ProdView &P, int t, unsigned hmask, int lane, double *acc)
{
    const int cb = P.C_tnnz[t], cn = P.C_tnnz[t + 1] - cb;
    if (cn == 0)
        return;
    const int i = P.C_row[t], j = P.C_col[t];
    const int abase = P.A_ptr[i], la = P.A_ptr[i + 1] - abase;
    const int bbase = P.B_cptr[j], lb = P.B_cptr[j + 1] - bbase;
    double *myrow = acc + lane * S3T_STRIDE;
    intersect_tiles(hmask, lane, P.A_col, abase, la, P.B_crow, P.B_cpos, bbase, lb, [&](int posA, int posB) {
        const int a0 = P.A_tnnz[posA], na = P.A_tnnz[posA + 1] - a0;
        const int sa = P.A_Ptr[(long long)posA * TSG_BS + lane];
        const int ea = lane == TSG_BS - 1 ? na : P.A_Ptr[(long long)posA * TSG_BS + lane + 1];
        const int b0 = P.B_tnnz[posB], nb = P.B_tnnz[posB + 1] - b0;
        const unsigned char *bp = P.B_Ptr + (long long)posB * TSG_BS;
        for (int x = sa; x < ea; x++)
        {
            const int ca = P.A_Colb[a0 + x] & 15;
            const double a = P.A_Val[a0 + x];
            const int sb = bp[ca];
            const int eb = ca == TSG_BS - 1 ? nb : bp[ca + 1];
            for (int y = sb; y < eb; y++)
            {
                const int c = P.B_Colb[b0 + y] & 15;
                myrow[c] = __dadd_rn(myrow[c], __dmul_rn(a, P.B_Val[b0 + y]));
            }
        }
    });
    __syncwarp(hmask);
    const int excl = P.C_Ptr[(long long)t * TSG_BS + lane];
    const unsigned mrev = __brev((unsigned)P.C_mask[(long long)t * TSG_BS + lane]) >> 16;
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
            double *cell = acc + r * S3T_STRIDE + c;
            P.C_Colb[cb + p] = (unsigned char)c;
            P.C_Val[cb + p] = *cell;
            *cell = 0.0;
        }
    }
    __syncwarp(hmask);
}

// ---------------------------------------------------------------------------
// Row-segment schedule (tile-level Gustavson).  A work item is W consecutive
// C tiles (global order), cut at tile-row boundaries into segments.  For a
// segment of C tile row i the half-warp walks A's tile row i in k order and,
// for each A tile (i,k), the tiles of B's tile row k whose columns fall in
// the segment's range (binary search for the first, then a merge against the
// segment's sorted C columns): every (A tile, B tile) pair is visited once
// and no intersection is searched.  Lane r owns row r of every C tile of the
// segment.
// ---------------------------------------------------------------------------
template <int W>
struct S2RowsSmem
{
    unsigned m[W][16];
    int col[W];
};

template <int W>
__device__ __forceinline__ void step2_rows_item(const ProdView &P, long long item, unsigned hmask, int lane,
                                                S2RowsSmem<W> &sm, int *s_bins)
{
    const long long tb = item * W;
    if (tb >= P.numC)
        return;
    const int t_end = (int)min((long long)P.numC, tb + W);
    int t = (int)tb;
    while (t < t_end)
    {
        const int i = P.C_row[t];
        const int seg_end = min(t_end, P.C_ptr[i + 1]);
        const int n = seg_end - t;
        for (int jl = lane; jl < n; jl += 16)
            sm.col[jl] = P.C_col[t + jl];
        for (int jl = 0; jl < n; jl++)
            sm.m[jl][lane] = 0u;
        __syncwarp(hmask);
        const int jlo = sm.col[0], jhi = sm.col[n - 1];
        for (int pa = P.A_ptr[i]; pa < P.A_ptr[i + 1]; pa++)
        {
            const int k = P.A_col[pa];
            const unsigned ma = P.A_mask[(long long)pa * TSG_BS + lane];
            const int b0 = P.B_ptr[k], b1 = P.B_ptr[k + 1];
            int jl = 0;
            for (int pb = b0 + lower_bound_int(P.B_col + b0, b1 - b0, jlo); pb < b1; pb++)
            {
                const int j = P.B_col[pb];
                if (j > jhi)
                    break;
                while (jl < n - 1 && sm.col[jl] != j)
                    jl++;
                const uint4 *mb = reinterpret_cast<const uint4 *>(P.B_mask + (long long)pb * TSG_BS);
                const uint4 q0 = __ldg(mb), q1 = __ldg(mb + 1);
                if (ma)
                    sm.m[jl][lane] |= bool_row(ma, q0, q1);
            }
        }
        __syncwarp(hmask);
        for (int jl = 0; jl < n; jl++)
            step2_store(P, t + jl, hmask, lane, sm.m[jl][lane], s_bins);
        __syncwarp(hmask);
        t = seg_end;
    }
}

// Per half-warp shared memory of the numeric row-segment step.
template <int W, int CAP>
struct S3RowsSmem
{
    double acc[CAP];
    unsigned bm[W * 16]; // (first slot of the row in the sub-chunk << 16) | row mask
    int col[W];
};

// Accumulates a*b into a compact FP64 buffer holding exactly the sub-chunk's
// nonzeros (slot = tile offset + row offset + popcount of the row mask left
// of the column); B rows are walked through their 16-bit masks (no column
// byte loads); the buffer is written out with contiguous stores.  A segment
// with more than CAP nonzeros is processed in tile sub-chunks.
template <int W, int CAP>
__device__ __forceinline__ void step3_rows_item(const ProdView &P, long long item, unsigned hmask, int lane,
                                                S3RowsSmem<W, CAP> &sm)
{
    const long long tb = item * W;
    if (tb >= P.numC)
        return;
    const int t_end = (int)min((long long)P.numC, tb + W);
    int t = (int)tb;
    while (t < t_end)
    {
        const int i = P.C_row[t];
        const int seg_end = min(t_end, P.C_ptr[i + 1]);
        int s = t;
        while (s < seg_end)
        {
            const int base0 = P.C_tnnz[s];
            int e = s + 1;
            while (e < seg_end && P.C_tnnz[e + 1] - base0 <= CAP)
                e++;
            const int n = e - s, cn = P.C_tnnz[e] - base0;
            for (int jl = lane; jl < n; jl += 16)
                sm.col[jl] = P.C_col[s + jl];
            for (int jl = 0; jl < n; jl++)
            {
                const long long tt = (long long)(s + jl) * TSG_BS + lane;
                const unsigned b = (unsigned)(P.C_tnnz[s + jl] - base0 + P.C_Ptr[tt]);
                sm.bm[jl * 16 + lane] = (b << 16) | P.C_mask[tt];
            }
            for (int q = lane; q < cn; q += 16)
                sm.acc[q] = 0.0;
            __syncwarp(hmask);
            const int jlo = sm.col[0], jhi = sm.col[n - 1];
            for (int pa = P.A_ptr[i]; pa < P.A_ptr[i + 1]; pa++)
            {
                const int k = P.A_col[pa];
                const int b0 = P.B_ptr[k], b1 = P.B_ptr[k + 1];
                const int pb0 = b0 + lower_bound_int(P.B_col + b0, b1 - b0, jlo);
                const int a0 = P.A_tnnz[pa];
                const int xa0 = a0 + P.A_Ptr[(long long)pa * TSG_BS + lane];
                const int xa1 = a0 + (lane == TSG_BS - 1 ? P.A_tnnz[pa + 1] - a0
                                                          : P.A_Ptr[(long long)pa * TSG_BS + lane + 1]);
                if (xa0 >= xa1)
                    continue;
                int jl = 0;
                for (int pb = pb0; pb < b1; pb++)
                {
                    const int j = P.B_col[pb];
                    if (j > jhi)
                        break;
                    while (jl < n - 1 && sm.col[jl] != j)
                        jl++;
                    const unsigned bm = sm.bm[jl * 16 + lane];
                    const int rb = (int)(bm >> 16);
                    const unsigned mk = bm & 0xFFFFu;
                    const double *bv = P.B_Val + P.B_tnnz[pb];
                    const unsigned short *bmask = P.B_mask + (long long)pb * TSG_BS;
                    const unsigned char *bp = P.B_Ptr + (long long)pb * TSG_BS;
                    for (int x = xa0; x < xa1; x++)
                    {
                        const int ca = P.A_Colb[x] & 15;
                        unsigned mb = bmask[ca];
                        if (!mb)
                            continue;
                        const double a = P.A_Val[x];
                        int y = bp[ca];
                        do // B row ca's columns, ascending (highest mask bit first)
                        {
                            const int bit = 31 - __clz(mb);
                            const int slot = rb + __popc(mk >> (bit + 1));
                            if (slot < CAP)
                                sm.acc[slot] = __dadd_rn(sm.acc[slot], __dmul_rn(a, bv[y]));
                            y++;
                            mb ^= 1u << bit;
                        } while (mb);
                    }
                }
            }
            __syncwarp(hmask);
            for (int q = lane; q < cn; q += 16)
                P.C_Val[base0 + q] = sm.acc[q];
            for (int jl = 0; jl < n; jl++)
            {
                const unsigned bm = sm.bm[jl * 16 + lane];
                unsigned mk = bm & 0xFFFFu;
                int p = base0 + (int)(bm >> 16);
                while (mk)
                {
                    const int bit = 31 - __clz(mk);
                    P.C_Colb[p++] = (unsigned char)(15 - bit);
                    mk ^= 1u << bit;
                }
            }
            __syncwarp(hmask);
            s = e;
        }
        t = seg_end;
    }
}

// ---------------------------------------------------------------------------
// Numeric step, SPA schedule (row Gustavson over B's row view).  One CTA of
// SPA_WARPS warps owns a segment of consecutive C tiles of one tile row I
// (at most SPA_CAP values, SPA_SEGT tiles, a tile-column window of SPA_WIN);
// warp r owns C row 16 I + r.  The segment's values are accumulated in shared
// memory in C's own output layout: the slot of C(r, c) is the tile's value
// offset + its row-r offset + the popcount of the row mask left of c, the
// tile found through a window map.  Warp r walks A's row r through the row's
// tiles in column order; for every A(r, k) it streams B's row k (scalar CSR:
// coalesced column and value loads, the next row's first 32 entries
// prefetched) and each lane adds a * b into the slot of its entry's column.
// A's entries of one row are applied one after another (warp barrier between
// them), so every C entry sums its products in k order -- the reference's
// order -- with multiply and add rounded separately.
// ---------------------------------------------------------------------------
#define SPA_WARPS 16
#define SPA_THREADS (SPA_WARPS * 32)
#define SPA_CAP 4096
#define SPA_SEGT 256
#define SPA_CMS (SPA_SEGT + 1) // row stride of the [row][tile] words: a tile's 16 rows in 16 banks
#define SPA_WIN 2048
#define SPA_STAGE 64
#define SPA_DENSE TSG_SPA_DENSE_DEFAULT
#define SPA_FLAT 16  // B rows averaging fewer entries (inside a segment) have their products flattened

// entry of A value v in a chunk of an A tile row: its tile p (the last of tile0[0..nt)
// starting at or before v, plus p0), its row (from the tile's row offsets)
// and its column k
__device__ __forceinline__ void a_entry(const ProdView &P, const int *tile0, int nt, int p0, bool ptr16, int v,
                                        int &row, int &k)
{
    int lo = 0, hi = nt - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (tile0[mid] <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int p = p0 + lo, o = v - tile0[lo];
    // the row: how many of the tile's row offsets 1..15 are at or below o
    const unsigned char *rp = P.A_Ptr + (long long)p * TSG_BS;
    uint4 w;
    if (ptr16)
        w = *reinterpret_cast<const uint4 *>(rp);
    else
    {
        unsigned u[4];
        for (int q = 0; q < 4; q++)
            u[q] = rp[4 * q] | (rp[4 * q + 1] << 8) | (rp[4 * q + 2] << 16) | ((unsigned)rp[4 * q + 3] << 24);
        w = make_uint4(u[0], u[1], u[2], u[3]);
    }
    const unsigned ob = (unsigned)o * 0x01010101u;
    row = (__popc(__vcmpleu4(w.x, ob)) + __popc(__vcmpleu4(w.y, ob)) + __popc(__vcmpleu4(w.z, ob)) +
           __popc(__vcmpleu4(w.w, ob))) / 8 - 1;
    k = P.A_col[p] * TSG_BS + (P.A_Colb[v] & 15);
}

// the first A tile of tile row [pa_beg, pa_end) holding value offset c0
__device__ __forceinline__ int a_tile_of(const ProdView &P, int pa_beg, int pa_end, int c0)
{
    int lo = pa_beg, hi = pa_end - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (P.A_tnnz[mid] <= c0)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

struct SpaStage
{
    int2 bl[SPA_STAGE]; // B row: first entry, length
    double a[SPA_STAGE];
};

// The FLAT form stages A's entries with the whole CTA, SPA_CO_CHUNK at a
// time (spa_coop_apply).
#define SPA_CO_CHUNK 768
#define SPA_CO_SLOTS (SPA_CO_CHUNK / 32)

struct SpaCoop
{
    int2 bl[SPA_CO_CHUNK];        // B row (first entry, length) of each staged A entry, grouped by row
    double a[SPA_CO_CHUNK];
    int tile0[SPA_CO_CHUNK + 1];  // value offset of each A tile the chunk can touch
    int wc[SPA_CO_SLOTS][TSG_BS]; // staged entries per (32-entry slot, row), then their offsets in the row
    int rbeg[TSG_BS + 1];         // first staged entry of each row
    int ptile;                    // the chunk's first A tile
};

struct SpaSmem
{
    double acc[SPA_CAP];
    unsigned cm[TSG_BS * SPA_CMS];  // [row][tile]: (entries of the row in earlier tiles << 16) | C row mask
    int rstart[TSG_BS];             // first accumulator slot of each row's private, column-sorted run
    unsigned short map[SPA_WIN];    // tile column - J0 -> segment tile, 0xFFFF none
    union
    {
        SpaStage stage[SPA_WARPS]; // per-row form
        SpaCoop co;                // FLAT form
    };
};

// accumulator slot of column col in the row (cmr, rs), -1 outside the segment
__device__ __forceinline__ int spa_slot(const SpaSmem &S, const unsigned *cmr, int rs, int J0, int J1, bool full,
                                        int col)
{
    const int J = col >> 4;
    if (!full && (J < J0 || J >= J1 || J - J0 >= SPA_WIN))
        return -1;
    const int slot = S.map[J - J0];
    if (slot >= SPA_SEGT)
        return -1;
    const unsigned cmw = cmr[slot];
    const int pos = rs + (int)(cmw >> 16) + __popc((cmw & 0xFFFFu) >> (16 - (col & 15)));
    return pos < SPA_CAP ? pos : -1;
}

__device__ __forceinline__ void spa_add(SpaSmem &S, const unsigned *cmr, int rs, int J0, int J1, bool full, int col,
                                        double a, double b)
{
    const int J = col >> 4;
    if (!full && (J < J0 || J >= J1 || J - J0 >= SPA_WIN))
        return;
    const int slot = S.map[J - J0];
    if (slot >= SPA_SEGT)
        return;
    const unsigned cmw = cmr[slot];
    const int pos = rs + (int)(cmw >> 16) + __popc((cmw & 0xFFFFu) >> (16 - (col & 15)));
    if (pos < SPA_CAP)
        S.acc[pos] = __dadd_rn(S.acc[pos], __dmul_rn(a, b));
}

// True when a product may meet short B rows in the numeric SPA step -- B's
// rows are short on average, or the mean C tile row is cut into several
// segments (B rows restricted to a segment's columns) -- so that it runs the
// FLAT form of step3_spa_segment.  The other form keeps the per-entry loop
// alone (and its registers).
__host__ __device__ __forceinline__ bool spa_wants_flat(int browB, long long numC, long long nnzC, int tilem)
{
    return browB < SPA_FLAT || numC > (long long)SPA_SEGT * tilem || nnzC > (long long)SPA_CAP * tilem;
}

// Applies ne (<= SPA_STAGE) staged entries A(r, k) of row r -- B row bounds
// bl (cut to the segment) and values a, in k order -- to the row's
// accumulator run.  FLATTEN: when their B rows hold fewer than SPA_FLAT
// entries on average, the products are flattened, 32 per batch in k order;
// lanes of a batch meeting the same slot are folded by the lowest of them in
// lane order and batches follow one another behind warp barriers, so every
// slot still sums its products in k order.  Otherwise (or !FLATTEN) a warp
// pass per entry streams its B row, the next row's first 32 entries
// prefetched.  bl is overwritten.
template <bool FLATTEN>
__device__ __forceinline__ void spa_apply_stage(const ProdView &P, SpaSmem &S, const unsigned *cmr, int rs, int J0,
                                                int J1, bool full, int2 *bl, const double *a, int ne, int lane)
{
    if (FLATTEN)
    {
        const int l0 = lane < ne ? bl[lane].y : 0;
        const int l1 = lane + 32 < ne ? bl[lane + 32].y : 0;
        int i0 = l0, i1 = l1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const int o0 = __shfl_up_sync(TSG_FULL_MASK, i0, d);
            const int o1 = __shfl_up_sync(TSG_FULL_MASK, i1, d);
            if (lane >= d)
            {
                i0 += o0;
                i1 += o1;
            }
        }
        const int h0 = __shfl_sync(TSG_FULL_MASK, i0, 31);
        const int ni = h0 + __shfl_sync(TSG_FULL_MASK, i1, 31);
        if (ni < SPA_FLAT * ne)
        {
            // entry e becomes (its first B index - its first item, its first item)
            if (lane < ne)
                bl[lane] = make_int2(bl[lane].x - (i0 - l0), i0 - l0);
            if (lane + 32 < ne)
                bl[lane + 32] = make_int2(bl[lane + 32].x - (h0 + i1 - l1), h0 + i1 - l1);
            __syncwarp();
            int ent = 0;
            for (int ib = 0; ib < ni; ib += 32)
            {
                const int item = ib + lane;
                int pos = -1 - lane; // distinct keys for lanes without a slot
                double prod = 0.0;
                if (item < ni)
                {
                    while (ent + 1 < ne && bl[ent + 1].y <= item)
                        ent++;
                    const int bi = bl[ent].x + item;
                    const int p = spa_slot(S, cmr, rs, J0, J1, full, P.B_rcol[bi]);
                    if (p >= 0)
                    {
                        pos = p;
                        prod = __dmul_rn(a[ent], P.B_rval[bi]);
                    }
                }
                const unsigned grp = __match_any_sync(TSG_FULL_MASK, pos);
                const bool lead = pos >= 0 && lane == __ffs(grp) - 1;
                const int rounds = __reduce_max_sync(TSG_FULL_MASK, pos >= 0 ? __popc(grp) : 0);
                double acc = lead ? S.acc[pos] : 0.0;
                unsigned gl = grp;
                for (int q = 0; q < rounds; q++)
                {
                    const double v = __shfl_sync(TSG_FULL_MASK, prod, gl ? __ffs(gl) - 1 : lane);
                    if (gl)
                    {
                        acc = __dadd_rn(acc, v);
                        gl &= gl - 1;
                    }
                }
                if (lead)
                    S.acc[pos] = acc;
                __syncwarp();
            }
            return;
        }
    }
    int2 nb = bl[0];
    int c_cur = -1;
    double v_cur = 0.0;
    if (lane < nb.y)
    {
        c_cur = P.B_rcol[nb.x + lane];
        v_cur = P.B_rval[nb.x + lane];
    }
    for (int i = 0; i < ne; i++)
    {
        const int2 cb = nb;
        int c_nxt = -1;
        double v_nxt = 0.0;
        if (i + 1 < ne)
        {
            nb = bl[i + 1];
            if (lane < nb.y)
            {
                c_nxt = P.B_rcol[nb.x + lane];
                v_nxt = P.B_rval[nb.x + lane];
            }
        }
        const double av = a[i];
        if (c_cur >= 0)
            spa_add(S, cmr, rs, J0, J1, full, c_cur, av, v_cur);
        if (cb.y > 32) // B rows longer than a warp
            for (int e = cb.x + 32 + lane; e < cb.x + cb.y; e += 32)
                spa_add(S, cmr, rs, J0, J1, full, P.B_rcol[e], av, P.B_rval[e]);
        __syncwarp();
        c_cur = c_nxt;
        v_cur = v_nxt;
    }
}

// FLAT form of a segment's apply phase, with A's entries staged by the
// whole CTA.  A's tile row I keeps its values contiguous, tile after tile
// in column order, each tile row-major, so every row meets its own entries
// in that order in k order.  The CTA takes them SPA_CO_CHUNK at a time:
// every thread stages entries -- the row from the tile's row offsets, the
// column from the entry's byte, B's row bounds cut to the segment's
// columns -- entries whose B row holds nothing there are dropped and the
// rest are grouped by row, keeping their order; then warp r applies its
// row's staged entries in order (spa_apply_stage).  A row with many A
// entries (R-MAT's hub rows) thus no longer stages them alone -- a binary
// search of B's row per entry -- while the segment's other warps wait.
__device__ __forceinline__ void spa_coop_apply(const ProdView &P, SpaSmem &S, int pa_beg, int pa_end, int J0, int J1,
                                               bool full, int r, int lane, int tid, const unsigned *cmr, int rs)
{
    SpaCoop &C = S.co;
    const bool ptr16 = (reinterpret_cast<unsigned long long>(P.A_Ptr) & 15ULL) == 0;
    const int v_beg = P.A_tnnz[pa_beg], v_end = P.A_tnnz[pa_end];
    for (int c0 = v_beg; c0 < v_end; c0 += SPA_CO_CHUNK)
    {
        const int ne = min(SPA_CO_CHUNK, v_end - c0);
        if (tid == 0)
            C.ptile = a_tile_of(P, pa_beg, pa_end, c0);
        for (int q = tid; q < SPA_CO_SLOTS * TSG_BS; q += SPA_THREADS)
            C.wc[q / TSG_BS][q % TSG_BS] = 0;
        __syncthreads();
        const int p0 = C.ptile;
        const int nt = min(ne, pa_end - p0); // tiles that can hold the chunk's entries
        for (int q = tid; q <= nt; q += SPA_THREADS)
            C.tile0[q] = P.A_tnnz[p0 + q];
        __syncthreads();
        int er[2], eb[2], el[2], ek[2];
        double ea[2];
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const int j = tid + h * SPA_THREADS;
            int row = TSG_BS, b0 = 0, len = 0;
            double av = 0.0;
            if (j < ne)
            {
                const int v = c0 + j;
                int k;
                a_entry(P, C.tile0, nt, p0, ptr16, v, row, k);
                av = P.A_Val[v];
                b0 = P.B_rptr[k];
                int b1 = P.B_rptr[k + 1];
                if (!full)
                {
                    b0 += lower_bound_int(P.B_rcol + b0, b1 - b0, J0 * TSG_BS);
                    b1 = b0 + lower_bound_int(P.B_rcol + b0, b1 - b0, J1 * TSG_BS);
                }
                len = b1 - b0;
                if (len == 0)
                    row = TSG_BS; // adds nothing to this segment
            }
            const unsigned peers = __match_any_sync(TSG_FULL_MASK, row);
            er[h] = row;
            eb[h] = b0;
            el[h] = len;
            ea[h] = av;
            ek[h] = __popc(peers & ((1u << lane) - 1u));
            if (row < TSG_BS && ek[h] == 0)
                C.wc[j >> 5][row] = __popc(peers);
        }
        __syncthreads();
        // warp 0: each row's entries before every slot, and the rows' starts
        if (tid < 32)
        {
            int run = 0;
            if (lane < TSG_BS)
                for (int q = 0; q < SPA_CO_SLOTS; q++)
                {
                    const int t = C.wc[q][lane];
                    C.wc[q][lane] = run;
                    run += t;
                }
            int incl = run;
#pragma unroll
            for (int d = 1; d < TSG_BS; d <<= 1)
            {
                const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
                if (lane >= d)
                    incl += o;
            }
            if (lane < TSG_BS)
                C.rbeg[lane] = incl - run;
            if (lane == TSG_BS - 1)
                C.rbeg[TSG_BS] = incl;
        }
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2; h++)
            if (er[h] < TSG_BS)
            {
                const int j = tid + h * SPA_THREADS;
                const int pos = C.rbeg[er[h]] + C.wc[j >> 5][er[h]] + ek[h];
                C.bl[pos] = make_int2(eb[h], el[h]);
                C.a[pos] = ea[h];
            }
        __syncthreads();
        const int e1 = C.rbeg[r + 1];
        for (int base = C.rbeg[r]; base < e1; base += SPA_STAGE)
            spa_apply_stage<true>(P, S, cmr, rs, J0, J1, full, C.bl + base, C.a + base, min(SPA_STAGE, e1 - base), lane);
        __syncthreads();
    }
}

// The CTA computes C tiles [t0, t1) (one tile row, limits as above).  FLAT:
// a stage of A entries whose B rows (inside the segment) hold fewer than
// SPA_FLAT entries on average has its products flattened -- 32 per batch in
// k order (A's entries in column order, each with its B row); lanes of a
// batch meeting the same slot are folded by the lowest of them in lane
// order, and batches follow one another behind warp barriers, so every slot
// still sums its products in k order.  Short B rows would otherwise leave
// most lanes idle, one A entry at a time.
template <bool FLAT>
__device__ __forceinline__ void step3_spa_segment(const ProdView &P, SpaSmem &S, int t0, int t1)
{
    const int tid = threadIdx.x, lane = tid & 31, r = tid >> 5;
    const int I = P.C_row[t0];
    const int J0 = P.C_col[t0], J1 = P.C_col[t1 - 1] + 1;
    const int base0 = P.C_tnnz[t0], cn = min(P.C_tnnz[t1] - base0, SPA_CAP);
    const int nt = min(t1 - t0, SPA_SEGT);
    const int win = min(J1 - J0, SPA_WIN);
    // a segment holding the whole C tile row meets only its own columns
    const bool full = t0 == P.C_ptr[I] && t1 == P.C_ptr[I + 1] && J1 - J0 <= SPA_WIN;
    __syncthreads();
    for (int q = tid; q < cn; q += SPA_THREADS)
        S.acc[q] = 0.0;
    for (int q = tid; q < win; q += SPA_THREADS)
        S.map[q] = 0xFFFF;
    __syncthreads();
    for (int u = tid; u < nt * TSG_BS; u += SPA_THREADS)
    {
        const int jl = u >> 4, rr = u & 15;
        S.cm[rr * SPA_CMS + jl] = P.C_mask[(long long)(t0 + jl) * TSG_BS + rr];
        if (rr == 0)
        {
            const int w = P.C_col[t0 + jl] - J0;
            if (w < win)
                S.map[w] = (unsigned short)jl;
        }
    }
    __syncthreads();
    // each row accumulates in a private run sorted by column (the entries
    // of one B row then hit nearly consecutive slots: few bank conflicts);
    // warp r: entries of row r in earlier tiles of the segment
    {
        int run = 0;
        for (int s0 = 0; s0 < nt; s0 += 32)
        {
            const int sl = s0 + lane;
            const unsigned m = sl < nt ? S.cm[r * SPA_CMS + sl] : 0u;
            const int c = __popc(m);
            int incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1)
            {
                const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
                if (lane >= d)
                    incl += o;
            }
            if (sl < nt)
                S.cm[r * SPA_CMS + sl] = ((unsigned)(run + incl - c) << 16) | m;
            run += __shfl_sync(TSG_FULL_MASK, incl, 31);
        }
        if (lane == 0)
            S.rstart[r] = run;
    }
    __syncthreads();
    if (tid == 0)
    {
        int acc0 = 0;
        for (int q = 0; q < TSG_BS; q++)
        {
            const int n = S.rstart[q];
            S.rstart[q] = acc0;
            acc0 += n;
        }
    }
    __syncthreads();
    const int rs = S.rstart[r];
    const unsigned *cmr = S.cm + r * SPA_CMS;
    const int pa_beg = P.A_ptr[I], pa_end = P.A_ptr[I + 1];
    if (FLAT)
    {
        spa_coop_apply(P, S, pa_beg, pa_end, J0, J1, full, r, lane, tid, cmr, rs);
    }
    else
    {
        // warp r walks A's row r by itself, 32 A tiles at a time
        SpaStage &G = S.stage[r];
        for (int g = pa_beg; g < pa_end; g += 32)
        {
            const int pa = g + lane;
            unsigned mr = 0;
            int st = 0, kb = 0;
            if (pa < pa_end)
            {
                mr = P.A_mask[(long long)pa * TSG_BS + r];
                st = P.A_tnnz[pa] + P.A_Ptr[(long long)pa * TSG_BS + r];
                kb = P.A_col[pa] * TSG_BS;
            }
            const int cnt = __popc(mr);
            int incl = cnt;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1)
            {
                const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
                if (lane >= d)
                    incl += o;
            }
            const int total = __shfl_sync(TSG_FULL_MASK, incl, 31);
            for (int base = 0; base < total; base += SPA_STAGE)
            {
                __syncwarp();
                // stage A(r, k) entries [base, base + SPA_STAGE) of this group in
                // column order: B row bounds and the A value
                unsigned bits = mr;
                for (int x = 0; x < cnt; x++)
                {
                    const int bit = 31 - __clz(bits);
                    bits ^= 1u << bit;
                    const int e = incl - cnt + x - base;
                    if (e >= 0 && e < SPA_STAGE)
                    {
                        const int k = kb + (15 - bit);
                        int b0 = P.B_rptr[k], b1 = P.B_rptr[k + 1];
                        if (!full)
                        {
                            // only B's entries inside this segment's columns
                            b0 += lower_bound_int(P.B_rcol + b0, b1 - b0, J0 * TSG_BS);
                            b1 = b0 + lower_bound_int(P.B_rcol + b0, b1 - b0, J1 * TSG_BS);
                        }
                        G.bl[e] = make_int2(b0, b1 - b0);
                        G.a[e] = P.A_Val[st + x];
                    }
                }
                __syncwarp();
                spa_apply_stage<false>(P, S, cmr, rs, J0, J1, full, G.bl, G.a, min(SPA_STAGE, total - base), lane);
            }
        }
    }
    __syncthreads();
    // out to C's tiled layout: tile row (jl, rr) starts at the tile's value
    // offset + its row offset; its values are the row's run from its prefix
    for (int u = tid; u < nt * TSG_BS; u += SPA_THREADS)
    {
        const int jl = u >> 4, rr = u & 15;
        const unsigned cmw = S.cm[rr * SPA_CMS + jl];
        unsigned mk = cmw & 0xFFFFu;
        if (!mk)
            continue;
        const long long tt = (long long)(t0 + jl) * TSG_BS + rr;
        int p = P.C_tnnz[t0 + jl] + P.C_Ptr[tt];
        int q = S.rstart[rr] + (int)(cmw >> 16);
        bool over = false;
        while (mk)
        {
            const int bit = 31 - __clz(mk);
            P.C_Colb[p] = (unsigned char)(15 - bit);
            if (q < SPA_CAP)
                P.C_Val[p] = S.acc[q];
            else
                over = true;
            p++;
            q++;
            mk ^= 1u << bit;
        }
        // segments are cut to hold at most SPA_CAP values; a value past the
        // accumulator is reported, not written as a silent zero
        if (over && P.status)
            atomicExch(P.status, TSG_ERR_OVERFLOW);
    }
}

// ---------------------------------------------------------------------------
// Step 2 for wide tile rows (more C tiles or a wider column window than the
// fused row pass holds), through B's row view.  One CTA owns a segment of
// consecutive C tiles of tile row I (at most SP2_SEGT tiles, a SP2_WIN
// tile-column window); warp r walks A's row r and, for every A(r, k), B's
// row k: each entry's column sets its bit in the 32-bit row-r mask word of
// its C tile (shared-memory atomicOr; the order does not matter for an OR).
// The masks then go out through step2_store like every other step-2 path.
// ---------------------------------------------------------------------------
#define SP2_SEGT 1024
#define SP2_MS (SP2_SEGT + 1) // row stride of the [row][tile] mask words (a tile's rows in distinct banks)
#define SP2_WIN 4096

#define SP2_CO_CHUNK 1024 // A entries the CTA stages per pass

struct Spa2Coop
{
    int bs[SP2_CO_CHUNK];          // B row start (cut to the segment) of each staged A entry
    int off[SP2_CO_CHUNK + 1];     // its first item (B entry) in the chunk; off[n] = items
    unsigned char row[SP2_CO_CHUNK];
    int tile0[SP2_CO_CHUNK + 1];   // value offset of each A tile the chunk can touch
    int wsum[SPA_WARPS];
    int ptile;                     // the chunk's first A tile
};

struct Spa2Smem
{
    unsigned m[TSG_BS * SP2_MS]; // [row][tile] mask words
    unsigned short map[SP2_WIN];
    Spa2Coop co;
};

// exclusive prefix of v over the CTA's SPA_THREADS threads (thread order)
// and the total; wsum holds SPA_WARPS ints
__device__ __forceinline__ int block_excl_scan(int v, int *wsum, int *total, int tid, int lane)
{
    int incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
    {
        const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
        if (lane >= d)
            incl += o;
    }
    const int warp = tid >> 5;
    if (lane == 31)
        wsum[warp] = incl;
    __syncthreads();
    int base = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < SPA_WARPS; w++)
    {
        const int x = wsum[w];
        base += w < warp ? x : 0;
        tot += x;
    }
    __syncthreads();
    *total = tot;
    return base + incl - v;
}


// The CTA (SPA_THREADS threads) computes the masks of C tiles [t0, t1).
__device__ __forceinline__ void step2_spa_segment(const ProdView &P, Spa2Smem &S, int t0, int t1, int *s_bins)
{
    const int tid = threadIdx.x, lane = tid & 31, r = tid >> 5;
    const int I = P.C_row[t0];
    const int J0 = P.C_col[t0], J1 = P.C_col[t1 - 1] + 1;
    const int nt = min(t1 - t0, SP2_SEGT);
    const int win = min(J1 - J0, SP2_WIN);
    const bool full = t0 == P.C_ptr[I] && t1 == P.C_ptr[I + 1];
    __syncthreads();
    for (int q = tid; q < nt * TSG_BS; q += SPA_THREADS)
        S.m[(q & 15) * SP2_MS + (q >> 4)] = 0u;
    for (int q = tid; q < win; q += SPA_THREADS)
        S.map[q] = 0xFFFF;
    __syncthreads();
    for (int jl = tid; jl < nt; jl += SPA_THREADS)
    {
        const int w = P.C_col[t0 + jl] - J0;
        if (w < win)
            S.map[w] = (unsigned short)jl;
    }
    __syncthreads();
    // A's entries of the tile row, SP2_CO_CHUNK at a time: every thread
    // stages entries (row, B's row cut to the segment's columns), then the
    // chunk's B entries are split evenly over the warps, each setting its
    // entry's column bit in the row's mask word (an OR: any order)
    Spa2Coop &C = S.co;
    const bool ptr16 = (reinterpret_cast<unsigned long long>(P.A_Ptr) & 15ULL) == 0;
    const int pa_beg = P.A_ptr[I], pa_end = P.A_ptr[I + 1];
    const int v_beg = P.A_tnnz[pa_beg], v_end = P.A_tnnz[pa_end];
    for (int c0 = v_beg; c0 < v_end; c0 += SP2_CO_CHUNK)
    {
        const int ne = min(SP2_CO_CHUNK, v_end - c0);
        if (tid == 0)
            C.ptile = a_tile_of(P, pa_beg, pa_end, c0);
        __syncthreads();
        const int p0 = C.ptile;
        const int ntl = min(ne, pa_end - p0); // tiles that can hold the chunk's entries
        for (int q = tid; q <= ntl; q += SPA_THREADS)
            C.tile0[q] = P.A_tnnz[p0 + q];
        __syncthreads();
        int len[2];
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const int j = tid + h * SPA_THREADS;
            len[h] = 0;
            if (j < ne)
            {
                int row, k;
                a_entry(P, C.tile0, ntl, p0, ptr16, c0 + j, row, k);
                int b0 = P.B_rptr[k], b1 = P.B_rptr[k + 1];
                if (!full)
                {
                    b0 += lower_bound_int(P.B_rcol + b0, b1 - b0, J0 * TSG_BS);
                    b1 = b0 + lower_bound_int(P.B_rcol + b0, b1 - b0, J1 * TSG_BS);
                }
                C.bs[j] = b0;
                C.row[j] = (unsigned char)row;
                len[h] = b1 - b0;
            }
        }
        int tot0, tot1;
        const int x0 = block_excl_scan(len[0], C.wsum, &tot0, tid, lane);
        const int x1 = block_excl_scan(len[1], C.wsum, &tot1, tid, lane);
        if (tid < ne)
            C.off[tid] = x0;
        if (tid + SPA_THREADS < ne)
            C.off[tid + SPA_THREADS] = tot0 + x1;
        if (tid == 0)
            C.off[ne] = tot0 + tot1;
        __syncthreads();
        const int items = tot0 + tot1;
        const int per = (items + SPA_WARPS - 1) / SPA_WARPS;
        const int w0 = r * per, w1 = min(items, w0 + per);
        if (w0 + lane < w1)
        {
            // the entry of this lane's first item: the last entry starting at or before it
            const int first = w0 + lane;
            int lo = 0, hi = ne - 1;
            while (lo < hi)
            {
                const int mid = (lo + hi + 1) >> 1;
                if (C.off[mid] <= first)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            int ent = lo;
            for (int item = first; item < w1; item += 32)
            {
                while (C.off[ent + 1] <= item)
                    ent++;
                const int col = P.B_rcol[C.bs[ent] + (item - C.off[ent])];
                const int J = col >> 4;
                if (J < J0 || J - J0 >= win)
                    continue;
                const int slot = S.map[J - J0];
                if (slot < nt)
                    atomicOr(&S.m[C.row[ent] * SP2_MS + slot], 1u << (15 - (col & 15)));
            }
        }
        __syncthreads();
    }
    __syncthreads();
    // half-warp per C tile: row offsets, masks, tile count, bin
    const unsigned hmask = TSG_HW_MASK(tid);
    for (int jl = tid >> 4; jl < nt; jl += SPA_THREADS / 16)
        step2_store(P, t0 + jl, hmask, tid & 15, S.m[(tid & 15) * SP2_MS + jl], s_bins);
}

// ---------------------------------------------------------------------------
// Hypersparse tile rows.  With very sparse, unstructured operands step 1's
// tile structure of a C tile row holds nearly every tile column while the
// row's scalar products reach only a few of those tiles (n = 65,536 with 8
// entries per row of A and B: ~4,000 C tiles and ~1,000 products per tile
// row).  The SPA segments would spend their time on empty tiles, segment
// after segment, each re-walking A's row.  A wide row whose scalar products
// (counted by the fused step-1/2 pass, wide_kind) are below HYP_RATIO per C
// tile is therefore done whole by one CTA:
//  - step 2 zero-fills the row's masks, row offsets and tile counts with
//    16-byte stores, ORs every product's bit into C's mask word in global
//    memory (two rows' 16-bit masks share a 32-bit word), notes the tiles
//    hit in a shared bitmap and finishes only those tiles, a thread per tile
//    (row offsets, count and bin from its 16 masks);
//  - step 3 zero-fills the row's values and adds every product into its
//    value slot -- the tile's value offset + the row offset + the popcount
//    of the row mask left of the column -- in global memory.  Warp r takes
//    row r's products in generation order (A's entries in column order, each
//    with its B row), 32 at a time; lanes of one batch that meet the same
//    slot are summed by the lowest of them in lane order, and batches follow
//    one another behind warp barriers, so every C entry sums its products in
//    k order, each product rounded before the add, as the reference does.
// The tile column -> tile map covers HYP_WIN tile columns.  Rows are marked
// hypersparse only when their C tiles span less than that (each further
// window would repeat the walk of the row's products); the routines still
// take any row, window by window, each pass adding the products in it.
// ---------------------------------------------------------------------------
#define HYP_WIN 16384
#define HYP_RATIO 4
static_assert(HYP_WIN / 32 <= SPA_THREADS, "one hit-bitmap word per thread");

struct HypStage
{
    int2 bl[SPA_STAGE];      // B row: first entry, length
    int off[SPA_STAGE + 1];  // first product of each staged entry
    double a[SPA_STAGE];     // A value of each staged entry
    double prod[32];         // products of the current batch, by lane
};

struct HypSmem
{
    unsigned short map[HYP_WIN]; // tile column - W0 -> tile - s0 (only C's columns are read);
                                 // step 2 then lists the window's hit tiles here
    unsigned hit[HYP_WIN / 32];  // tiles of the window that received a product (step 2)
    int wsum[SPA_WARPS];
    int win_end;
    HypStage stage[SPA_WARPS];
};

// Exclusive scan of v over the CTA (SPA_THREADS threads); total = the sum.
__device__ __forceinline__ int hyp_cta_scan(int v, int *wsum, int &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
    {
        const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
        if (lane >= d)
            incl += o;
    }
    if (lane == 31)
        wsum[w] = incl;
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int q = 0; q < SPA_WARPS; q++)
    {
        const int x = wsum[q];
        off += q < w ? x : 0;
        tot += x;
    }
    total = tot;
    __syncthreads();
    return off + incl - v;
}

// 2 when the wide A tile row i is hypersparse, else 1: B has a row view,
// the row's C tiles span less than one map window (HYP_WIN tile columns), and
// the row's scalar products -- counted exactly, sum over A's entries of the
// length of B's row -- are below HYP_RATIO per C tile.  The count stops at
// that limit.  Warp-uniform; every lane calls it, after the row's C columns
// are emitted (and visible to the warp).
__device__ __forceinline__ int wide_kind(const ProdView &P, int i, int lane)
{
    if (!P.B_rptr)
        return 1;
    const int rs = P.C_ptr[i], re = P.C_ptr[i + 1];
    if (re == rs || P.C_col[re - 1] - P.C_col[rs] >= HYP_WIN)
        return 1;
    const long long lim = (long long)HYP_RATIO * (re - rs);
    const int a0 = P.A_ptr[i], a1 = P.A_ptr[i + 1];
    long long np = 0;
    for (int g = a0; g < a1; g += 32)
    {
        const int pa = g + lane; // lane per A tile: its entries' B row lengths
        if (pa < a1)
        {
            const int kb = P.A_col[pa] * TSG_BS;
            const int e1 = P.A_tnnz[pa + 1];
            for (int e = P.A_tnnz[pa]; e < e1; e++)
            {
                const int k = kb + (P.A_Colb[e] & 15);
                np += P.B_rptr[k + 1] - P.B_rptr[k];
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1)
            np += __shfl_xor_sync(TSG_FULL_MASK, np, d);
        if (np >= lim)
            return 1;
        np = lane == 0 ? np : 0; // keep the running total in one lane
    }
    return 2;
}

// Warp r enumerates the products of C row 16 I + r: A's entries of the row in
// column order, each with its B row (row view), flattened 32 products at a
// time.  f(valid, e, bi) is called with the whole warp converged; e is the
// staged entry (G.a[e] its A value when VAL), bi the product's index in B's
// row view.  Lane order within a batch, and batch order, follow k.
template <bool VAL, typename F>
__device__ __forceinline__ void hyp_walk(const ProdView &P, HypStage &G, int I, int r, int lane, F f)
{
    const int pa_beg = P.A_ptr[I], pa_end = P.A_ptr[I + 1];
    for (int g = pa_beg; g < pa_end; g += 32)
    {
        const int pa = g + lane;
        unsigned mr = 0;
        int st = 0, kb = 0;
        if (pa < pa_end)
        {
            mr = P.A_mask[(long long)pa * TSG_BS + r];
            if (mr)
            {
                kb = P.A_col[pa] * TSG_BS;
                if (VAL)
                    st = P.A_tnnz[pa] + P.A_Ptr[(long long)pa * TSG_BS + r];
            }
        }
        const int cnt = __popc(mr);
        int incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
            if (lane >= d)
                incl += o;
        }
        const int total = __shfl_sync(TSG_FULL_MASK, incl, 31);
        for (int base = 0; base < total; base += SPA_STAGE)
        {
            __syncwarp();
            unsigned bits = mr;
            for (int x = 0; x < cnt; x++)
            {
                const int bit = 31 - __clz(bits);
                bits ^= 1u << bit;
                const int e = incl - cnt + x - base;
                if (e >= 0 && e < SPA_STAGE)
                {
                    const int k = kb + (15 - bit);
                    const int b0 = P.B_rptr[k];
                    G.bl[e] = make_int2(b0, P.B_rptr[k + 1] - b0);
                    if (VAL)
                        G.a[e] = P.A_Val[st + x];
                }
            }
            __syncwarp();
            const int ne = min(SPA_STAGE, total - base);
            {
                const int l0 = lane < ne ? G.bl[lane].y : 0;
                const int l1 = lane + 32 < ne ? G.bl[lane + 32].y : 0;
                int i0 = l0, i1 = l1;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1)
                {
                    const int o0 = __shfl_up_sync(TSG_FULL_MASK, i0, d);
                    const int o1 = __shfl_up_sync(TSG_FULL_MASK, i1, d);
                    if (lane >= d)
                    {
                        i0 += o0;
                        i1 += o1;
                    }
                }
                const int t0s = __shfl_sync(TSG_FULL_MASK, i0, 31);
                if (lane < ne)
                    G.off[lane] = i0 - l0;
                if (lane + 32 < ne)
                    G.off[lane + 32] = t0s + i1 - l1;
                if (lane == 31)
                    G.off[ne] = t0s + i1;
            }
            __syncwarp();
            const int ni = G.off[ne];
            int ent = 0;
            for (int ib = 0; ib < ni; ib += 32)
            {
                const int item = ib + lane;
                const bool valid = item < ni;
                if (valid)
                    while (G.off[ent + 1] <= item)
                        ent++;
                f(valid, ent, valid ? G.bl[ent].x + (item - G.off[ent]) : 0);
            }
        }
    }
}

// First tile of the window starting at tile s0 of a row ending at re: tiles
// [s0, end) have tile columns below C_col[s0] + HYP_WIN.  Fills the map.
__device__ __forceinline__ int hyp_window(const ProdView &P, HypSmem &S, int s0, int re, int W0)
{
    if (threadIdx.x == 0)
        S.win_end = s0 + lower_bound_int(P.C_col + s0, re - s0, W0 + HYP_WIN);
    __syncthreads();
    const int s1 = S.win_end;
    for (int q = threadIdx.x; q < s1 - s0; q += SPA_THREADS)
        S.map[P.C_col[s0 + q] - W0] = (unsigned short)q;
    __syncthreads();
    return s1;
}

// Step 2 of hypersparse tile row I by the CTA (SPA_THREADS threads).
__device__ __forceinline__ void step2_hyper_row(const ProdView &P, HypSmem &S, int I, int *s_bins)
{
    const int tid = threadIdx.x, lane = tid & 31, r = tid >> 5;
    const int rs = P.C_ptr[I], re = P.C_ptr[I + 1];
    __syncthreads();
    {
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        uint4 *mk = reinterpret_cast<uint4 *>(P.C_mask + (long long)rs * TSG_BS);
        uint4 *pt = reinterpret_cast<uint4 *>(P.C_Ptr + (long long)rs * TSG_BS);
        for (int q = tid; q < 2 * (re - rs); q += SPA_THREADS)
            mk[q] = z;
        for (int q = tid; q < re - rs; q += SPA_THREADS)
        {
            pt[q] = z;
            P.C_tnnz[rs + q] = 0;
        }
    }
    __threadfence_block();
    for (int s0 = rs; s0 < re;)
    {
        __syncthreads();
        const int W0 = P.C_col[s0];
        for (int q = tid; q < HYP_WIN / 32; q += SPA_THREADS)
            S.hit[q] = 0u;
        const int s1 = hyp_window(P, S, s0, re, W0);
        const int nw = s1 - s0;
        hyp_walk<false>(P, S.stage[r], I, r, lane, [&](bool valid, int, int bi) {
            if (!valid)
                return;
            const int col = P.B_rcol[bi];
            const int w = (col >> 4) - W0;
            if (w < 0 || w >= HYP_WIN)
                return; // another window's product
            const int sl = S.map[w];
            if (sl >= nw)
                return;
            const long long t = (long long)s0 + sl;
            unsigned *word = reinterpret_cast<unsigned *>(P.C_mask + t * TSG_BS + (r & ~1));
            atomicOr(word, 1u << ((15 - (col & 15)) + ((r & 1) << 4)));
            const unsigned hb = 1u << (sl & 31);
            if (!(S.hit[sl >> 5] & hb))
                atomicOr(&S.hit[sl >> 5], hb);
        });
        __threadfence_block();
        __syncthreads();
        // list the tiles that received a product (over the map), then a
        // thread per listed tile: its 16 row masks (two 16-byte loads from
        // L2), row offsets, count and bin
        const unsigned hw = tid < ((nw + 31) >> 5) ? S.hit[tid] : 0u;
        int nh;
        int at = hyp_cta_scan(__popc(hw), S.wsum, nh);
        for (unsigned b = hw; b; b &= b - 1)
            S.map[at++] = (unsigned short)(tid * 32 + __ffs(b) - 1);
        __syncthreads();
        for (int j = tid; j < nh; j += SPA_THREADS)
        {
            const long long t = (long long)s0 + S.map[j];
            const uint4 *mp = reinterpret_cast<const uint4 *>(P.C_mask + t * TSG_BS);
            const uint4 m0 = __ldcg(mp), m1 = __ldcg(mp + 1);
            const unsigned w2[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
            unsigned pk[4] = {0u, 0u, 0u, 0u};
            int run = 0;
#pragma unroll
            for (int rr = 0; rr < TSG_BS; rr++)
            {
                pk[rr >> 2] |= (unsigned)run << ((rr & 3) * 8);
                run += __popc((w2[rr >> 1] >> ((rr & 1) * 16)) & 0xFFFFu);
            }
            *reinterpret_cast<uint4 *>(P.C_Ptr + t * TSG_BS) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            P.C_tnnz[t] = run;
            if (s_bins)
                atomicAdd(&s_bins[nnz_bin(run)], 1);
        }
        s0 = s1;
    }
}

// Step 3 of hypersparse tile row I by the CTA.
__device__ __forceinline__ void step3_hyper_row(const ProdView &P, HypSmem &S, int I)
{
    const int tid = threadIdx.x, lane = tid & 31, r = tid >> 5;
    const int rs = P.C_ptr[I], re = P.C_ptr[I + 1];
    __syncthreads();
    {
        const int v1 = P.C_tnnz[re];
        for (int q = P.C_tnnz[rs] + tid; q < v1; q += SPA_THREADS)
            P.C_Val[q] = 0.0;
    }
    __threadfence_block();
    HypStage &G = S.stage[r];
    for (int s0 = rs; s0 < re;)
    {
        __syncthreads();
        const int W0 = P.C_col[s0];
        const int s1 = hyp_window(P, S, s0, re, W0);
        const int nw = s1 - s0;
        hyp_walk<true>(P, G, I, r, lane, [&](bool valid, int e, int bi) {
            int pos = -1 - lane; // distinct keys for lanes without a slot
            double prod = 0.0;
            if (valid)
            {
                const int col = P.B_rcol[bi];
                const int w = (col >> 4) - W0;
                if (w >= 0 && w < HYP_WIN)
                {
                    const int sl = S.map[w];
                    if (sl < nw)
                    {
                        const long long t = (long long)s0 + sl;
                        const unsigned m = P.C_mask[t * TSG_BS + r];
                        const int cc = col & 15;
                        if ((m >> (15 - cc)) & 1u)
                        {
                            pos = P.C_tnnz[t] + P.C_Ptr[t * TSG_BS + r] + __popc(m >> (16 - cc));
                            prod = __dmul_rn(G.a[e], P.B_rval[bi]);
                            P.C_Colb[pos] = (unsigned char)cc;
                        }
                    }
                }
            }
            const unsigned grp = __match_any_sync(TSG_FULL_MASK, pos);
            G.prod[lane] = prod;
            __syncwarp();
            if (pos >= 0 && lane == __ffs(grp) - 1)
            {
                double acc = __ldcg(P.C_Val + pos);
                unsigned gl = grp;
                while (gl)
                {
                    const int l = __ffs(gl) - 1;
                    gl &= gl - 1;
                    acc = __dadd_rn(acc, G.prod[l]);
                }
                P.C_Val[pos] = acc;
            }
            __syncwarp();
        });
        s0 = s1;
    }
}

// ---------------------------------------------------------------------------
// Work item of the SPA steps: a block of SPA_BLK consecutive C tiles (global
// tile order).  Ownership: a row of at most SPA_BLK tiles belongs, whole, to
// the block holding its first tile; a longer row is cut into SPA_BLK-tile
// chunks from its start, each belonging to the block holding the chunk's
// first tile.  So every tile is done once, short rows are never cut, and a
// long row is spread over many blocks (and CTAs).  The CTA cuts each piece
// further into segments within the SPA limits.  A hypersparse row belongs
// whole to the block holding its first tile.
#define SPA_BLK 256
// the numeric step's block for products whose C tiles average at least
// SPA_BLK_NARROW_VALUES values (wide rows of skewed products such as R-MAT):
// twice the blocks, so a hub row's segments spread over more CTAs
#define SPA_BLK_NARROW 128
#define SPA_BLK_NARROW_VALUES 4

// calls piece(I, t0, t1) for the pieces [t0, t1) owned by block [tb, te),
// rows longer than CH tiles being cut into CH-tile chunks.  [tb, te) may be a
// block clamped to a range of whole tile rows: it then yields the block's
// pieces of those rows only.
template <int CH, typename F>
__device__ __forceinline__ void spa_block_pieces(const ProdView &P, int tb, int te, F piece)
{
    int t = tb;
    {
        const int I = P.C_row[tb];
        const int rs = P.C_ptr[I], re = P.C_ptr[I + 1];
        if (rs < tb)
        {
            if (re - rs > CH)
                for (int cs = rs + ((tb - rs + CH - 1) / CH) * CH; cs < te && cs < re; cs += CH)
                    piece(I, cs, min(cs + CH, re));
            t = re;
        }
    }
    while (t < te)
    {
        const int I = P.C_row[t];
        const int re = P.C_ptr[I + 1];
        if (re - t <= CH)
            piece(I, t, re);
        else
            for (int cs = t; cs < te && cs < re; cs += CH)
                piece(I, cs, min(cs + CH, re));
        t = re;
    }
}

// A block lying inside a hypersparse row (kind[I] == 2) that an earlier block
// owns has no work, nor have the row's following blocks before the one
// holding the row's end: the claiming thread raises the block counter ctr
// (blocks of this product numbered from base) past them.
template <int BLK = SPA_BLK>
__device__ __forceinline__ void spa_skip_hyper(const ProdView &P, const int *__restrict__ kind, int tb,
                                               unsigned *ctr, long long base)
{
    if (!kind)
        return;
    const int I = P.C_row[tb];
    if (kind[I] != 2 || P.C_ptr[I] >= tb)
        return;
    const long long next = base + P.C_ptr[I + 1] / BLK;
    if (next > base + tb / BLK + 1)
        atomicMax(ctr, (unsigned)next);
}

// Hypersparse rows (kind[I] == 2, kind may be null) are done whole by the
// block owning their first tile.
static_assert(sizeof(HypSmem) <= sizeof(SpaSmem) && sizeof(HypSmem) <= sizeof(Spa2Smem), "hyper scratch");

// only (may be null): only the tile rows I with only[I] != 0 (the rows the
// staged numeric step left).
template <bool FLAT, int BLK = SPA_BLK>
__device__ __forceinline__ void step3_spa_block(const ProdView &P, SpaSmem &S, int tb, int te,
                                                const int *__restrict__ kind, const int *__restrict__ only = nullptr)
{
    spa_block_pieces<BLK>(P, tb, te, [&](int I, int ps, int pe) {
        if (only && !only[I])
            return;
        if (kind && kind[I] == 2)
        {
            if (ps == P.C_ptr[I])
                step3_hyper_row(P, reinterpret_cast<HypSmem &>(S), I);
            return;
        }
        for (int t0 = ps; t0 < pe;)
        {
            const int cand = t0 + 1 + (int)threadIdx.x;
            const bool ok = threadIdx.x < SPA_SEGT && cand <= pe && P.C_tnnz[cand] - P.C_tnnz[t0] <= SPA_CAP &&
                            P.C_col[cand - 1] - P.C_col[t0] < SPA_WIN;
            const int n = __syncthreads_count(ok);
            const int t1 = t0 + (n > 0 ? n : 1);
            step3_spa_segment<FLAT>(P, S, t0, t1);
            t0 = t1;
        }
    });
}

// Symbolic counterpart, for the pieces of wide rows only (wide[I] != 0;
// 2 marks a hypersparse row).  Long rows go in chunks of SP2_SEGT tiles, one
// segment's worth: each segment walks A's whole row, so shorter chunks would
// repeat that walk.
__device__ __forceinline__ void step2_spa_block(const ProdView &P, Spa2Smem &S, int tb, int te,
                                                const int *__restrict__ wide, int *s_bins)
{
    spa_block_pieces<SP2_SEGT>(P, tb, te, [&](int I, int ps, int pe) {
        const int kind = wide[I];
        if (!kind)
            return;
        if (kind == 2)
        {
            if (ps == P.C_ptr[I])
                step2_hyper_row(P, reinterpret_cast<HypSmem &>(S), I, s_bins);
            return;
        }
        for (int t0 = ps; t0 < pe;)
        {
            const int cand = t0 + 1 + (int)threadIdx.x;
            const bool ok = threadIdx.x < SP2_SEGT && cand <= pe && P.C_col[cand - 1] - P.C_col[t0] < SP2_WIN;
            const int n = __syncthreads_count(ok);
            const int t1 = t0 + (n > 0 ? n : 1);
            step2_spa_segment(P, S, t0, t1, s_bins);
            t0 = t1;
        }
    });
}

// ---------------------------------------------------------------------------
// Element schedule for step 3: one warp per C tile, lane = one nonzero
// (r, c) of the tile (from step 2's masks), for chunks of 32 nonzeros.  For
// every matched tile pair (A tile (i,k), B tile (k,j)), the A columns that
// meet B rows with an entry in column c are maskA[r] & maskT_B[c]; each such
// ca contributes A(r,ca) * B(ca,c), both fetched by popcount rank.  The
// accumulator lives in a register, the order is k ascending then ca
// ascending -- the oracle's order for row-sorted inputs -- and the results
// are stored with coalesced writes.  The matched pairs are found once per
// tile (half-warp intersection, identical in both halves) and cached in
// shared memory for the chunks of dense tiles.
// ---------------------------------------------------------------------------
#define S3E_PAIRS 96

__device__ __forceinline__ double elem_pair(const ProdView &P, int posA, int posB, int r, int c, double acc)
{
    const unsigned ma = P.A_mask[(long long)posA * TSG_BS + r];
    unsigned tb = ma & P.B_maskT[(long long)posB * TSG_BS + c];
    if (tb)
    {
        const double *av = P.A_Val + P.A_tnnz[posA] + P.A_Ptr[(long long)posA * TSG_BS + r];
        const double *bv = P.B_Val + P.B_tnnz[posB];
        const unsigned short *bm = P.B_mask + (long long)posB * TSG_BS;
        const unsigned char *bp = P.B_Ptr + (long long)posB * TSG_BS;
        do
        {
            const int bit = 31 - __clz(tb); // bit 15-ca: highest first = ca ascending
            const int ca = 15 - bit;
            const double a = av[__popc(ma >> (bit + 1))];
            const double b = bv[bp[ca] + __popc((unsigned)bm[ca] >> (16 - c))];
            acc = __dadd_rn(acc, __dmul_rn(a, b));
            tb ^= 1u << bit;
        } while (tb);
    }
    return acc;
}

// warp per C tile t; s_pairs: S3E_PAIRS int2 of this warp
__device__ __forceinline__ void step3_elems_tile(const ProdView &P, int t, int2 *s_pairs)
{
    const int lane = threadIdx.x & 31, l16 = lane & 15;
    const unsigned hmask = TSG_HW_MASK(threadIdx.x);
    const int cb = P.C_tnnz[t], cn = P.C_tnnz[t + 1] - cb;
    if (cn == 0)
        return;
    const int i = P.C_row[t], j = P.C_col[t];
    const int abase = P.A_ptr[i], la = P.A_ptr[i + 1] - abase;
    const int bbase = P.B_cptr[j], lb = P.B_cptr[j + 1] - bbase;
    int np = 0;
    intersect_tiles(hmask, l16, P.A_col, abase, la, P.B_crow, P.B_cpos, bbase, lb, [&](int posA, int posB) {
        if (np < S3E_PAIRS && lane == 0)
            s_pairs[np] = make_int2(posA, posB);
        np++;
    });
    __syncwarp();
    const int excl = P.C_Ptr[(long long)t * TSG_BS + l16];
    const unsigned mrev = __brev((unsigned)P.C_mask[(long long)t * TSG_BS + l16]) >> 16;
    for (int e0 = 0; e0 < cn; e0 += 32)
    {
        const int e = e0 + lane;
        int r = 0;
#pragma unroll
        for (int s = 8; s >= 1; s >>= 1)
        {
            const int v = __shfl_sync(TSG_FULL_MASK, excl, r + s, 16);
            if (v <= e)
                r += s;
        }
        const unsigned mr = __shfl_sync(TSG_FULL_MASK, mrev, r, 16);
        const int rank = e - __shfl_sync(TSG_FULL_MASK, excl, r, 16);
        const bool valid = e < cn;
        const int c = valid ? ((int)__fns(mr, 0, rank + 1) & 15) : 0;
        double acc = 0.0;
        if (np <= S3E_PAIRS)
        {
            for (int q = 0; q < np; q++)
            {
                const int2 pr = s_pairs[q];
                if (valid)
                    acc = elem_pair(P, pr.x, pr.y, r, c, acc);
            }
        }
        else
        {
            intersect_tiles(hmask, l16, P.A_col, abase, la, P.B_crow, P.B_cpos, bbase, lb, [&](int posA, int posB) {
                if (valid)
                    acc = elem_pair(P, posA, posB, r, c, acc);
            });
        }
        if (valid)
        {
            P.C_Colb[cb + e] = (unsigned char)c;
            P.C_Val[cb + e] = acc;
        }
    }
    __syncwarp();
}

// Supported (W, CAP) pairs of the row schedule; the dispatch macro expands
// X(W, CAP) for each.
#define TSG_ROW_CONFIGS(X) X(8, 256) X(8, 512) X(8, 1024) X(16, 512) X(16, 1024) X(16, 2048) X(32, 1024) X(32, 2048)
