// Numeric step (step 3) with its operands staged in shared memory by TMA
// bulk copies -- the SPA schedule's step 3 for products whose B rows are not
// short (spa_wants_flat false), e.g. stencils and banded-by-stencil mixes.
//
// Restates the numeric step of the reference's tilespgemm()
// (src/tilespgemm-cuda.h:1505-2608, driver :3006-3118) as a row Gustavson
// over B's row view; the arithmetic order is the reference CPU oracle's
// (src/spgemm-cpu.h:330): every C entry is 0.0 + p1 + p2 + ... over k
// ascending, multiply and add rounded separately.
//
// A persistent CTA holds STG_CONS consumer warps and a producer warp for
// each of its two stages.  A producer claims C tile rows from a device
// counter.  For its next tile row it reads the row bounds, A's tile masks
// and B's row pointers and lays the stage out while the consumers work; as
// soon as its stage is released it fills it with everything that tile row's
// numeric step reads, by
// cp.async.bulk (global -> shared, no multicast) completing on the stage's
// mbarrier:
//   * A's tile row: row masks, row offsets, tile value offsets, tile
//     columns and values;
//   * C's tile row: row masks, row offsets, value offsets, tile columns;
//   * for every A tile (I, K): the rows 16 K + c of B's row view for the
//     columns c its entries use -- consecutive rows, so one contiguous run
//     of column indices and one of values -- and those rows' pointers.
// Consumer warp r owns C row 16 I + r and reads only shared memory.
//
// The tile row goes in segments (one for every tile row of a 3-D 27-point
// stencil).  Row r accumulates in a private column-sorted run (the SPA
// segment's layout), a product's slot found by one word load and a
// popcount; a segment holding the whole tile row first replaces every
// staged B column index by its key (tile, column).  Idle lanes add into a
// sink slot instead of branching, the next A entry's slots and products are
// computed before the current entry's read-modify-write, and a warp barrier
// between A entries keeps each C entry's sum in k order.  The values, laid
// out in C's order, and the column bytes leave by bulk stores (shared ->
// global) that overlap the next segment's set-up.
//
// A tile row whose stage would not fit STG_BYTES (or that the fused step
// 1/2 pass marked hypersparse) is flagged in `left` and done afterwards by
// the SPA kernel (k_step3_rest).  Every wait on an mbarrier is bounded
// (STG_WAIT_NS of %globaltimer); a wait that runs out records
// TSG_ERR_TIMEOUT in *status, the consumer warps agree on it at a named
// barrier, and every warp returns.
#pragma once

#include <stddef.h>

#include "tsg_device.cuh"

#define STG_CONS 16                       // consumer warps, one per row of a tile row
#define STG_THREADS ((STG_CONS + 2) * 32) // + a producer warp per stage
#define STG_CONS_THREADS (STG_CONS * 32)
#define STG_BYTES (68 * 1024)     // one stage
#define STG_WAIT_NS 2000000000ULL // bound of every mbarrier wait
#define STG_SUSPEND_NS 20000u     // sleep hint of one test of a phase
#define STG_RPB 24                // ints of an A tile's row-pointer block (17 pointers rounded out to 16 bytes)
#define STG_STAGE 32              // A entries a warp stages per pass
#define STG_CAP 3072              // C values of a segment

static_assert(STG_CONS == TSG_BS, "one consumer warp per row of a tile row");

// Where tile row I's arrays sit in its stage (byte offsets), and the global
// element index each staged int / double array starts at (copies begin on
// 16-byte boundaries, so a staged array may start a few elements early).
struct StgHdr
{
    int I;    // tile row; -1: no more tile rows
    int skip; // 1: left to the SPA kernel
    int nA, nC;
    int at0, ac0, av0, ct0, cc0; // first staged global index of A_tnnz, A_col, A_Val, C_tnnz, C_col
    int a0, c0;                  // first A tile, first C tile of the tile row
    int nb;                      // staged B entries (runs rounded out to 16-byte blocks)
    int oAm, oAP, oAt, oAc, oAv, oCm, oCP, oCt, oCc, oRp, oTb, oBv, oBc;
};

// a staged A entry of a warp's row: its B row (stage index, length) and its
// value, read in one 16-byte load
struct __align__(16) StgEnt
{
    int b0;                   // first staged entry of the B row
    unsigned short len, last; // its length, and max(length - 1, 0)
    double a;
};

struct StgSmem
{
    unsigned char stage[2][STG_BYTES];
    double acc[STG_CAP + 2];             // a segment's rows' runs, then the sink (and 16-byte padding)
    double outbuf[STG_CAP + 2];          // the segment's C values in C's order at their 16-byte phase
    unsigned cm[TSG_BS][SPA_SEGT + 1];   // per row and tile: (row's entries in earlier tiles << 16) | row mask
                                         // (rows padded by a word: a tile's 16 rows in 16 banks)
    unsigned char colbuf[STG_CAP + 16];  // the segment's C column bytes at their 16-byte phase
    int rtot[TSG_BS];                    // entries of each row in the segment
    int rbase[TSG_BS];                   // first slot of each row's run
    StgEnt ent[STG_CONS][STG_STAGE + 3]; // per warp: staged A entries; three empty entries after the last
    unsigned short map[SPA_WIN];         // tile column - J0 -> tile of the segment
    StgHdr hdr[2];
    unsigned long long full[2], empty[2];
};

static_assert(sizeof(StgSmem) <= 227 * 1024, "staged step 3 exceeds a CTA's shared memory");
static_assert(offsetof(StgSmem, outbuf) % 16 == 0 && offsetof(StgSmem, colbuf) % 16 == 0 &&
                  offsetof(StgSmem, stage) % 16 == 0 && STG_BYTES % 16 == 0,
              "bulk copies need 16-byte aligned shared memory");

// ---------------------------------------------------------------------------
// mbarrier / bulk-copy primitives (PTX)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned stg_sa(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void stg_bar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(stg_sa(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void stg_bar_arrive(unsigned long long *bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(stg_sa(bar)) : "memory");
}

__device__ __forceinline__ void stg_bar_arrive_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                     stg_sa(bar)),
                 "r"(bytes)
                 : "memory");
}

// one test of the phase; the thread may sleep up to STG_SUSPEND_NS in it
// (woken when the phase completes), so idle warps do not spin
__device__ __forceinline__ bool stg_bar_try(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, "
                 "0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(stg_sa(bar)), "r"(parity), "r"(STG_SUSPEND_NS)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long stg_clock_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase of the given parity to complete, at most STG_WAIT_NS;
// false (and TSG_ERR_TIMEOUT in *status) when the bound ran out.
__device__ __forceinline__ bool stg_bar_wait(unsigned long long *bar, unsigned parity, int *status)
{
    if (stg_bar_try(bar, parity))
        return true;
    const unsigned long long t0 = stg_clock_ns();
    while (!stg_bar_try(bar, parity))
        if (stg_clock_ns() - t0 > STG_WAIT_NS)
        {
            atomicExch(status, TSG_ERR_TIMEOUT);
            return false;
        }
    return true;
}

// global -> shared bulk copy of `bytes` (a multiple of 16; both addresses
// 16-byte aligned), completing on bar
__device__ __forceinline__ void stg_bulk(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     stg_sa(dst)),
                 "l"(src), "r"(bytes), "r"(stg_sa(bar))
                 : "memory");
}

// consumer warps only (named barrier 1)
__device__ __forceinline__ void stg_cons_sync()
{
    asm volatile("bar.sync 1, %0;" ::"r"(STG_CONS_THREADS) : "memory");
}

__device__ __forceinline__ int stg_cons_count(bool pred)
{
    int n;
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, 0;\n\tbarrier.red.popc.u32 %0, 1, %2, p;\n\t}"
                 : "=r"(n)
                 : "r"((unsigned)pred), "r"(STG_CONS_THREADS)
                 : "memory");
    return n;
}

__device__ __forceinline__ int stg_down4(int x)
{
    return x & ~3;
}
__device__ __forceinline__ int stg_up4(int x)
{
    return (x + 3) & ~3;
}

// ---------------------------------------------------------------------------
// Producer.  stg_plan reads a tile row's bounds and its A tiles' B runs and
// lays its stage out (every lane holds the plan; lane a also the B run of A
// tile a of the first 32); stg_issue writes the stage's header and table,
// announces the copies' byte total on the stage's full barrier and issues
// the copies.  Global arrays are read up to 15 bytes past their last element
// when a copy's end is rounded up: the library pads every allocation by 16
// bytes.
// ---------------------------------------------------------------------------
// The B rows of one A tile: rows [k0, k1) = 16 K + c for the columns c its
// entries use, one run [e0, e1) of B's row view.
struct StgBrun
{
    int k0, k1, e0, e1;
};

__device__ __forceinline__ StgBrun stg_brun(const ProdView &P, int a)
{
    const uint4 *mp = reinterpret_cast<const uint4 *>(P.A_mask + (long long)a * TSG_BS);
    const uint4 m0 = mp[0], m1 = mp[1];
    unsigned o = m0.x | m0.y | m0.z | m0.w | m1.x | m1.y | m1.z | m1.w;
    o = (o | (o >> 16)) & 0xFFFFu; // bit 15 - c: column c used by some row
    const int kb = P.A_col[a] * TSG_BS;
    StgBrun b;
    b.k0 = kb + (o ? __clz(o) - 16 : 0); // a tile holds at least one entry
    b.k1 = kb + (o ? 17 - __ffs(o) : 0);
    b.e0 = P.B_rptr[b.k0];
    b.e1 = P.B_rptr[b.k1];
    return b;
}

// stage sizes of an A tile's B rows: the run (elements, whole 16-byte blocks
// of column indices), its values copy (elements), its row pointers (ints)
__device__ __forceinline__ int stg_bsize(const StgBrun &b)
{
    return stg_up4(b.e1) - stg_down4(b.e0);
}
__device__ __forceinline__ int stg_vsize(const StgBrun &b)
{
    return ((b.e1 + 1) & ~1) - (b.e0 & ~1);
}
__device__ __forceinline__ int stg_rsize(const StgBrun &b)
{
    return stg_up4(b.k1 + 1) - stg_down4(b.k0);
}

struct StgPlan
{
    int I; // >= the range's end: no more tile rows
    int a0, a1, c0, c1, v0, v1;
    bool fits;
    long long nb, btx;       // staged B entries; bytes of the B runs' and row pointers' copies
    long long oTb, oBv, oBc; // the regions after the fixed ones
    StgBrun mine;            // this lane's A tile among the first 32
};

// fixed regions, in order: A masks, A row offsets, A tile value offsets,
// A tile columns, A values, C masks, C row offsets, C value offsets, C tile
// columns (all copied: [0, oRp)), then the B row-pointer blocks at oRp
struct StgFixed
{
    long long oAm, oAP, oAt, oAc, oAv, oCm, oCP, oCt, oCc, oRp;
};

__device__ __forceinline__ StgFixed stg_fixed(const StgPlan &L)
{
    const int nA = L.a1 - L.a0, nC = L.c1 - L.c0;
    StgFixed F;
    F.oAm = 0;
    F.oAP = F.oAm + 32LL * nA;
    F.oAt = F.oAP + 16LL * nA;
    F.oAc = F.oAt + 4LL * (stg_up4(L.a1 + 1) - stg_down4(L.a0));
    F.oAv = F.oAc + 4LL * (stg_up4(L.a1) - stg_down4(L.a0));
    F.oCm = F.oAv + 8LL * (((L.v1 + 1) & ~1) - (L.v0 & ~1));
    F.oCP = F.oCm + 32LL * nC;
    F.oCt = F.oCP + 16LL * nC;
    F.oCc = F.oCt + 4LL * (stg_up4(L.c1 + 1) - stg_down4(L.c0));
    F.oRp = F.oCc + 4LL * (stg_up4(L.c1) - stg_down4(L.c0));
    return F;
}

__device__ StgPlan stg_plan(const ProdView &P, int I, int r_end, const int *__restrict__ kind, int lane)
{
    StgPlan L;
    L.I = I;
    L.fits = false;
    L.a0 = L.a1 = L.c0 = L.c1 = L.v0 = L.v1 = 0;
    L.nb = L.btx = L.oTb = L.oBv = L.oBc = 0;
    L.mine = {0, 0, 0, 0};
    if (I >= r_end)
        return L;
    // the tile row's bounds, a lane per load
    int x = 0;
    if (lane < 2)
        x = P.A_ptr[I + lane];
    else if (lane < 4)
        x = P.C_ptr[I + lane - 2];
    else if (lane == 4 && kind)
        x = kind[I];
    L.a0 = __shfl_sync(TSG_FULL_MASK, x, 0);
    L.a1 = __shfl_sync(TSG_FULL_MASK, x, 1);
    L.c0 = __shfl_sync(TSG_FULL_MASK, x, 2);
    L.c1 = __shfl_sync(TSG_FULL_MASK, x, 3);
    const bool hyper = __shfl_sync(TSG_FULL_MASK, x, 4) == 2;
    int y = 0;
    if (lane < 2)
        y = P.A_tnnz[lane == 0 ? L.a0 : L.a1];
    L.v0 = __shfl_sync(TSG_FULL_MASK, y, 0);
    L.v1 = __shfl_sync(TSG_FULL_MASK, y, 1);
    const int nA = L.a1 - L.a0;
    const StgFixed F = stg_fixed(L);
    L.oTb = F.oRp + 4LL * STG_RPB * nA;
    const long long off = L.oTb + ((8LL * nA + 15) & ~15LL);
    // B runs: region of A tile a = [start_a, start_a + bsize) elements,
    // start_a a multiple of 4; entry e of its rows at e + start_a - down4(e0)
    bool fits = !hyper && off <= STG_BYTES;
    for (int g = 0; g < nA && fits; g += 32)
    {
        const int a = g + lane;
        int sz = 0, vb = 0, rb = 0;
        if (a < nA)
        {
            const StgBrun b = stg_brun(P, L.a0 + a);
            if (g == 0)
                L.mine = b;
            sz = stg_bsize(b);
            vb = stg_vsize(b);
            rb = stg_rsize(b);
        }
        const int tsz = __reduce_add_sync(TSG_FULL_MASK, sz);
        L.nb += tsz;
        L.btx += 4LL * tsz + 8LL * __reduce_add_sync(TSG_FULL_MASK, vb) + 4LL * __reduce_add_sync(TSG_FULL_MASK, rb);
        fits = off + 12LL * L.nb <= STG_BYTES;
    }
    L.fits = fits;
    L.oBv = off;
    L.oBc = off + 8LL * L.nb;
    return L;
}

__device__ void stg_issue(const ProdView &P, StgSmem &S, int s, const StgPlan &L, int *__restrict__ left, int lane)
{
    StgHdr &H = S.hdr[s];
    unsigned char *st = S.stage[s];
    if (!L.fits)
    {
        if (lane == 0)
        {
            H.I = L.I;
            H.skip = 1;
            left[L.I] = 1;
            atomicAdd(&left[P.tilemA], 1);
        }
        __syncwarp();
        stg_bar_arrive(&S.full[s]);
        return;
    }
    const int nA = L.a1 - L.a0;
    const StgFixed F = stg_fixed(L);
    if (lane == 0)
    {
        H.I = L.I;
        H.skip = 0;
        H.nA = nA;
        H.nC = L.c1 - L.c0;
        H.a0 = L.a0;
        H.c0 = L.c0;
        H.nb = (int)L.nb;
        H.at0 = stg_down4(L.a0);
        H.ac0 = stg_down4(L.a0);
        H.av0 = L.v0 & ~1;
        H.ct0 = stg_down4(L.c0);
        H.cc0 = stg_down4(L.c0);
        H.oAm = (int)F.oAm;
        H.oAP = (int)F.oAP;
        H.oAt = (int)F.oAt;
        H.oAc = (int)F.oAc;
        H.oAv = (int)F.oAv;
        H.oCm = (int)F.oCm;
        H.oCP = (int)F.oCP;
        H.oCt = (int)F.oCt;
        H.oCc = (int)F.oCc;
        H.oRp = (int)F.oRp;
        H.oTb = (int)L.oTb;
        H.oBv = (int)L.oBv;
        H.oBc = (int)L.oBc;
        // bytes the copies below deliver (the A tiles' table is written here)
        stg_bar_arrive_tx(&S.full[s], (unsigned)(F.oRp + L.btx));
    }
    __syncwarp();
    // fixed regions, a lane per copy
    {
        const void *src = nullptr;
        long long o = 0, n = 0;
        switch (lane)
        {
        case 0: src = P.A_mask + (long long)L.a0 * TSG_BS; o = F.oAm; n = F.oAP - F.oAm; break;
        case 1: src = P.A_Ptr + (long long)L.a0 * TSG_BS; o = F.oAP; n = F.oAt - F.oAP; break;
        case 2: src = P.A_tnnz + stg_down4(L.a0); o = F.oAt; n = F.oAc - F.oAt; break;
        case 3: src = P.A_col + stg_down4(L.a0); o = F.oAc; n = F.oAv - F.oAc; break;
        case 4: src = P.A_Val + (L.v0 & ~1); o = F.oAv; n = F.oCm - F.oAv; break;
        case 5: src = P.C_mask + (long long)L.c0 * TSG_BS; o = F.oCm; n = F.oCP - F.oCm; break;
        case 6: src = P.C_Ptr + (long long)L.c0 * TSG_BS; o = F.oCP; n = F.oCt - F.oCP; break;
        case 7: src = P.C_tnnz + stg_down4(L.c0); o = F.oCt; n = F.oCc - F.oCt; break;
        case 8: src = P.C_col + stg_down4(L.c0); o = F.oCc; n = F.oRp - F.oCc; break;
        default: break;
        }
        if (n > 0)
            stg_bulk(st + o, src, (unsigned)n, &S.full[s]);
    }
    // per A tile: its row pointers, B run and table entry, a lane per A tile
    int2 *tb = reinterpret_cast<int2 *>(st + L.oTb);
    long long start = 0;
    for (int g = 0; g < nA; g += 32)
    {
        const int a = g + lane;
        int sz = 0;
        StgBrun b = L.mine;
        if (a < nA)
        {
            if (g > 0)
                b = stg_brun(P, L.a0 + a);
            sz = stg_bsize(b);
        }
        int incl = sz;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const int o = __shfl_up_sync(TSG_FULL_MASK, incl, d);
            if (lane >= d)
                incl += o;
        }
        if (a < nA)
        {
            const int my = (int)start + incl - sz; // the tile's region start (a multiple of 4)
            // B row k of the tile starts at stage index blk[k - down4(k0)] + delta
            tb[a] = make_int2(stg_down4(b.k0), my - stg_down4(b.e0));
            stg_bulk(st + F.oRp + 4LL * STG_RPB * a, P.B_rptr + stg_down4(b.k0), 4u * stg_rsize(b), &S.full[s]);
            if (sz > 0)
                stg_bulk(st + L.oBc + 4LL * my, P.B_rcol + stg_down4(b.e0), 4u * sz, &S.full[s]);
            const int vb = stg_vsize(b);
            if (vb > 0)
                stg_bulk(st + L.oBv + 8LL * (my + (b.e0 & ~1) - stg_down4(b.e0)), P.B_rval + (b.e0 & ~1), 8u * vb,
                         &S.full[s]);
        }
        start += __shfl_sync(TSG_FULL_MASK, incl, 31);
    }
    __syncwarp();
    if (lane != 0)
        stg_bar_arrive(&S.full[s]);
}

// ---------------------------------------------------------------------------
// Consumers
// ---------------------------------------------------------------------------
// Staged tile row, as pointers into its stage.
struct StgView
{
    const unsigned short *Am, *Cm;
    const unsigned char *AP, *CP;
    const int *At, *Ac, *Ct, *Cc; // indexed by the tile's position in the tile row
    const double *Av;             // indexed by global value index - av0
    const int *rp;                // [A tile][STG_RPB]: B's row pointers of the tile's rows
    const int2 *tb;               // [A tile]: (first staged row pointer's row, stage index - B entry index)
    int *Bc;                      // B's column indices (keys after a whole-row segment's conversion)
    const double *Bv;
    int nA, nC, nB, av0;
};

__device__ __forceinline__ StgView stg_view(StgSmem &S, int s)
{
    const StgHdr &H = S.hdr[s];
    unsigned char *st = S.stage[s];
    StgView V;
    V.Am = reinterpret_cast<const unsigned short *>(st + H.oAm);
    V.AP = st + H.oAP;
    V.At = reinterpret_cast<const int *>(st + H.oAt) + (H.a0 - H.at0);
    V.Ac = reinterpret_cast<const int *>(st + H.oAc) + (H.a0 - H.ac0);
    V.Av = reinterpret_cast<const double *>(st + H.oAv);
    V.Cm = reinterpret_cast<const unsigned short *>(st + H.oCm);
    V.CP = st + H.oCP;
    V.Ct = reinterpret_cast<const int *>(st + H.oCt) + (H.c0 - H.ct0);
    V.Cc = reinterpret_cast<const int *>(st + H.oCc) + (H.c0 - H.cc0);
    V.rp = reinterpret_cast<const int *>(st + H.oRp);
    V.tb = reinterpret_cast<const int2 *>(st + H.oTb);
    V.Bc = reinterpret_cast<int *>(st + H.oBc);
    V.Bv = reinterpret_cast<const double *>(st + H.oBv);
    V.nA = H.nA;
    V.nC = H.nC;
    V.nB = H.nb;
    V.av0 = H.av0;
    return V;
}

// The ne staged A entries of warp r in order, as a four-stage pipeline so
// that no chain of shared loads lies inside one iteration: iteration j
// loads staged entry j + 3 (A), reads B's column and value for entry j + 2
// (B), loads the row word of entry j + 1's tile and forms its product (C),
// and adds entry j's product into its slot (D) -- the only dependence left
// inside an iteration is that read-modify-write, and a warp barrier between
// iterations keeps each slot's sum in k order.  Every lane reads a staged
// B entry of its entry's row (its own, or the row's first when idle); idle
// lanes add into the sink slot STG_CAP, so the loop has no branch but its
// own.  The three staged entries after the last are empty.  LONG: some
// staged B row has more than 32 entries (lanes loop over the rest of it).
struct StgB // stage B result
{
    int x;    // B column index, or key
    double v; // B value
    double a; // A value
    bool ok;  // the lane holds an entry
};
struct StgC // stage C result
{
    unsigned w; // the row's word of the entry's tile
    double p;   // product
};

__device__ __forceinline__ StgB stg_stage_b(const StgView &V, const StgEnt &E, int lane)
{
    const int e = E.b0 + min(lane, (int)E.last);
    StgB b;
    b.x = V.Bc[e];
    b.v = V.Bv[e];
    b.a = E.a;
    b.ok = lane < E.len;
    return b;
}

// KEYED: x is a key, tile << 16 | the mask of the columns before the entry's
// (bit 15 - c for column c); otherwise a column index, its tile by the map
template <bool KEYED>
__device__ __forceinline__ StgC stg_stage_c(const StgSmem &S, const unsigned *cmr, int J0, const StgB &b)
{
    unsigned t;
    if (KEYED)
        t = ((unsigned)b.x >> 16) & (SPA_SEGT - 1);
    else
        t = S.map[min((unsigned)((b.x >> 4) - J0), (unsigned)(SPA_WIN - 1))];
    StgC c;
    c.w = cmr[t];
    c.p = __dmul_rn(b.a, b.v);
    return c;
}

template <bool KEYED>
__device__ __forceinline__ int stg_pos(const StgB &b, const StgC &c, int rs)
{
    const unsigned before = KEYED ? (unsigned)b.x : (0xFFFF0000u >> (b.x & 15)); // columns before the entry's
    const int p = rs + (int)(c.w >> 16) + __popc(c.w & before & 0xFFFFu);
    return b.ok ? min(p, STG_CAP - 1) : STG_CAP;
}

// the key of a column index (its tile t in the segment)
__device__ __forceinline__ int stg_key(int t, int col)
{
    return (t << 16) | ((0xFFFF0000u >> (col & 15)) & 0xFFFFu);
}

template <bool KEYED, bool LONG>
__device__ __forceinline__ void stg_apply(const StgSmem &S, const StgView &V, double *acc, const unsigned *cmr,
                                          int rs, int J0, const StgEnt *ent, int ne, int lane)
{
    StgEnt E2 = ent[2];
    StgB B0 = stg_stage_b(V, ent[0], lane), B1 = stg_stage_b(V, ent[1], lane);
    StgC C0 = stg_stage_c<KEYED>(S, cmr, J0, B0);
#pragma unroll 4
    for (int j = 0; j < ne; j++)
    {
        const StgEnt E3 = ent[j + 3];
        const StgB B2 = stg_stage_b(V, E2, lane);
        const StgC C1 = stg_stage_c<KEYED>(S, cmr, J0, B1);
        const int p = stg_pos<KEYED>(B0, C0, rs);
        acc[p] = __dadd_rn(acc[p], C0.p);
        if (LONG)
        {
            const StgEnt Ej = ent[j];
            for (int e = Ej.b0 + 32 + lane; e < Ej.b0 + Ej.len; e += 32)
            {
                StgB b;
                b.x = V.Bc[e];
                b.v = V.Bv[e];
                b.a = Ej.a;
                b.ok = true;
                const StgC c = stg_stage_c<KEYED>(S, cmr, J0, b);
                const int q = stg_pos<KEYED>(b, c, rs);
                acc[q] = __dadd_rn(acc[q], c.p);
            }
        }
        __syncwarp();
        E2 = E3;
        B0 = B1;
        B1 = B2;
        C0 = C1;
    }
}

// A's row r of the staged tile row applied in column order, STG_STAGE
// entries at a time (lane per A tile stages its entries of the row); B rows
// restricted to the segment's tile columns [J0, J1) unless KEYED (a segment
// holding the whole tile row).
template <bool KEYED>
__device__ __forceinline__ void stg_row(StgSmem &S, const StgView &V, double *acc, const unsigned *cmr, int rs,
                                        int J0, int J1, int r, int lane)
{
    StgEnt *ent = S.ent[r];
    for (int g = 0; g < V.nA; g += 32)
    {
        const int a = g + lane;
        unsigned mr = 0u;
        int stv = 0, kb = 0;
        int2 tba = make_int2(0, 0);
        if (a < V.nA)
        {
            mr = V.Am[a * TSG_BS + r];
            if (mr)
            {
                stv = V.At[a] + V.AP[a * TSG_BS + r] - V.av0;
                kb = V.Ac[a] * TSG_BS;
                tba = V.tb[a];
            }
        }
        const int *blk = V.rp + a * STG_RPB; // B row k's pointer at blk[k - tba.x]
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
        for (int base = 0; base < total; base += STG_STAGE)
        {
            __syncwarp();
            bool lng = false;
            unsigned bits = mr;
            for (int x = 0; x < cnt; x++)
            {
                const int bit = 31 - __clz(bits);
                bits ^= 1u << bit;
                const int e = incl - cnt + x - base;
                if (e >= 0 && e < STG_STAGE)
                {
                    const int k = kb + 15 - bit;
                    int b0 = blk[k - tba.x] + tba.y, b1 = blk[k + 1 - tba.x] + tba.y;
                    if (!KEYED)
                    {
                        // only B's entries inside this segment's columns
                        b0 += lower_bound_int(V.Bc + b0, b1 - b0, J0 * TSG_BS);
                        b1 = b0 + lower_bound_int(V.Bc + b0, b1 - b0, J1 * TSG_BS);
                    }
                    StgEnt E;
                    E.b0 = b0;
                    E.len = (unsigned short)(b1 - b0);
                    E.last = (unsigned short)max(b1 - b0 - 1, 0);
                    E.a = V.Av[stv + x];
                    ent[e] = E;
                    lng |= b1 - b0 > 32;
                }
            }
            const int ne = min(STG_STAGE, total - base);
            if (lane < 3)
            {
                StgEnt E;
                E.b0 = 0;
                E.len = E.last = 0;
                E.a = 0.0;
                ent[ne + lane] = E; // the three empty entries after the last
            }
            __syncwarp();
            if (__any_sync(TSG_FULL_MASK, lng))
                stg_apply<KEYED, true>(S, V, acc, cmr, rs, J0, ent, ne, lane);
            else
                stg_apply<KEYED, false>(S, V, acc, cmr, rs, J0, ent, ne, lane);
        }
    }
}

// ---------------------------------------------------------------------------
// bulk stores (shared -> global), one group per segment
// ---------------------------------------------------------------------------
__device__ __forceinline__ void stg_bulk_store(void *dst, const void *src, unsigned bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(stg_sa(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void stg_bulk_commit()
{
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// the issuing thread's bulk stores have finished reading shared memory
__device__ __forceinline__ void stg_bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// ... and have completed
__device__ __forceinline__ void stg_bulk_wait()
{
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// A segment: C tiles [t0, t1) of the staged tile row (at most SPA_SEGT
// tiles and STG_CAP values, tile columns less than SPA_WIN past the first).
// Row r accumulates in a private run sorted by column (the SPA segment's
// layout: a B row's products then spread over the banks), its word of tile
// t = (entries of the row in earlier tiles << 16) | row mask, so a
// product's slot is the row's start + one word load and a popcount; a
// segment holding the whole tile row (KEYED) first replaces every staged B
// column index by its key (stg_key).  The values are then laid
// out in C's order next to the column bytes and leave by bulk stores (their
// unaligned ends by plain stores), which read shared memory while the next
// segment is set up.  All consumer threads call it.
__device__ __forceinline__ void stg_segment(const ProdView &P, StgSmem &S, const StgView &V, int t0, int t1)
{
    const int tid = threadIdx.x, lane = tid & 31, r = tid >> 5;
    const int J0 = V.Cc[t0], J1 = V.Cc[t1 - 1] + 1;
    const int nt = min(t1 - t0, SPA_SEGT);
    const int g0 = V.Ct[t0], cn = min(V.Ct[t1] - g0, STG_CAP); // C values [g0, g0 + cn)
    const bool keyed = t0 == 0 && t1 == V.nC && J1 - J0 <= SPA_WIN;
    // the previous segment's bulk stores have read the output buffers
    if (tid == 0)
        stg_bulk_wait_read();
    for (int q = tid; q < cn; q += STG_CONS_THREADS)
        S.acc[q] = 0.0;
    for (int u = tid; u < nt * TSG_BS; u += STG_CONS_THREADS)
    {
        const int jl = u >> 4, rr = u & 15;
        S.cm[rr][jl] = V.Cm[(t0 + jl) * TSG_BS + rr];
        if (rr == 0)
        {
            const int w = V.Cc[t0 + jl] - J0;
            if (w < SPA_WIN)
                S.map[w] = (unsigned short)jl;
        }
    }
    stg_cons_sync();
    unsigned *cmr = S.cm[r];
    {
        // row r's run: its entries in earlier tiles of the segment
        int run = 0;
        for (int s0 = 0; s0 < nt; s0 += 32)
        {
            const int sl = s0 + lane;
            const unsigned m = sl < nt ? cmr[sl] : 0u;
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
                cmr[sl] = ((unsigned)(run + incl - c) << 16) | m;
            run += __shfl_sync(TSG_FULL_MASK, incl, 31);
        }
        if (lane == 0)
            S.rtot[r] = run;
    }
    if (keyed)
        for (int e = tid; e < V.nB; e += STG_CONS_THREADS)
        {
            const int col = V.Bc[e]; // the rounding's extra entries too: their keys are never read
            const unsigned w = min((unsigned)((col >> 4) - J0), (unsigned)(SPA_WIN - 1));
            V.Bc[e] = stg_key(S.map[w], col);
        }
    stg_cons_sync();
    const int rs = __reduce_add_sync(TSG_FULL_MASK, lane < r ? S.rtot[lane] : 0);
    if (lane == 0)
        S.rbase[r] = rs;
    if (keyed)
        stg_row<true>(S, V, S.acc, cmr, rs, J0, J1, r, lane);
    else
        stg_row<false>(S, V, S.acc, cmr, rs, J0, J1, r, lane);
    stg_cons_sync();
    // C's values and column bytes of the segment, in C's order, at the
    // 16-byte phase of their global range
    double *out = S.outbuf + (g0 & 1);
    unsigned char *colb = S.colbuf + (g0 & 15);
    for (int u = tid; u < nt * TSG_BS; u += STG_CONS_THREADS)
    {
        const int jl = u >> 4, rr = u & 15;
        const unsigned w = S.cm[rr][jl];
        unsigned mk = w & 0xFFFFu;
        int q = S.rbase[rr] + (int)(w >> 16);
        int p = V.Ct[t0 + jl] - g0 + V.CP[(t0 + jl) * TSG_BS + rr];
        while (mk)
        {
            const int bit = 31 - __clz(mk);
            mk ^= 1u << bit;
            const int pc = min(p, STG_CAP - 1);
            out[pc] = S.acc[min(q, STG_CAP - 1)];
            colb[pc] = (unsigned char)(15 - bit);
            p++;
            q++;
        }
    }
    // out: 16-byte aligned interiors by bulk stores, the ends by plain stores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    stg_cons_sync();
    const long long e0 = g0, e1 = (long long)g0 + cn;
    const long long v0 = (e0 + 1) & ~1LL, v1 = e1 & ~1LL;   // values: 2 per 16 bytes
    const long long b0 = (e0 + 15) & ~15LL, b1 = e1 & ~15LL; // bytes: 16 per 16 bytes
    if (tid == 0)
    {
        if (v1 > v0)
            stg_bulk_store(P.C_Val + v0, out + (v0 - e0), 8u * (unsigned)(v1 - v0));
        if (b1 > b0)
            stg_bulk_store(P.C_Colb + b0, colb + (b0 - e0), (unsigned)(b1 - b0));
        stg_bulk_commit();
    }
    if (tid < 32)
    {
        // values outside the bulk interior [v0, v1): at most one at each end
        // (all of them, at most three, when there is no interior)
        const long long hv = v1 > v0 ? v0 : e1;
        long long q = e0 + tid;
        if (q < hv)
            P.C_Val[q] = out[q - e0];
        q = v1 + tid;
        if (v1 > v0 && q < e1)
            P.C_Val[q] = out[q - e0];
    }
    else if (tid < 64)
    {
        // bytes outside the bulk interior [b0, b1): at most 15 at each end
        // (all of them, at most 31, when there is no interior)
        const int i = tid - 32;
        const long long hb = b1 > b0 ? b0 : e1;
        long long q = e0 + i;
        if (q < hb)
            P.C_Colb[q] = colb[q - e0];
        q = b1 + i;
        if (b1 > b0 && q < e1)
            P.C_Colb[q] = colb[q - e0];
    }
}

// The staged tile row by the consumer warps: segments within the SPA
// limits (one segment when the tile row fits them).
__device__ __forceinline__ void stg_tile_row(const ProdView &P, StgSmem &S, int s)
{
    const StgView V = stg_view(S, s);
    for (int t0 = 0; t0 < V.nC;)
    {
        const int cand = t0 + 1 + (int)threadIdx.x;
        const bool ok = threadIdx.x < SPA_SEGT && cand <= V.nC && V.Ct[cand] - V.Ct[t0] <= STG_CAP &&
                        V.Cc[cand - 1] - V.Cc[t0] < SPA_WIN;
        const int n = stg_cons_count(ok);
        const int t1 = t0 + (n > 0 ? n : 1);
        stg_segment(P, S, V, t0, t1);
        t0 = t1;
    }
}

// RANGED: only the tile rows [row0, row1).  ctr: the tile-row claim
// counter (zeroed); left[tilemA + 1] zeroed: rows left to the SPA kernel
// and their count.
template <bool RANGED>
__global__ void __launch_bounds__(STG_THREADS, 1) k_step3_stg(ProdView P, const int *__restrict__ kind, int row0,
                                                              int row1, unsigned *__restrict__ ctr,
                                                              int *__restrict__ left, int *__restrict__ status)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    StgSmem &S = *reinterpret_cast<StgSmem *>(s_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int q = tid; q < SPA_WIN; q += STG_THREADS)
        S.map[q] = 0; // every map entry names a tile of a segment
    if (tid == 0)
    {
        stg_bar_init(&S.full[0], 32);
        stg_bar_init(&S.full[1], 32);
        stg_bar_init(&S.empty[0], 1);
        stg_bar_init(&S.empty[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int r_beg = RANGED ? row0 : 0, r_end = RANGED ? row1 : P.tilemA;
    if (warp >= STG_CONS)
    {
        // producer of stage s: its plan of the next tile row is made while
        // the stage's copies are in flight and the consumers work; the two
        // producers claim tile rows independently
        const int s = warp - STG_CONS;
        unsigned nxt = 0;
        if (lane == 0)
            nxt = atomicAdd(ctr, 1u);
        StgPlan L = stg_plan(P, r_beg + (int)__shfl_sync(TSG_FULL_MASK, nxt, 0), r_end, kind, lane);
        for (int k = 0;; k++) // k-th fill of stage s
        {
            if (L.I < r_end && lane == 0)
                nxt = atomicAdd(ctr, 1u); // the tile row after it
            if (k >= 1)
            {
                bool ok = true;
                if (lane == 0)
                    ok = stg_bar_wait(&S.empty[s], (k - 1) & 1, status);
                if (!__shfl_sync(TSG_FULL_MASK, (int)ok, 0))
                    return;
            }
            if (L.I >= r_end)
            {
                if (lane == 0)
                    S.hdr[s].I = -1;
                __syncwarp();
                stg_bar_arrive(&S.full[s]);
                return;
            }
            stg_issue(P, S, s, L, left, lane);
            L = stg_plan(P, r_beg + (int)__shfl_sync(TSG_FULL_MASK, nxt, 0), r_end, kind, lane);
        }
    }
    // consumers: the stages in turn; a stage whose producer has finished is
    // passed over, and the consumers leave when both have
    bool done0 = false, done1 = false;
    for (int n = 0;; n++)
    {
        const int s = n & 1;
        if (s ? done1 : done0)
            continue;
        const bool ok = stg_bar_wait(&S.full[s], (n >> 1) & 1, status);
        if (stg_cons_count(!ok) > 0)
            break; // some consumer gave up waiting: all leave together
        if (S.hdr[s].I < 0)
        {
            (s ? done1 : done0) = true;
            if (done0 && done1)
                break;
            continue;
        }
        if (!S.hdr[s].skip)
            stg_tile_row(P, S, s);
        stg_cons_sync();
        if (tid == 0)
            stg_bar_arrive(&S.empty[s]);
    }
    if (tid == 0)
        stg_bulk_wait(); // the last segment's stores, before the CTA's shared memory goes
}
