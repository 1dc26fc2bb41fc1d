/*
 * CPU oracle for the tiled SpGEMM path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates the reference's CPU algorithms in plain C so that the
 * GPU library can be checked bit for bit.  It is linked only by tests/, the
 * smoke check and bench.py's CPU-baseline leg; the product never calls it.
 * Build: oracle/Makefile (-O3 -ffp-contract=off: multiply and add are rounded
 * separately, exactly like the reference's x86-64 build).
 *
 * Reference files (for-the-juan/RW-SpGEMM, relative to its root):
 *   src/csr2tile.h         CSR -> tiles (row-major A, column-major B)
 *   src/spgemm-cpu.h       tiled SpGEMM steps 1-4 (structure, mask, values)
 *   src/tile2csr.h         tiles -> CSR
 *   src/spgemm_serialref_spa_new.h   element-level SPA (structure)
 *   src/main.cu:392-397    product count nnzCub
 *   src/reorder.h:2429-2551          bipermutation apply / restore
 *   reorder_algorithm/common/order_utils.py:78-81   degree ordering
 */
#include "tsg_oracle.h"

#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#define BS 16

static int ceil_div16(int x) { return (x + BS - 1) / BS; }

static void *xcalloc(size_t n, size_t sz)
{
    void *p = calloc(n ? n : 1, sz ? sz : 1);
    if (!p)
        abort();
    return p;
}

static void *xmalloc(size_t sz)
{
    void *p = malloc(sz ? sz : 1);
    if (!p)
        abort();
    return p;
}

static int cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* ------------------------------------------------------------------------ */
/* CSR -> row-major tiles: src/csr2tile.h:6-259.                             */
/* Per tile row the distinct tile columns are sorted (:226-230); entries are */
/* placed per tile row-major, each row in CSR order (:152-189); the column   */
/* byte is (row<<4)|col (:185); mask bit 15-col (:186); tile_csr_Ptr is an  */
/* exclusive scan over the 16 row counts, so rows past the edge hold the     */
/* tile nnz (:234-237).                                                      */
/* ------------------------------------------------------------------------ */
static void build_row_major(OMatrix *mat, int packed)
{
    const int m = mat->m;
    mat->tilem = ceil_div16(m);
    mat->tilen = ceil_div16(mat->n);
    const int tilem = mat->tilem, tilen = mat->tilen;
    int *slot = (int *)xmalloc((size_t)tilen * sizeof(int));
    for (int j = 0; j < tilen; j++)
        slot[j] = -1;
    int *cols = (int *)xmalloc((size_t)(tilen > 0 ? tilen : 1) * sizeof(int));

    /* pass 1: count tiles per tile row */
    mat->tile_ptr = (int *)xcalloc((size_t)tilem + 1, sizeof(int));
    for (int bi = 0; bi < tilem; bi++)
    {
        int r0 = bi * BS, r1 = (bi + 1) * BS < m ? (bi + 1) * BS : m;
        int cnt = 0;
        for (int p = mat->rowpointer[r0]; p < mat->rowpointer[r1]; p++)
        {
            int jc = mat->columnindex[p] / BS;
            if (slot[jc] < 0)
            {
                slot[jc] = 0;
                cols[cnt++] = jc;
            }
        }
        for (int t = 0; t < cnt; t++)
            slot[cols[t]] = -1;
        mat->tile_ptr[bi + 1] = mat->tile_ptr[bi] + cnt;
    }
    const int T = mat->tile_ptr[tilem];
    mat->numtile = T;
    mat->tile_columnidx = (int *)xcalloc((size_t)T, sizeof(int));
    mat->tile_rowidx = (int *)xcalloc((size_t)T, sizeof(int));
    mat->tile_nnz = (int *)xcalloc((size_t)T + 1, sizeof(int));
    mat->tile_csr_Ptr = (unsigned char *)xcalloc((size_t)T * BS, 1);
    mat->tile_csr_Col = (unsigned char *)xcalloc((size_t)mat->nnz, 1);
    mat->tile_csr_Value = (double *)xcalloc((size_t)mat->nnz, sizeof(double));
    mat->mask = (unsigned short *)xcalloc((size_t)T * BS, sizeof(unsigned short));
    int *fill = (int *)xcalloc((size_t)T * BS, sizeof(int));

    /* pass 2: sorted tile columns, per-(tile,row) counts */
    for (int bi = 0; bi < tilem; bi++)
    {
        int r0 = bi * BS, r1 = (bi + 1) * BS < m ? (bi + 1) * BS : m;
        int base = mat->tile_ptr[bi], cnt = 0;
        for (int p = mat->rowpointer[r0]; p < mat->rowpointer[r1]; p++)
        {
            int jc = mat->columnindex[p] / BS;
            if (slot[jc] < 0)
            {
                slot[jc] = 0;
                cols[cnt++] = jc;
            }
        }
        qsort(cols, (size_t)cnt, sizeof(int), cmp_int);
        for (int t = 0; t < cnt; t++)
        {
            slot[cols[t]] = base + t;
            mat->tile_columnidx[base + t] = cols[t];
            mat->tile_rowidx[base + t] = bi;
        }
        for (int r = r0; r < r1; r++)
            for (int p = mat->rowpointer[r]; p < mat->rowpointer[r + 1]; p++)
            {
                int t = slot[mat->columnindex[p] / BS];
                mat->tile_nnz[t + 1]++;
                mat->tile_csr_Ptr[(size_t)t * BS + (r - r0)]++;
            }
        for (int t = 0; t < cnt; t++)
            slot[cols[t]] = -1;
    }
    for (int t = 0; t < T; t++)
        mat->tile_nnz[t + 1] += mat->tile_nnz[t];
    for (int t = 0; t < T; t++)
    {
        unsigned char run = 0;
        for (int r = 0; r < BS; r++)
        {
            unsigned char c = mat->tile_csr_Ptr[(size_t)t * BS + r];
            mat->tile_csr_Ptr[(size_t)t * BS + r] = run;
            run = (unsigned char)(run + c);
        }
    }
    /* pass 3: scatter in CSR order */
    for (int bi = 0; bi < tilem; bi++)
    {
        int r0 = bi * BS, r1 = (bi + 1) * BS < m ? (bi + 1) * BS : m;
        int base = mat->tile_ptr[bi], cnt = mat->tile_ptr[bi + 1] - base;
        for (int t = 0; t < cnt; t++)
            slot[mat->tile_columnidx[base + t]] = base + t;
        for (int r = r0; r < r1; r++)
            for (int p = mat->rowpointer[r]; p < mat->rowpointer[r + 1]; p++)
            {
                int c = mat->columnindex[p];
                int t = slot[c / BS];
                int ri = r - r0, ci = c % BS;
                size_t dst = (size_t)mat->tile_nnz[t] + mat->tile_csr_Ptr[(size_t)t * BS + ri] +
                             fill[(size_t)t * BS + ri]++;
                mat->tile_csr_Col[dst] = (unsigned char)(packed ? ((ri << 4) + ci) : ci);
                mat->tile_csr_Value[dst] = mat->value[p];
                mat->mask[(size_t)t * BS + ri] |= (unsigned short)(1u << (BS - ci - 1));
            }
        for (int t = 0; t < cnt; t++)
            slot[mat->tile_columnidx[base + t]] = -1;
    }
    free(fill);
    free(slot);
    free(cols);
}

void tsgo_csr2tile_row_major(OMatrix *mat)
{
    build_row_major(mat, 1);
    mat->csc_tile_ptr = NULL;
    mat->csc_tile_rowidx = NULL;
}

/* ------------------------------------------------------------------------ */
/* CSR -> column-major tiles: src/csr2tile.h:261-478.                        */
/* Tiles ordered by tile column, then tile row (csc_tile_ptr /               */
/* csc_tile_rowidx, :290-329); tile_nnz is the scan in that order (:303);    */
/* each tile holds an in-tile CSR with ascending plain column bytes (:437-   */
/* 456; the sub-transposes sort columns); tile_csr_Ptr of rows past the edge */
/* equals the tile nnz (:460-463); tile_ptr / tile_columnidx are the         */
/* row-major structure for step 1 (:310-349, :366-370) and tile_rowidx stays */
/* zero-filled (:318-319, never written).                                    */
/* ------------------------------------------------------------------------ */
typedef struct
{
    int col;
    int pos;
} ColPos;

static int cmp_colpos(const void *a, const void *b)
{
    const ColPos *x = (const ColPos *)a, *y = (const ColPos *)b;
    if (x->col != y->col)
        return (x->col > y->col) - (x->col < y->col);
    return (x->pos > y->pos) - (x->pos < y->pos);
}

void tsgo_csr2tile_col_major(OMatrix *mat)
{
    OMatrix rm;
    memset(&rm, 0, sizeof(rm));
    rm.m = mat->m;
    rm.n = mat->n;
    rm.nnz = mat->nnz;
    rm.rowpointer = mat->rowpointer;
    rm.columnindex = mat->columnindex;
    rm.value = mat->value;
    build_row_major(&rm, 0);

    const int T = rm.numtile, tilem = rm.tilem, tilen = rm.tilen;
    mat->tilem = tilem;
    mat->tilen = tilen;
    mat->numtile = T;
    mat->tile_ptr = rm.tile_ptr;
    mat->tile_columnidx = rm.tile_columnidx;
    mat->tile_rowidx = (int *)xcalloc((size_t)T, sizeof(int));

    /* sort each in-tile row by column (stable), keeping values */
    ColPos *buf = (ColPos *)xmalloc(BS * sizeof(ColPos));
    double vtmp[BS];
    for (int t = 0; t < T; t++)
    {
        int tn = rm.tile_nnz[t + 1] - rm.tile_nnz[t];
        for (int r = 0; r < BS; r++)
        {
            int s = rm.tile_csr_Ptr[(size_t)t * BS + r];
            int e = r == BS - 1 ? tn : rm.tile_csr_Ptr[(size_t)t * BS + r + 1];
            int len = e - s;
            if (len <= 1)
                continue;
            size_t off = (size_t)rm.tile_nnz[t] + s;
            for (int q = 0; q < len; q++)
            {
                buf[q].col = rm.tile_csr_Col[off + q];
                buf[q].pos = q;
                vtmp[q] = rm.tile_csr_Value[off + q];
            }
            qsort(buf, (size_t)len, sizeof(ColPos), cmp_colpos);
            for (int q = 0; q < len; q++)
            {
                rm.tile_csr_Col[off + q] = (unsigned char)buf[q].col;
                rm.tile_csr_Value[off + q] = vtmp[buf[q].pos];
            }
        }
    }
    free(buf);

    /* column-major order: counting sort of tiles by tile column, stable */
    int *cptr = (int *)xcalloc((size_t)tilen + 1, sizeof(int));
    for (int t = 0; t < T; t++)
        cptr[rm.tile_columnidx[t] + 1]++;
    for (int j = 0; j < tilen; j++)
        cptr[j + 1] += cptr[j];
    int *cur = (int *)xmalloc(((size_t)tilen + 1) * sizeof(int));
    memcpy(cur, cptr, ((size_t)tilen + 1) * sizeof(int));
    int *perm = (int *)xmalloc((size_t)(T ? T : 1) * sizeof(int)); /* colmajor idx -> rowmajor idx */
    mat->csc_tile_rowidx = (int *)xcalloc((size_t)T, sizeof(int));
    for (int bi = 0; bi < tilem; bi++)
        for (int t = rm.tile_ptr[bi]; t < rm.tile_ptr[bi + 1]; t++)
        {
            int q = cur[rm.tile_columnidx[t]]++;
            perm[q] = t;
            mat->csc_tile_rowidx[q] = bi;
        }
    free(cur);
    mat->csc_tile_ptr = cptr;

    mat->tile_nnz = (int *)xcalloc((size_t)T + 1, sizeof(int));
    for (int q = 0; q < T; q++)
        mat->tile_nnz[q + 1] = mat->tile_nnz[q] + (rm.tile_nnz[perm[q] + 1] - rm.tile_nnz[perm[q]]);
    mat->tile_csr_Ptr = (unsigned char *)xcalloc((size_t)T * BS, 1);
    mat->mask = (unsigned short *)xcalloc((size_t)T * BS, sizeof(unsigned short));
    mat->tile_csr_Col = (unsigned char *)xcalloc((size_t)mat->nnz, 1);
    mat->tile_csr_Value = (double *)xcalloc((size_t)mat->nnz, sizeof(double));
    for (int q = 0; q < T; q++)
    {
        int t = perm[q];
        int tn = rm.tile_nnz[t + 1] - rm.tile_nnz[t];
        memcpy(mat->tile_csr_Ptr + (size_t)q * BS, rm.tile_csr_Ptr + (size_t)t * BS, BS);
        memcpy(mat->mask + (size_t)q * BS, rm.mask + (size_t)t * BS, BS * sizeof(unsigned short));
        memcpy(mat->tile_csr_Col + mat->tile_nnz[q], rm.tile_csr_Col + rm.tile_nnz[t], (size_t)tn);
        memcpy(mat->tile_csr_Value + mat->tile_nnz[q], rm.tile_csr_Value + rm.tile_nnz[t],
               (size_t)tn * sizeof(double));
    }
    free(perm);
    free(rm.tile_rowidx);
    free(rm.tile_nnz);
    free(rm.tile_csr_Ptr);
    free(rm.tile_csr_Col);
    free(rm.tile_csr_Value);
    free(rm.mask);
}

/* ------------------------------------------------------------------------ */
/* Tiled SpGEMM: src/spgemm-cpu.h.                                           */
/* step1/step2 (:3-96): C tile (i,j) exists iff some k has A-tile(i,k) and   */
/* B-tile(k,j) non-empty; columns ascending per tile row.                    */
/* step3/step4 (:185-367): for every C tile, matched k ascending (merge of   */
/* A's tile row with B's tile column), for each row ri, each A entry in      */
/* stored order (column = byte & 0xf, the unpack the shipped oracle lacks),  */
/* each B entry of row cola in stored order: blkcval[ri][colb] += a*b        */
/* (:330).  Output per C tile: entries row-major, columns ascending          */
/* (:351-364), Ptr = running count, mask bit 15-col.                         */
/* ------------------------------------------------------------------------ */
void tsgo_spgemm_tiled(const OMatrix *A, const OMatrix *B, OMatrix *C)
{
    const int tilemA = A->tilem, tilenB = B->tilen;
    memset(C, 0, sizeof(*C));
    C->m = A->m;
    C->n = B->n;
    C->tilem = tilemA;
    C->tilen = tilenB;

    /* step 1: structure, per tile row union of B tile rows */
    int *mark = (int *)xmalloc((size_t)(tilenB ? tilenB : 1) * sizeof(int));
    for (int j = 0; j < tilenB; j++)
        mark[j] = -1;
    int *cols = (int *)xmalloc((size_t)(tilenB ? tilenB : 1) * sizeof(int));
    C->tile_ptr = (int *)xcalloc((size_t)tilemA + 1, sizeof(int));
    size_t cap = 1024, used = 0;
    int *ccol = (int *)xmalloc(cap * sizeof(int));
    for (int i = 0; i < tilemA; i++)
    {
        int cnt = 0;
        for (int pa = A->tile_ptr[i]; pa < A->tile_ptr[i + 1]; pa++)
        {
            int k = A->tile_columnidx[pa];
            for (int pb = B->tile_ptr[k]; pb < B->tile_ptr[k + 1]; pb++)
            {
                int j = B->tile_columnidx[pb];
                if (mark[j] != i)
                {
                    mark[j] = i;
                    cols[cnt++] = j;
                }
            }
        }
        qsort(cols, (size_t)cnt, sizeof(int), cmp_int);
        if (used + (size_t)cnt > cap)
        {
            while (used + (size_t)cnt > cap)
                cap *= 2;
            ccol = (int *)realloc(ccol, cap * sizeof(int));
            if (!ccol)
                abort();
        }
        memcpy(ccol + used, cols, (size_t)cnt * sizeof(int));
        used += (size_t)cnt;
        C->tile_ptr[i + 1] = (int)used;
    }
    free(mark);
    free(cols);
    const int TC = (int)used;
    C->numtile = TC;
    C->tile_columnidx = ccol;
    C->tile_rowidx = (int *)xcalloc((size_t)TC, sizeof(int));
    for (int i = 0; i < tilemA; i++)
        for (int t = C->tile_ptr[i]; t < C->tile_ptr[i + 1]; t++)
            C->tile_rowidx[t] = i;

    /* steps 2+3: per C tile dense 16x16 accumulation in k order */
    C->tile_nnz = (int *)xcalloc((size_t)TC + 1, sizeof(int));
    C->tile_csr_Ptr = (unsigned char *)xcalloc((size_t)TC * BS, 1);
    C->mask = (unsigned short *)xcalloc((size_t)TC * BS, sizeof(unsigned short));
    size_t vcap = 4096, vused = 0;
    unsigned char *vcol = (unsigned char *)xmalloc(vcap);
    double *vval = (double *)xmalloc(vcap * sizeof(double));
    double acc[BS * BS];
    unsigned char hit[BS * BS];
    for (int i = 0; i < tilemA; i++)
    {
        const int rowlen = i == tilemA - 1 ? A->m - (tilemA - 1) * BS : BS;
        for (int t = C->tile_ptr[i]; t < C->tile_ptr[i + 1]; t++)
        {
            const int j = C->tile_columnidx[t];
            memset(acc, 0, sizeof(acc));
            memset(hit, 0, sizeof(hit));
            int pa = A->tile_ptr[i], ea = A->tile_ptr[i + 1];
            int pb = B->csc_tile_ptr[j], eb = B->csc_tile_ptr[j + 1];
            while (pa < ea && pb < eb)
            {
                int ka = A->tile_columnidx[pa], kb = B->csc_tile_rowidx[pb];
                if (ka < kb)
                    pa++;
                else if (ka > kb)
                    pb++;
                else
                {
                    const int na = A->tile_nnz[pa + 1] - A->tile_nnz[pa];
                    const int nb = B->tile_nnz[pb + 1] - B->tile_nnz[pb];
                    const unsigned char *aptr = A->tile_csr_Ptr + (size_t)pa * BS;
                    const unsigned char *bptr = B->tile_csr_Ptr + (size_t)pb * BS;
                    const unsigned char *acol = A->tile_csr_Col + A->tile_nnz[pa];
                    const unsigned char *bcol = B->tile_csr_Col + B->tile_nnz[pb];
                    const double *aval = A->tile_csr_Value + A->tile_nnz[pa];
                    const double *bval = B->tile_csr_Value + B->tile_nnz[pb];
                    for (int ri = 0; ri < rowlen; ri++)
                    {
                        int sa = aptr[ri], stopa = ri == BS - 1 ? na : aptr[ri + 1];
                        for (int x = sa; x < stopa; x++)
                        {
                            int cola = acol[x] & 0xf;
                            double a = aval[x];
                            int sb = bptr[cola], stopb = cola == BS - 1 ? nb : bptr[cola + 1];
                            for (int y = sb; y < stopb; y++)
                            {
                                int colb = bcol[y];
                                acc[ri * BS + colb] += a * bval[y];
                                hit[ri * BS + colb] = 1;
                            }
                        }
                    }
                    pa++;
                    pb++;
                }
            }
            int count = 0;
            if (vused + BS * BS > vcap)
            {
                while (vused + BS * BS > vcap)
                    vcap *= 2;
                vcol = (unsigned char *)realloc(vcol, vcap);
                vval = (double *)realloc(vval, vcap * sizeof(double));
                if (!vcol || !vval)
                    abort();
            }
            for (int ri = 0; ri < BS; ri++)
            {
                C->tile_csr_Ptr[(size_t)t * BS + ri] = (unsigned char)count;
                unsigned short mk = 0;
                for (int ci = 0; ci < BS; ci++)
                    if (hit[ri * BS + ci])
                    {
                        vcol[vused + count] = (unsigned char)ci;
                        vval[vused + count] = acc[ri * BS + ci];
                        mk |= (unsigned short)(1u << (BS - 1 - ci));
                        count++;
                    }
                C->mask[(size_t)t * BS + ri] = mk;
            }
            vused += (size_t)count;
            C->tile_nnz[t + 1] = (int)vused;
        }
    }
    C->nnz = (int)vused;
    C->tile_csr_Col = vcol;
    C->tile_csr_Value = vval;
}

/* ------------------------------------------------------------------------ */
/* Tiles -> CSR: src/tile2csr.h:8-137.  Row r of tile row i gets, tile by    */
/* tile in tile order, the entries [Ptr[r], Ptr[r+1]) (the last real row     */
/* ends at the tile nnz), column = 16*tilecol + byte; zeros are kept.        */
/* ------------------------------------------------------------------------ */
void tsgo_tile2csr(OMatrix *mat)
{
    const int m = mat->m, tilem = mat->tilem;
    mat->rowpointer = (int *)xcalloc((size_t)m + 1, sizeof(int));
    for (int i = 0; i < tilem; i++)
    {
        int rowlen = i == tilem - 1 ? m - (tilem - 1) * BS : BS;
        for (int t = mat->tile_ptr[i]; t < mat->tile_ptr[i + 1]; t++)
        {
            int tn = mat->tile_nnz[t + 1] - mat->tile_nnz[t];
            const unsigned char *ptr = mat->tile_csr_Ptr + (size_t)t * BS;
            for (int r = 0; r < rowlen; r++)
            {
                int e = r == rowlen - 1 ? tn : ptr[r + 1];
                mat->rowpointer[i * BS + r + 1] += e - ptr[r];
            }
        }
    }
    for (int r = 0; r < m; r++)
        mat->rowpointer[r + 1] += mat->rowpointer[r];
    const int nnz = mat->rowpointer[m];
    mat->nnz = nnz;
    mat->columnindex = (int *)xcalloc((size_t)nnz, sizeof(int));
    mat->value = (double *)xcalloc((size_t)nnz, sizeof(double));
    int *fill = (int *)xcalloc((size_t)m + 1, sizeof(int));
    for (int i = 0; i < tilem; i++)
    {
        int rowlen = i == tilem - 1 ? m - (tilem - 1) * BS : BS;
        for (int t = mat->tile_ptr[i]; t < mat->tile_ptr[i + 1]; t++)
        {
            int tn = mat->tile_nnz[t + 1] - mat->tile_nnz[t];
            const unsigned char *ptr = mat->tile_csr_Ptr + (size_t)t * BS;
            int tc = mat->tile_columnidx[t];
            for (int r = 0; r < rowlen; r++)
            {
                int e = r == rowlen - 1 ? tn : ptr[r + 1];
                for (int q = ptr[r]; q < e; q++)
                {
                    int g = i * BS + r;
                    int dst = mat->rowpointer[g] + fill[g]++;
                    mat->columnindex[dst] = tc * BS + mat->tile_csr_Col[mat->tile_nnz[t] + q];
                    mat->value[dst] = mat->tile_csr_Value[mat->tile_nnz[t] + q];
                }
            }
        }
    }
    free(fill);
}

void tsgo_free_tiles(OMatrix *mat)
{
    free(mat->tile_ptr);
    free(mat->tile_columnidx);
    free(mat->tile_rowidx);
    free(mat->tile_nnz);
    free(mat->tile_csr_Ptr);
    free(mat->tile_csr_Col);
    free(mat->tile_csr_Value);
    free(mat->mask);
    free(mat->csc_tile_ptr);
    free(mat->csc_tile_rowidx);
    mat->tile_ptr = mat->tile_columnidx = mat->tile_rowidx = mat->tile_nnz = NULL;
    mat->tile_csr_Ptr = mat->tile_csr_Col = NULL;
    mat->tile_csr_Value = NULL;
    mat->mask = NULL;
    mat->csc_tile_ptr = mat->csc_tile_rowidx = NULL;
}

void tsgo_free_csr(OMatrix *mat)
{
    free(mat->rowpointer);
    free(mat->columnindex);
    free(mat->value);
    mat->rowpointer = mat->columnindex = NULL;
    mat->value = NULL;
}

/* nnzCub, src/main.cu:392-397 */
long long tsgo_count_products(int nnzA, const int *a_colidx, const int *b_rowptr)
{
    long long s = 0;
    for (int i = 0; i < nnzA; i++)
        s += b_rowptr[a_colidx[i] + 1] - b_rowptr[a_colidx[i]];
    return s;
}

/* ------------------------------------------------------------------------ */
/* Element-level Gustavson.  Structure as spgemm_spa                         */
/* (src/spgemm_serialref_spa_new.h:7-105: per row a column bitmask, popcount,*/
/* then columns emitted ascending); values accumulated per output element in */
/* A-row order, which for sorted rows is the tiled oracle's order            */
/* (k-tile ascending, in-tile column ascending, src/spgemm-cpu.h:330).       */
/* ------------------------------------------------------------------------ */
#ifdef _OPENMP
#include <omp.h>
#endif

long long tsgo_gustavson_symbolic(int m, int n,
                                  const int *a_rowptr, const int *a_col,
                                  const int *b_rowptr, const int *b_col,
                                  int *c_rowptr, int nthreads)
{
    if (nthreads <= 0)
        nthreads = 1;
    c_rowptr[0] = 0;
#pragma omp parallel num_threads(nthreads)
    {
        int *mark = (int *)xmalloc((size_t)(n ? n : 1) * sizeof(int));
        for (int j = 0; j < n; j++)
            mark[j] = -1;
#pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < m; i++)
        {
            int cnt = 0;
            for (int p = a_rowptr[i]; p < a_rowptr[i + 1]; p++)
            {
                int k = a_col[p];
                for (int q = b_rowptr[k]; q < b_rowptr[k + 1]; q++)
                {
                    int j = b_col[q];
                    if (mark[j] != i)
                    {
                        mark[j] = i;
                        cnt++;
                    }
                }
            }
            c_rowptr[i + 1] = cnt;
        }
        free(mark);
    }
    long long s = 0;
    for (int i = 0; i < m; i++)
    {
        s += c_rowptr[i + 1];
        if (s > 2147483647LL)
            return -1;
        c_rowptr[i + 1] = (int)s;
    }
    return s;
}

/* Per-row nnz of C = A*B (structure only, element level), as the symbolic
 * pass above but without a 32-bit row pointer: counts[i] = nnz(C row i),
 * returns the total as 64 bits (products of more than 2^31 nonzeros). */
long long tsgo_gustavson_row_nnz(int m, int n,
                                 const int *a_rowptr, const int *a_col,
                                 const int *b_rowptr, const int *b_col,
                                 int *counts, int nthreads)
{
    if (nthreads <= 0)
        nthreads = 1;
    long long total = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
    {
        int *mark = (int *)xmalloc((size_t)(n ? n : 1) * sizeof(int));
        for (int j = 0; j < n; j++)
            mark[j] = -1;
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < m; i++)
        {
            int cnt = 0;
            for (int p = a_rowptr[i]; p < a_rowptr[i + 1]; p++)
            {
                int k = a_col[p];
                for (int q = b_rowptr[k]; q < b_rowptr[k + 1]; q++)
                {
                    int j = b_col[q];
                    if (mark[j] != i)
                    {
                        mark[j] = i;
                        cnt++;
                    }
                }
            }
            counts[i] = cnt;
            total += cnt;
        }
        free(mark);
    }
    return total;
}

void tsgo_gustavson_numeric(int m, int n,
                            const int *a_rowptr, const int *a_col, const double *a_val,
                            const int *b_rowptr, const int *b_col, const double *b_val,
                            const int *c_rowptr, int *c_col, double *c_val, int nthreads)
{
    if (nthreads <= 0)
        nthreads = 1;
#pragma omp parallel num_threads(nthreads)
    {
        double *acc = (double *)xcalloc((size_t)(n ? n : 1), sizeof(double));
        int *mark = (int *)xmalloc((size_t)(n ? n : 1) * sizeof(int));
        for (int j = 0; j < n; j++)
            mark[j] = -1;
#pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < m; i++)
        {
            int base = c_rowptr[i], cnt = 0;
            for (int p = a_rowptr[i]; p < a_rowptr[i + 1]; p++)
            {
                int k = a_col[p];
                double a = a_val[p];
                for (int q = b_rowptr[k]; q < b_rowptr[k + 1]; q++)
                {
                    int j = b_col[q];
                    if (mark[j] != i)
                    {
                        mark[j] = i;
                        acc[j] = 0.0;
                        c_col[base + cnt++] = j;
                    }
                    acc[j] += a * b_val[q];
                }
            }
            qsort(c_col + base, (size_t)cnt, sizeof(int), cmp_int);
            for (int q = 0; q < cnt; q++)
                c_val[base + q] = acc[c_col[base + q]];
        }
        free(acc);
        free(mark);
    }
}

/* ------------------------------------------------------------------------ */
/* Orderings (new -> old).                                                   */
/* ------------------------------------------------------------------------ */

/* degree: sorted by (-degree, id), reorder_algorithm/common/order_utils.py:78-81,
 * degree = entries in the row (mirrored for symmetric inputs, as the CSR is). */
typedef struct
{
    long long k0, k1;
    int id;
} Key3;

static int cmp_key3(const void *a, const void *b)
{
    const Key3 *x = (const Key3 *)a, *y = (const Key3 *)b;
    if (x->k0 != y->k0)
        return (x->k0 > y->k0) - (x->k0 < y->k0);
    if (x->k1 != y->k1)
        return (x->k1 > y->k1) - (x->k1 < y->k1);
    return (x->id > y->id) - (x->id < y->id);
}

void tsgo_order_degree(int n, const int *rowptr, int *order)
{
    Key3 *k = (Key3 *)xmalloc((size_t)(n ? n : 1) * sizeof(Key3));
    for (int i = 0; i < n; i++)
    {
        k[i].k0 = -(long long)(rowptr[i + 1] - rowptr[i]);
        k[i].k1 = 0;
        k[i].id = i;
    }
    qsort(k, (size_t)n, sizeof(Key3), cmp_key3);
    for (int i = 0; i < n; i++)
        order[i] = k[i].id;
    free(k);
}

/* The reference's random ordering, order_utils.py:70-75:
 * random.Random(seed).shuffle(list(range(n))) of CPython, restated from its
 * published algorithm.  The generator is MT19937 (Matsumoto & Nishimura,
 * 1998) seeded by init_by_array with the seed's 32-bit words, low word
 * first (one word for seeds below 2^32, at least one); the shuffle is
 * Fisher-Yates from the last position down, position i swapped with
 * j = randbelow(i + 1), where randbelow(m) draws k = bit_length(m) bits
 * (the top k bits of one 32-bit output) until the value is below m. */
#define MT_N 624
#define MT_M 397

typedef struct
{
    unsigned int mt[MT_N];
    int next;
} Mt19937;

static void mt_init(Mt19937 *g, unsigned int s)
{
    g->mt[0] = s;
    for (int i = 1; i < MT_N; i++)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (unsigned int)i;
    g->next = MT_N;
}

static void mt_init_by_array(Mt19937 *g, const unsigned int *key, int len)
{
    mt_init(g, 19650218u);
    int i = 1, j = 0;
    for (int k = MT_N > len ? MT_N : len; k > 0; k--)
    {
        g->mt[i] = (g->mt[i] ^ ((g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) * 1664525u)) + key[j] + (unsigned int)j;
        i++;
        j++;
        if (i >= MT_N)
        {
            g->mt[0] = g->mt[MT_N - 1];
            i = 1;
        }
        if (j >= len)
            j = 0;
    }
    for (int k = MT_N - 1; k > 0; k--)
    {
        g->mt[i] = (g->mt[i] ^ ((g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) * 1566083941u)) - (unsigned int)i;
        i++;
        if (i >= MT_N)
        {
            g->mt[0] = g->mt[MT_N - 1];
            i = 1;
        }
    }
    g->mt[0] = 0x80000000u;
}

static unsigned int mt_twist_word(unsigned int hi, unsigned int lo, unsigned int far)
{
    const unsigned int y = (hi & 0x80000000u) | (lo & 0x7fffffffu);
    return far ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

static unsigned int mt_u32(Mt19937 *g)
{
    if (g->next >= MT_N)
    {
        for (int k = 0; k < MT_N; k++)
            g->mt[k] = mt_twist_word(g->mt[k], g->mt[(k + 1) % MT_N], g->mt[(k + MT_M) % MT_N]);
        g->next = 0;
    }
    unsigned int y = g->mt[g->next++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

void tsgo_order_random(int n, unsigned long long seed, int *order)
{
    unsigned int key[2] = {(unsigned int)seed, (unsigned int)(seed >> 32)};
    Mt19937 g;
    mt_init_by_array(&g, key, key[1] ? 2 : 1);
    for (int i = 0; i < n; i++)
        order[i] = i;
    for (int i = n - 1; i > 0; i--)
    {
        const unsigned int m = (unsigned int)i + 1u;
        int k = 0;
        while ((m >> k) != 0u)
            k++;
        unsigned int r;
        do
            r = mt_u32(&g) >> (32 - k);
        while (r >= m);
        const int t = order[i];
        order[i] = order[r];
        order[r] = t;
    }
}

/* Symmetrised off-diagonal adjacency (pattern of A + A^T without the
 * diagonal), rows sorted and duplicate-free. */
static void symmetric_graph(int n, const int *rowptr, const int *col, int **gptr_out, int **gadj_out)
{
    int *deg = (int *)xcalloc((size_t)n + 1, sizeof(int));
    for (int i = 0; i < n; i++)
        for (int p = rowptr[i]; p < rowptr[i + 1]; p++)
        {
            int j = col[p];
            if (j == i || j < 0 || j >= n)
                continue;
            deg[i + 1]++;
            deg[j + 1]++;
        }
    for (int i = 0; i < n; i++)
        deg[i + 1] += deg[i];
    int *adj = (int *)xmalloc((size_t)(deg[n] ? deg[n] : 1) * sizeof(int));
    int *cur = (int *)xmalloc(((size_t)n + 1) * sizeof(int));
    memcpy(cur, deg, ((size_t)n + 1) * sizeof(int));
    for (int i = 0; i < n; i++)
        for (int p = rowptr[i]; p < rowptr[i + 1]; p++)
        {
            int j = col[p];
            if (j == i || j < 0 || j >= n)
                continue;
            adj[cur[i]++] = j;
            adj[cur[j]++] = i;
        }
    /* sort + unique each row */
    int *gptr = (int *)xcalloc((size_t)n + 1, sizeof(int));
    int w = 0;
    for (int i = 0; i < n; i++)
    {
        int s = deg[i], e = deg[i + 1];
        qsort(adj + s, (size_t)(e - s), sizeof(int), cmp_int);
        int start = w;
        for (int p = s; p < e; p++)
            if (p == s || adj[p] != adj[p - 1])
                adj[w++] = adj[p];
        gptr[i] = start;
        gptr[i + 1] = w;
    }
    free(cur);
    free(deg);
    *gptr_out = gptr;
    *gadj_out = adj;
}

/* Reverse Cuthill-McKee on the symmetrised pattern.  Seeds: the unvisited
 * vertex with the smallest (degree, id); each visited vertex appends its
 * unvisited neighbours sorted by (degree, id); the final order is reversed.
 * This is the sequential scheme of scipy's reverse_cuthill_mckee (used by
 * reorder_algorithm/common/order_utils.py:84-104) with the (degree, id)
 * tie-break of src/reorder.h:1678-1722. */
void tsgo_order_rcm(int n, const int *rowptr, const int *col, int *order)
{
    int *gptr, *adj;
    symmetric_graph(n, rowptr, col, &gptr, &adj);
    Key3 *seeds = (Key3 *)xmalloc((size_t)(n > 0 ? n : 1) * sizeof(Key3));
    for (int i = 0; i < n; i++)
    {
        seeds[i].k0 = gptr[i + 1] - gptr[i];
        seeds[i].k1 = 0;
        seeds[i].id = i;
    }
    qsort(seeds, (size_t)n, sizeof(Key3), cmp_key3);
    unsigned char *vis = (unsigned char *)xcalloc((size_t)(n ? n : 1), 1);
    int *q = (int *)xmalloc((size_t)(n ? n : 1) * sizeof(int));
    Key3 *nb = (Key3 *)xmalloc((size_t)(n ? n : 1) * sizeof(Key3));
    int len = 0;
    for (int s = 0; s < n; s++)
    {
        int seed = seeds[s].id;
        if (vis[seed])
            continue;
        vis[seed] = 1;
        q[len++] = seed;
        for (int head = len - 1; head < len; head++)
        {
            int v = q[head], cnt = 0;
            for (int p = gptr[v]; p < gptr[v + 1]; p++)
            {
                int u = adj[p];
                if (vis[u])
                    continue;
                vis[u] = 1;
                nb[cnt].k0 = gptr[u + 1] - gptr[u];
                nb[cnt].k1 = 0;
                nb[cnt].id = u;
                cnt++;
            }
            qsort(nb, (size_t)cnt, sizeof(Key3), cmp_key3);
            for (int c = 0; c < cnt; c++)
                q[len++] = nb[c].id;
        }
    }
    for (int i = 0; i < n; i++)
        order[i] = q[n - 1 - i];
    free(q);
    free(nb);
    free(vis);
    free(seeds);
    free(gptr);
    free(adj);
}

/* Gray-code ordering (after Zhao et al.'s Gray-code row ordering, the scheme
 * SparseBase's gray_order implements; that tool is absent, so this is the
 * library's own definition).  Each row gets a 32-bit signature, bit (31-s)
 * set when the row has an entry in column segment s = col*32/ncols; rows are
 * split into a sparse group (length <= 2*ceil(nnz/n)) and a dense group, and
 * sorted by (group, Gray-decoded signature, id). */
static unsigned int gray_decode32(unsigned int g)
{
    g ^= g >> 1;
    g ^= g >> 2;
    g ^= g >> 4;
    g ^= g >> 8;
    g ^= g >> 16;
    return g;
}

void tsgo_order_gray(int n, int ncols, const int *rowptr, const int *col, int *order)
{
    long long nnz = n ? rowptr[n] : 0;
    long long thr = n ? 2 * ((nnz + n - 1) / n) : 0;
    Key3 *k = (Key3 *)xmalloc((size_t)(n ? n : 1) * sizeof(Key3));
    for (int i = 0; i < n; i++)
    {
        unsigned int sig = 0;
        for (int p = rowptr[i]; p < rowptr[i + 1]; p++)
        {
            long long s = ncols > 0 ? ((long long)col[p] * 32) / ncols : 0;
            if (s > 31)
                s = 31;
            sig |= 1u << (31 - (int)s);
        }
        int len = rowptr[i + 1] - rowptr[i];
        k[i].k0 = len > thr ? 1 : 0;
        k[i].k1 = gray_decode32(sig);
        k[i].id = i;
    }
    qsort(k, (size_t)n, sizeof(Key3), cmp_key3);
    for (int i = 0; i < n; i++)
        order[i] = k[i].id;
    free(k);
}

/* P_r * A * P_c^T, src/reorder.h:2429-2504 (rows gathered by new->old, columns
 * mapped old->new, each row sorted by new column with its values). */
void tsgo_apply_bipermutation(int m, const int *rowptr, const int *col, const double *val,
                              const int *row_old, const int *col_new,
                              int *out_rowptr, int *out_col, double *out_val)
{
    out_rowptr[0] = 0;
    for (int r = 0; r < m; r++)
    {
        int o = row_old[r];
        out_rowptr[r + 1] = out_rowptr[r] + (rowptr[o + 1] - rowptr[o]);
    }
    ColPos *buf = NULL;
    size_t bcap = 0;
    double *vb = NULL;
    for (int r = 0; r < m; r++)
    {
        int o = row_old[r];
        int s = rowptr[o], len = rowptr[o + 1] - s;
        if ((size_t)len > bcap)
        {
            bcap = (size_t)len * 2;
            buf = (ColPos *)realloc(buf, bcap * sizeof(ColPos));
            vb = (double *)realloc(vb, bcap * sizeof(double));
            if (!buf || !vb)
                abort();
        }
        for (int q = 0; q < len; q++)
        {
            buf[q].col = col_new[col[s + q]];
            buf[q].pos = q;
            vb[q] = val[s + q];
        }
        qsort(buf, (size_t)len, sizeof(ColPos), cmp_colpos);
        for (int q = 0; q < len; q++)
        {
            out_col[out_rowptr[r] + q] = buf[q].col;
            out_val[out_rowptr[r] + q] = vb[buf[q].pos];
        }
    }
    free(buf);
    free(vb);
}
