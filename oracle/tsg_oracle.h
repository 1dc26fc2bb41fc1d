/*
 * CPU oracle for the tiled SpGEMM path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference algorithm (for-the-juan/RW-SpGEMM,
 * TileSpGEMM).  It is the checker for the GPU library: only tests/, the
 * smoke check and bench.py's CPU-baseline leg may load it.  The product path
 * never calls it.  Every function cites the reference code it restates.
 *
 * Pinned by tests/test_oracle.py against (a) the reference's own CPU code
 * compiled from its sources into oracle/_ref/ (when the reference tree is
 * present) and (b) the known-answer fixtures in tests/golden/.
 */
#ifndef TSG_ORACLE_H
#define TSG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as the reference SMatrix (src/common.h:113-135). */
typedef struct
{
    int m;
    int n;
    int nnz;
    int isSymmetric;
    double *value;
    int *columnindex;
    int *rowpointer;
    int tilem;
    int tilen;
    int *tile_ptr;
    int *tile_columnidx;
    int *tile_rowidx;
    int *tile_nnz;
    int numtile;
    double *tile_csr_Value;
    unsigned char *tile_csr_Col;
    unsigned char *tile_csr_Ptr;
    unsigned short *mask;
    int *csc_tile_ptr;
    int *csc_tile_rowidx;
} OMatrix;

void tsgo_csr2tile_row_major(OMatrix *mat);
void tsgo_csr2tile_col_major(OMatrix *mat);
/* C = A*B on tiles; A row-major (packed Col), B column-major (plain Col).
 * Fills C: m, n, tilem, tilen, numtile, nnz, tile_ptr, tile_columnidx,
 * tile_rowidx, tile_nnz, tile_csr_Ptr, tile_csr_Col, tile_csr_Value, mask. */
void tsgo_spgemm_tiled(const OMatrix *A, const OMatrix *B, OMatrix *C);
void tsgo_tile2csr(OMatrix *mat);
void tsgo_free_tiles(OMatrix *mat);
void tsgo_free_csr(OMatrix *mat);

long long tsgo_count_products(int nnzA, const int *a_colidx, const int *b_rowptr);

/* Element-level CSR SpGEMM: symbolic pass (row lengths) and numeric pass
 * (sorted columns, FP64 values accumulated in A-row order).  nthreads <= 0
 * uses one thread.  Returns nnz(C) or -1. */
long long tsgo_gustavson_symbolic(int m, int n,
                                  const int *a_rowptr, const int *a_col,
                                  const int *b_rowptr, const int *b_col,
                                  int *c_rowptr, int nthreads);
long long tsgo_gustavson_row_nnz(int m, int n,
                                 const int *a_rowptr, const int *a_col,
                                 const int *b_rowptr, const int *b_col,
                                 int *counts, int nthreads);
void tsgo_gustavson_numeric(int m, int n,
                            const int *a_rowptr, const int *a_col, const double *a_val,
                            const int *b_rowptr, const int *b_col, const double *b_val,
                            const int *c_rowptr, int *c_col, double *c_val, int nthreads);

/* Orderings: new -> old permutations of n rows. */
void tsgo_order_degree(int n, const int *rowptr, int *order);
void tsgo_order_random(int n, unsigned long long seed, int *order);
void tsgo_order_rcm(int n, const int *rowptr, const int *col, int *order);
void tsgo_order_gray(int n, int ncols, const int *rowptr, const int *col, int *order);

/* P_r * A * P_c^T with rows sorted by new column; old_row = row_old[new_row],
 * new_col = col_new[old_col]. */
void tsgo_apply_bipermutation(int m, const int *rowptr, const int *col, const double *val,
                              const int *row_old, const int *col_new,
                              int *out_rowptr, int *out_col, double *out_val);


#ifdef __cplusplus
}
#endif

#endif
