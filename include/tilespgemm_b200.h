/*
 * tilespgemm_b200.h -- C ABI of the B200 (sm_100a) tiled SpGEMM library.
 *
 * Two layers are exported by libtilespgemm_b200.so:
 *
 *  1. Drop-in entry points with the exact signatures, struct layouts and
 *     ownership rules of the TileSpGEMM reference (for-the-juan/RW-SpGEMM).
 *     Each declaration names the reference function it replaces (file:line).
 *     All of them take HOST buffers, run the work on the current CUDA device
 *     and return host arrays that the caller frees (matrix_destroy / free).
 *
 *  2. A handle API (tsg_*) over device-resident tiled matrices.  Every pointer
 *     inside tsg_tiled is a DEVICE pointer owned by the library; status codes
 *     are returned instead of printing.  Batching, serving and the benchmarks
 *     are built on this layer.
 *
 * Tile format (16x16 tiles, identical to the reference's SMatrix):
 *   tile_ptr[tilem+1]       tiles of each tile row (row-major tile order)
 *   tile_columnidx[T]       tile column of each tile, ascending within a row
 *   tile_rowidx[T]          tile row of each tile
 *   tile_nnz[T+1]           exclusive scan of nonzeros per tile (value offsets)
 *   tile_csr_Ptr[16T]       per-tile, per-row offset (uint8) of the row's first
 *                           nonzero; rows past the matrix edge hold the tile nnz
 *   tile_csr_Col[nnz]       in-tile column byte; (row<<4)|col for a row-major
 *                           "A" operand, plain col for B and C
 *   tile_csr_Value[nnz]     FP64 values, row-major inside the tile
 *   mask[16T]               per-row 16-bit mask, bit (15-col) set per nonzero
 *   csc_tile_ptr/rowidx     column-major tile view (B operand)
 */
#ifndef TILESPGEMM_B200_H
#define TILESPGEMM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TSG_BLOCK_SIZE 16

/* ------------------------------------------------------------------------ */
/* Layer 1: drop-in surface of the reference                                */
/* ------------------------------------------------------------------------ */

/* Matrix container; field order and types identical to src/common.h:113-135
 * (MAT_VAL_TYPE = double, MAT_PTR_TYPE = int) so that callers compiled
 * against the reference header link unchanged. */
#ifndef SMATRIX
#define SMATRIX
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
} SMatrix;
#endif

/* CSR -> row-major tiles with packed (row<<4)|col bytes.
 * Replaces csr2tile_row_major, src/csr2tile.h:196-259.
 * Reads m, n, nnz, rowpointer, columnindex, value; mallocs and fills tilem,
 * tilen, numtile, tile_ptr, tile_columnidx, tile_rowidx, tile_nnz,
 * tile_csr_Ptr, tile_csr_Col, tile_csr_Value, mask.  Rows must be sorted by
 * strictly increasing column; any input error is printed and aborts the
 * process (the reference function returns void and has no error path). */
void csr2tile_row_major(SMatrix *matrix);

/* CSR -> tiles stored in column-major tile order with in-tile CSR and plain
 * column bytes, plus the row-major tile_ptr/tile_columnidx used by step 1.
 * Replaces csr2tile_col_major, src/csr2tile.h:261-478. */
void csr2tile_col_major(SMatrix *matrix);

/* The reference driver's intersection bitmaps (src/main.cu:430-465), built on
 * the GPU: len = ceil(A->tilen / 32); A's tile row i sets bit (31 - j % 32) of
 * word i * len + j / 32 for each of its tile columns j (tile_ptr,
 * tile_columnidx of csr2tile_row_major); B's tile column i the same for each
 * of its tile rows (csc_tile_ptr, csc_tile_rowidx of csr2tile_col_major).
 * *bitmask_A (tilem x len words) and *bitmask_B (B->tilen x len) are
 * malloc'd, the caller frees them.  Returns 0 or a TSG_ERR_* code. */
int tile_intersection_bitmaps(const SMatrix *A, const SMatrix *B, unsigned int **bitmask_A,
                              unsigned int **bitmask_B, int *bitmask_len);

/* Tiled SpGEMM C = A*B.  A from csr2tile_row_major, B from
 * csr2tile_col_major.  Replaces tilespgemm, src/tilespgemm-cuda.h:2610-2624.
 * The intersection bitmaps (tile_intersection_bitmaps above) and the
 * densities are accepted for ABI compatibility and IGNORED: this
 * implementation's steps read A's and B's tile columns, masks and column
 * view directly instead of intersecting bitmaps.  Runs the product REPEAT (5) times,
 * reports the minimum time of the reference's window (C allocation through
 * the numeric step), and fills matrixC's host tile arrays (tile_ptr,
 * tile_columnidx, tile_rowidx, tile_nnz, tile_csr_Ptr, tile_csr_Col,
 * tile_csr_Value, mask, numtile, nnz, m, n, tilem, tilen). */
void tilespgemm(SMatrix *matrixA,
                SMatrix *matrixB,
                SMatrix *matrixC,
                unsigned int *blk_intersec_bitmask_A,
                unsigned int *blk_intersec_bitmask_B,
                int blk_intersec_bitmask_len,
                double densityA,
                double densityB,
                unsigned long long int nnzCub,
                unsigned long long int *nnzC_computed,
                double *compression_rate,
                double *time_tile,
                double *gflops_tile,
                char *filename,
                double *time_step1, double *time_step2, double *time_step3, double *time_malloc);

/* Tiles -> CSR with ascending columns; zeros are kept.
 * Replaces tile2csr, src/tile2csr.h:71-137. */
void tile2csr(SMatrix *matrix);

/* Frees the tile arrays (and only those), src/csr2tile.h:481-492. */
void matrix_destroy(SMatrix *matrix);

/* Reordering types, src/reorder.h:26-77 (field order kept). */
typedef struct
{
    int n;
    int *old_id; /* new id -> original id */
    int *new_id; /* original id -> new id */
} AxisPermutation;

typedef struct
{
    int enabled;
    int n;
    AxisPermutation row_perm;
    AxisPermutation inner_perm;
    AxisPermutation col_perm;
    long long input_tiles_A_before;
    long long input_tiles_A_after;
    long long input_tiles_B_before;
    long long input_tiles_B_after;
    long long estimated_c_tiles_before;
    long long estimated_c_tiles_after;
    double reorder_time_ms;
    double signature_time_ms;
    double tile_profile_time_ms;
    double affinity_time_ms;
    double sort_time_ms;
    double local_refine_time_ms;
    double proxy_time_ms;
    double permute_time_ms;
    double risk_input_tile_ratio;
    double risk_c_tile_ratio;
    int local_refine_window;
    int proxy_sample_rows;
    int guard_degraded_to_identity;
    int structural_conservative;
    int shared_symmetric_csr;
    char mode[64];
    char risk_reason[128];
} ReorderInfo;

typedef enum
{
    REORDER_PROBLEM_AA = 0,
    REORDER_PROBLEM_AAT = 1,
    REORDER_PROBLEM_AB = 2
} ReorderProblemKind;

/* src/reorder.h:72-77 (field order kept). */
typedef struct
{
    ReorderProblemKind kind;
    const SMatrix *matrixA;
    const SMatrix *matrixB; /* AA: may be matrixA or NULL; AAT: A's transpose */
} ReorderProblem;

void reorder_info_init(ReorderInfo *info);
void reorder_info_destroy(ReorderInfo *info);

/* The tile-aware planner (TASA, the CLI's default -reorder_algo); replaces
 * build_reorder_plan, src/reorder.h:2407-2428, with the same plans, modes,
 * risk guard and return codes (0, or -1 bad problem / non-square AA, -2.. on
 * failure).  A*A of a symmetric matrix (isSymmetric): identity for n <=
 * 50,000 with < 32 tiles per tile row, reverse Cuthill-McKee refined in
 * windows of 32 for other n <= 50,000, windowed packing into 16-row groups
 * above; general A*A, A*B and A*A^T: every axis sorted by tile signatures
 * (computed on the GPU).  Environment: TASA_FORCE_ACTIVE=1 accepts any plan,
 * TASA_AB_SHARED_SYM=1 lets A*B of two symmetric matrices use the symmetric
 * plan. */
int build_reorder_plan(const ReorderProblem *problem, ReorderInfo *info);

/* Identity plan; replaces build_original_reorder_plan,
 * src/external_reorder.h:173-202.  Returns 0 or a negative code. */
int build_original_reorder_plan(ReorderProblemKind kind,
                                const SMatrix *matrixA,
                                const SMatrix *matrixB,
                                ReorderInfo *info);

/* Named ordering computed on the GPU ("original", "rcm", "degree", "gray",
 * "random"); replaces build_external_reorder_plan,
 * src/external_reorder.h:204-321, which ran reorder_algorithm/<algo>/order_gen
 * in a child process.  The matrix paths are accepted and unused (the order is
 * computed from matrixA / matrixB in memory); ordergen_ms receives the GPU
 * ordering time.  AA/AAT apply A's order to all three axes; AB uses A's order
 * for rows and inner axis and B's order for the column axis.  Returns 0, or
 * -20 for an algorithm this library does not provide (the reference's return
 * for an order generator that did not run, src/external_reorder.h:133). */
int build_external_reorder_plan(ReorderProblemKind kind,
                                const char *algorithm,
                                const char *matrix_path_A,
                                const char *matrix_path_B,
                                const SMatrix *matrixA,
                                const SMatrix *matrixB,
                                ReorderInfo *info,
                                double *ordergen_ms);

/* output = P_row * input * P_col^T in CSR with sorted rows (GPU).
 * Replaces apply_bipermutation_csr, src/reorder.h:2429-2504. */
int apply_bipermutation_csr(const SMatrix *input,
                            const AxisPermutation *row_perm,
                            const AxisPermutation *col_perm,
                            SMatrix *output);

/* Un-permutes rows and columns of a CSR matrix in place, rows re-sorted
 * (GPU).  Replaces restore_bipermutation_csr, src/reorder.h:2506-2551. */
int restore_bipermutation_csr(SMatrix *matrix,
                              const AxisPermutation *row_perm,
                              const AxisPermutation *col_perm);

/* ------------------------------------------------------------------------ */
/* Layer 2: handle API over device-resident tiled matrices                  */
/* ------------------------------------------------------------------------ */

typedef enum
{
    TSG_OK = 0,
    TSG_ERR_INVALID = -1,     /* bad argument                          */
    TSG_ERR_CUDA = -2,        /* CUDA runtime error                    */
    TSG_ERR_OOM = -3,         /* device allocation failed              */
    TSG_ERR_INPUT = -4,       /* malformed CSR (range, order, ptr)     */
    TSG_ERR_OVERFLOW = -5,    /* result exceeds 32-bit offsets / cap   */
    TSG_ERR_UNSUPPORTED = -6, /* feature not provided                  */
    TSG_ERR_TIMEOUT = -7,     /* a bounded device wait gave up         */
    TSG_ERR_REJECTED = -8     /* admission refused (memory cap)        */
} tsg_status;

/* Flags for tsg_csr_to_tiled. */
#define TSG_TILED_PACKED_COL 1 /* A operand: Col bytes are (row<<4)|col    */
#define TSG_TILED_CSC_VIEW 2   /* B operand: build the column-major view   */

typedef struct tsg_context tsg_context;

/* Device-resident tiled matrix.  Tile data is stored in row-major tile order;
 * the optional column view lists, per tile column, the tile rows
 * (csc_tile_rowidx) and the row-major tile index (csc_tile_pos) of each tile.
 * Matrices converted for the B role (TSG_TILED_CSC_VIEW) also carry a row
 * view: the same matrix as scalar CSR (row_ptr[m+1], row_col[nnz],
 * row_val[nnz]), read by the numeric step of TSG_SCHED_SPA.
 * All pointers are device pointers owned by the library. */
typedef struct
{
    int m, n, nnz;
    int tilem, tilen, numtile;
    int col_packed;
    int *tile_ptr;
    int *tile_columnidx;
    int *tile_rowidx;
    int *tile_nnz;
    unsigned char *tile_csr_Ptr;
    unsigned char *tile_csr_Col;
    double *tile_csr_Value;
    unsigned short *mask;
    int *csc_tile_ptr;
    int *csc_tile_rowidx;
    int *csc_tile_pos;
    unsigned short *mask_t; /* B operand: per tile column masks, bit (15-row) */
    int *row_ptr;           /* B operand: row view (scalar CSR)             */
    int *row_col;
    double *row_val;
    void *_alloc;           /* internal: non-NULL marks a borrowed view      */
} tsg_tiled;

/* Per-product statistics filled by tsg_spgemm. */
typedef struct
{
    long long numtile_C;
    long long nnz_C;
    long long nnzCub;     /* scalar products, sum over A nonzeros of |B row| */
    long long tile_pairs; /* matched (A tile, B tile) pairs                   */
    double ms_step1, ms_step2, ms_step3, ms_total;
    int bins[4];          /* C tiles by nnz: <=32, <=224, <256, ==256         */
    int step3_kernel;     /* numeric step that ran: TSG_STEP3_*               */
} tsg_spgemm_info;

/* tsg_spgemm_info.step3_kernel */
#define TSG_STEP3_NONE 0   /* C has no nonzeros                               */
#define TSG_STEP3_TILES 1  /* k_step3: half-warp per C tile                   */
#define TSG_STEP3_ELEMS 2  /* k_step3_elems: warp per C tile, per element     */
#define TSG_STEP3_ROWS 3   /* k_step3_rows: half-warp per run of C tiles      */
#define TSG_STEP3_FLAT 4   /* k_step3_spa<flat>: SPA, CTA per C tile block    */
#define TSG_STEP3_SPA 5    /* k_step3_spa: SPA, CTA per tile-row segment      */
#define TSG_STEP3_STAGED 6 /* k_step3_stg + k_step3_rest: SPA with operands
                            * staged in shared memory by bulk copies          */

const char *tsg_status_string(int status);
/* Message describing the last failure on the calling thread. */
const char *tsg_last_error(void);

int tsg_context_create(int device, tsg_context **ctx);
int tsg_context_destroy(tsg_context *ctx);
/* Use an existing cudaStream_t (passed as void*) for all work; NULL = the
 * context's own stream again.  For the legacy default stream pass
 * cudaStreamLegacy, not 0. */
int tsg_context_set_stream(tsg_context *ctx, void *cuda_stream);
/* Work schedule of steps 2 and 3 (results are bit-identical either way):
 * TSG_SCHED_TILES  one half-warp per C tile, intersecting A's tile row with
 *                  B's tile column (the reference's decomposition);
 * TSG_SCHED_ROWS   one half-warp per run of seg_tiles C tiles of one tile
 *                  row, walking A's tile row and B's tile rows (no
 *                  intersection search), accumulating into acc_cap FP64
 *                  shared-memory slots.  seg_tiles in {8, 16}; acc_cap in
 *                  {256, 512, 1024, 2048}. */
#define TSG_SCHED_TILES 0
#define TSG_SCHED_ROWS 1
/* TSG_SCHED_ELEMS  step 2 as TILES; step 3 with one warp per C tile and one
 *                  lane per C nonzero, accumulating across matched tile pairs
 *                  through A's row masks and B's column masks (register
 *                  accumulator, no shared-memory scatter). */
#define TSG_SCHED_ELEMS 2
/* TSG_SCHED_SPA    step 2 as TILES; step 3 as a row Gustavson over B's row
 *                  view (scalar CSR): a CTA per run of C tiles of one tile
 *                  row, a warp per C row, products accumulated in shared
 *                  memory in C's tiled layout.  B without a row view runs
 *                  TSG_SCHED_TILES. */
#define TSG_SCHED_SPA 3
int tsg_context_set_schedule(tsg_context *ctx, int schedule, int seg_tiles, int acc_cap);
/* TSG_SCHED_SPA: a product whose C tiles hold at least values_per_tile
 * values on average (nnz(C) / tiles(C), known after step 2) runs the numeric
 * step with the tile kernel instead of the sparse accumulator; 0 restores
 * the default (64); 257 never switches.  Results are identical either way. */
int tsg_context_set_dense_threshold(tsg_context *ctx, int values_per_tile);
/* 1 (default): step-1 emit and step 2 run as one row-wise pass for tile rows
 * with at most 128 C tiles (others fall back to step 2 per tile); 0: separate
 * step 2 of the schedule.  Results are identical. */
int tsg_context_set_fusion(tsg_context *ctx, int fuse_step12);
/* 0 when all work queued on the context's stream has finished, 1 while
 * some is pending, a negative status on error (non-blocking). */
int tsg_context_query(tsg_context *ctx);
/* Blocks until all work queued on the context's stream has finished; returns
 * an error a kernel recorded in the context's device status word since the
 * last check (TSG_ERR_TIMEOUT: a bounded wait gave up; TSG_ERR_OVERFLOW: an
 * accumulator bound was exceeded) and clears it. */
int tsg_context_synchronize(tsg_context *ctx);
/* Number of this library's kernels launched on the context so far. */
long long tsg_context_launches(tsg_context *ctx);
/* Number of device allocations the library made on the context so far (its
 * stream-ordered pool requests; no reference counterpart). */
long long tsg_context_allocations(tsg_context *ctx);
/* Record per-step CUDA-event timings into tsg_spgemm_info. */
int tsg_context_set_timing(tsg_context *ctx, int enabled);

/* GPU CSR -> tiles.  d_rowptr/d_colidx/d_val are device pointers; rows must
 * be sorted by strictly increasing column.  flags: TSG_TILED_* above. */
int tsg_csr_to_tiled(tsg_context *ctx, int m, int n, int nnz,
                     const int *d_rowptr, const int *d_colidx, const double *d_val,
                     int flags, tsg_tiled *out);

/* Upload a host tiled matrix produced by csr2tile_row_major (role A) or
 * csr2tile_col_major (role B: column-major data, identity csc_tile_pos). */
int tsg_tiled_upload_rowmajor(tsg_context *ctx, const SMatrix *host, tsg_tiled *out);
int tsg_tiled_upload_colmajor(tsg_context *ctx, const SMatrix *host, tsg_tiled *out);

int tsg_tiled_free(tsg_context *ctx, tsg_tiled *mat);
/* Device bytes the library holds for a tiled matrix: every array present,
 * as allocated (16-byte rounding plus 16 bytes of slack each); 0 for a
 * borrowed view.  For admission control (no reference counterpart). */
long long tsg_tiled_device_bytes(const tsg_tiled *mat);
/* Bytes in use in the device's default stream-ordered memory pool, from
 * which the library allocates (cudaMemPoolAttrUsedMemCurrent). */
int tsg_context_pool_used(tsg_context *ctx, unsigned long long *bytes);

/* C = A*B on the device.  A needs col_packed tiles (row role), B needs the
 * column view.  C is allocated by the library (row-major, plain Col bytes,
 * masks set, no column view). */
int tsg_spgemm(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B,
               tsg_tiled *C, tsg_spgemm_info *info);

/* Tiles -> CSR into caller-provided device buffers: d_rowptr[m+1],
 * d_colidx[nnz], d_val[nnz]. */
int tsg_tiled_to_csr(tsg_context *ctx, const tsg_tiled *C,
                     int *d_rowptr, int *d_colidx, double *d_val);

/* Tiles -> CSR with no allocation at all (no counterpart in the reference;
 * its tile2csr, src/tile2csr.h:71, is a host conversion).  Same outputs as
 * tsg_tiled_to_csr.  The row-pointer scan keeps its block sums in a fixed
 * file-scope device array of 4096 entries (32 KB per device) instead of
 * taking them from the context's memory pool, so C may have at most
 * 4096 * 8192 = 33,554,432 rows; larger C returns TSG_ERR_INVALID before
 * anything is launched.  For callers that must not allocate here: those that
 * have handed all device memory to their own fixed arena or admission budget
 * (the pool would grow behind it), and those on a path where a pool growth,
 * which can synchronise the device, is not allowed.
 *   - Nothing in the scratch has to start at zero: each call writes every
 *     block sum it reads.
 *   - The scratch is one per device, shared by all contexts, streams and
 *     threads: calls that may overlap on one device race on it; order them
 *     (same stream, or an event between them).
 *   - The scratch address is looked up (cudaGetSymbolAddress) when a context
 *     is created on the device, so the call itself makes no runtime call but
 *     its launches; after a cudaDeviceReset create a new context. */
int tsg_tiled_to_csr_noalloc(tsg_context *ctx, const tsg_tiled *C,
                             int *d_rowptr, int *d_colidx, double *d_val);

/* Copy a device tiled matrix into host arrays of an SMatrix (malloc'd,
 * caller frees).  colmajor != 0 writes B's reference layout (column-major
 * tile data, plain Col bytes, csc_tile_ptr/csc_tile_rowidx). */
int tsg_tiled_download(tsg_context *ctx, const tsg_tiled *src, int colmajor, SMatrix *dst);

/* End to end with HOST buffers: CSR A (m x k) times CSR B (k x n) -> CSR C.
 * Copies inputs to the device, converts, multiplies, converts back and copies
 * the result to freshly malloc'd host arrays (*c_rowptr, *c_colidx, *c_val;
 * caller frees).  B may alias A. */
int tsg_spgemm_csr_host(tsg_context *ctx,
                        int m, int k, int n,
                        int nnzA, const int *a_rowptr, const int *a_colidx, const double *a_val,
                        int nnzB, const int *b_rowptr, const int *b_colidx, const double *b_val,
                        int *nnzC, int **c_rowptr, int **c_colidx, double **c_val,
                        tsg_spgemm_info *info);

/* GPU orderings of the rows of a CSR matrix, written to d_order as a
 * new -> old permutation (reorder_algorithm/README.md:6-12 convention):
 * TSG_ORDER_ORIGINAL identity; TSG_ORDER_RCM reverse Cuthill-McKee on the
 * symmetrised pattern with (degree, id) tie-break (square only);
 * TSG_ORDER_DEGREE by (-degree, id); TSG_ORDER_GRAY by (density group,
 * Gray-decoded column signature, id); TSG_ORDER_RANDOM the permutation of
 * Python's random.Random(seed).shuffle(list(range(m))), bit for bit (made on
 * the host: one sequential chain of draws).  Replaces the order_gen adapters of
 * reorder_algorithm/{original,rcm,degree,gray,random}/ (run through
 * src/external_reorder.h:100-141). */
#define TSG_ORDER_ORIGINAL 0
#define TSG_ORDER_RCM 1
#define TSG_ORDER_DEGREE 2
#define TSG_ORDER_GRAY 3
#define TSG_ORDER_RANDOM 4
int tsg_order(tsg_context *ctx, int kind, int m, int n, int nnz,
              const int *d_rowptr, const int *d_col, unsigned long long seed, int *d_order);
/* A plan's tile-count estimates for the permutations already in info
 * (row_perm, inner_perm, col_perm): input_tiles_{A,B}_{before,after},
 * estimated_c_tiles_{before,after} and the two risk ratios, computed as the
 * reference's plans compute them (src/external_reorder.h:143-171): sampled
 * over 24 evenly strided tile rows and scaled (src/reorder.h:785-975), on the
 * host.  build_original_reorder_plan and build_external_reorder_plan fill
 * them the same way.  No reference counterpart as a public call (the
 * reference's fill_reorder_estimates is file-local). */
int tsg_reorder_estimates(ReorderProblemKind kind, const SMatrix *matrixA, const SMatrix *matrixB,
                          ReorderInfo *info);
/* TSG_ORDER_RANDOM's permutation written to host memory (no device work):
 * order[0..n) = random.Random(seed).shuffle(list(range(n))) of CPython. */
int tsg_order_random_host(int n, unsigned long long seed, int *order);
/* "original", "rcm", "degree", "gray", "random" -> TSG_ORDER_*, else -1. */
int tsg_order_from_name(const char *name);

/* Device bipermutation: out = P_row * A * P_col^T with rows sorted by column;
 * output row r is input row d_row_old[r], column c becomes d_col_new[c].
 * Output arrays are caller-allocated (m+1, nnz, nnz).  The device form of
 * apply_bipermutation_csr, src/reorder.h:2429-2504. */
int tsg_permute_csr(tsg_context *ctx, int m, int n, int nnz,
                    const int *d_rowptr, const int *d_col, const double *d_val,
                    const int *d_row_old, const int *d_col_new,
                    int *d_out_rowptr, int *d_out_col, double *d_out_val);

/* As tsg_spgemm_csr_host; with TSG_HOST_PINNED_OUTPUT in flags the three
 * output arrays are page-locked host memory (faster device->host copies),
 * released with tsg_host_free instead of free. */
#define TSG_HOST_PINNED_OUTPUT 1
int tsg_spgemm_csr_host_ex(tsg_context *ctx,
                           int m, int k, int n,
                           int nnzA, const int *a_rowptr, const int *a_colidx, const double *a_val,
                           int nnzB, const int *b_rowptr, const int *b_colidx, const double *b_val,
                           int *nnzC, int **c_rowptr, int **c_colidx, double **c_val,
                           tsg_spgemm_info *info, int flags);
void tsg_host_free(void *p);

/* Two-phase end-to-end call for callers that own their output buffers
 * (e.g. reused page-locked buffers): _start copies the host CSR inputs to the
 * device and computes C there (as CSR), returning nnz(C); tsg_result_copy
 * copies it into rowptr[m+1], colidx[nnzC], val[nnzC]; tsg_result_free
 * releases the device result. */
typedef struct tsg_result tsg_result;
int tsg_spgemm_csr_host_start(tsg_context *ctx,
                              int m, int k, int n,
                              int nnzA, const int *a_rowptr, const int *a_colidx, const double *a_val,
                              int nnzB, const int *b_rowptr, const int *b_colidx, const double *b_val,
                              tsg_result **res, int *nnzC, tsg_spgemm_info *info);
int tsg_result_copy(tsg_result *res, int *rowptr, int *colidx, double *val);
int tsg_result_free(tsg_result *res);

/* One end-to-end call into caller-owned host buffers: C = A*B (B may alias
 * A's arrays) lands in c_rowptr[m+1], c_colidx[nnz_cap], c_val[nnz_cap],
 * with the device-to-host copy overlapping the numeric step -- C's row
 * pointer is final after the symbolic steps and goes out first; then the
 * tile rows of C are computed and converted in chunks on the context's
 * stream while earlier chunks are copied out on a second stream.  The
 * buffers should be page-locked (pageable memory is correct but the copies
 * then serialise).  When nnz(C) > nnz_cap nothing but *nnzC is written and
 * TSG_ERR_OVERFLOW is returned: grow the buffers (tsg_product_bounds gives
 * an upper bound) and call again.  Synchronous.  No reference counterpart:
 * the reference returns C through tilespgemm (src/tilespgemm-cuda.h:2610)
 * and tile2csr (src/tile2csr.h:71), in sequence. */
int tsg_spgemm_csr_host_into(tsg_context *ctx,
                             int m, int k, int n,
                             int nnzA, const int *a_rowptr, const int *a_colidx, const double *a_val,
                             int nnzB, const int *b_rowptr, const int *b_colidx, const double *b_val,
                             int *c_rowptr, int *c_colidx, double *c_val, long long nnz_cap,
                             int *nnzC, tsg_spgemm_info *info);

/* Host CSR -> device tiles in one call (copies through pooled device memory;
 * the host arrays may be pageable or pinned). */
int tsg_csr_host_to_tiled(tsg_context *ctx, int m, int n, int nnz,
                          const int *h_rowptr, const int *h_colidx, const double *h_val,
                          int flags, tsg_tiled *out);
/* Device tiles -> host CSR; arrays allocated like tsg_spgemm_csr_host_ex
 * (TSG_HOST_PINNED_OUTPUT: page-locked, release with tsg_host_free). */
int tsg_tiled_to_csr_host(tsg_context *ctx, const tsg_tiled *C, int flags,
                          int **rowptr, int **colidx, double **val);

/* Upper bounds of one product from the tile structure alone: scalar
 * products (= nnzCub >= nnz(C)) and matched tile pairs (>= C tiles). */
int tsg_product_bounds(tsg_context *ctx, const tsg_tiled *A, const tsg_tiled *B,
                       long long *products, long long *tile_pairs);
/* The same for count products A[p]*B[p] with one synchronisation; c_tiles
 * (may be NULL) receives each product's exact number of C tiles (step 1's
 * count pass). */
int tsg_product_bounds_many(tsg_context *ctx, int count, const tsg_tiled *A, const tsg_tiled *B,
                            long long *products, long long *tile_pairs, long long *c_tiles);

/* ------------------------------------------------------------------------ */
/* Batched products: many independent C_p = A_p * B_p of uneven size run in  */
/* one persistent, cooperatively launched kernel captured in a CUDA graph.   */
/* ------------------------------------------------------------------------ */
typedef struct
{
    int schedule;  /* TSG_SCHED_TILES or TSG_SCHED_ROWS                  */
    int seg_tiles; /* row schedule: C tiles per work item                */
    int acc_cap;   /* row schedule: FP64 accumulator slots per half-warp */
    int use_graph; /* capture the launch in a CUDA graph                 */
    int dense_threshold; /* TSG_SCHED_SPA: C values per tile from which a
                          * product takes the tile kernel (0: 64)       */
} tsg_batch_params;

typedef struct tsg_batch tsg_batch;

/* Plans a batch over count device-resident operand pairs (A[p] row tiles,
 * B[p] with column view; they must stay alive), computes per-product upper
 * bounds on the device, allocates one result arena and captures the launch.
 * params NULL = row schedule (16, 1024) with a graph. */
int tsg_batch_create(tsg_context *ctx, int count, const tsg_tiled *A, const tsg_tiled *B,
                     const tsg_batch_params *params, tsg_batch **out);
/* tsg_batch_create with the bounds already known (products and c_tiles of
 * tsg_product_bounds_many, one entry per product): plans without running a
 * kernel or waiting for the device, so a caller can form the next batch
 * while another stream's batch holds the GPU.  Smaller bounds than the true
 * ones make the run fail with TSG_ERR_OVERFLOW. */
int tsg_batch_create_bounded(tsg_context *ctx, int count, const tsg_tiled *A, const tsg_tiled *B,
                             const tsg_batch_params *params, const long long *products,
                             const long long *c_tiles, tsg_batch **out);
/* Queues one execution of the whole batch on the context's stream. */
int tsg_batch_run(tsg_batch *b);
/* Waits for the last run and reads per-product sizes; reports a device wait
 * that gave up (TSG_ERR_TIMEOUT) or an exceeded bound (TSG_ERR_OVERFLOW). */
int tsg_batch_sync(tsg_batch *b, long long *total_tiles, long long *total_nnz);
/* View of product p's result inside the arena (valid until the next run or
 * destroy; tsg_tiled_free on it only clears the struct). */
int tsg_batch_product(tsg_batch *b, int p, tsg_tiled *C);
int tsg_batch_info(tsg_batch *b, int *graph, int *grid, size_t *arena_bytes, long long *launches);
/* Duration (ms, GPU global timer) of each of the seven phases of the last
 * finished run: step-1 counts, C row-pointer scans, work-item prefixes,
 * step-1 emit + fused step 2, step 2 of the remaining tiles, tile-count scans,
 * numeric step. */
int tsg_batch_phase_ms(tsg_batch *b, double *ms);
/* Sets how long (seconds) a block of the batch kernel waits at its grid
 * barrier before it gives up, sets TSG_ERR_TIMEOUT for tsg_batch_sync and
 * leaves (the batch stays usable: the next run starts clean).  The default
 * is 2 s plus 10 ns per scalar product of the whole batch.  A graph captured
 * at creation reads the limit from device memory, so it applies to it too.
 * No reference counterpart (the reference has no batched path). */
int tsg_batch_set_wait_limit(tsg_batch *b, double seconds);
int tsg_batch_destroy(tsg_batch *b);

/* ------------------------------------------------------------------------ */
/* Learned selector: row statistics of a device CSR and a small FP32 MLP     */
/* (F -> H -> H -> O, ReLU) trained and evaluated by hand-written kernels.   */
/* ------------------------------------------------------------------------ */
#define TSG_NFEAT_RAW 24
/* out[0] sum of row lengths, [1] sum of squares, [2] max length, [3] sum of
 * |i-j|, [4] max |i-j|, [5] empty rows, [6..17] row-length histogram
 * (0, 1, 2-3, 4-7, ..., >= 1024), [18] entries with |i-j| < 16. */
int tsg_row_features(tsg_context *ctx, int m, const int *d_rowptr, const int *d_col,
                     unsigned long long *h_out);

typedef struct tsg_mlp tsg_mlp;
/* F <= 32 inputs, H <= 64 hidden units (two layers), O <= 32 outputs; He
 * initialisation from seed. */
int tsg_mlp_create(tsg_context *ctx, int F, int H, int O, unsigned long long seed, tsg_mlp **out);
int tsg_mlp_destroy(tsg_mlp *m);
int tsg_mlp_num_params(const tsg_mlp *m);
/* One forward + backward (masked mean squared error) + Adam step on a device
 * minibatch of B <= 64 rows: X[B][F], T[B][O], M[B][O] (NULL = all 1).
 * lr <= 0 only computes the gradients (read them with tsg_mlp_get(m, 1, .)).
 * *loss receives the minibatch loss before the update (NULL: no sync). */
int tsg_mlp_train_step(tsg_mlp *m, int B, const float *d_X, const float *d_T, const float *d_M,
                       float lr, float *loss);
/* Y[n][O] = network(X[n][F]), device arrays. */
int tsg_mlp_forward(tsg_mlp *m, int n, const float *d_X, float *d_Y);
/* which = 0 parameters, 1 last gradients; layout W1[F][H] b1 W2[H][H] b2
 * W3[H][O] b3, row-major. */
int tsg_mlp_get(tsg_mlp *m, int which, float *host);
int tsg_mlp_set(tsg_mlp *m, const float *host);

/* Scalar product count nnzCub = sum over A nonzeros (i,k) of nnz(B row k),
 * computed on the device from device CSR arrays. */
int tsg_count_products(tsg_context *ctx, int nnzA, const int *d_a_colidx,
                       const int *d_b_rowptr, long long *nnzCub);

#ifdef __cplusplus
}
#endif

#endif /* TILESPGEMM_B200_H */
