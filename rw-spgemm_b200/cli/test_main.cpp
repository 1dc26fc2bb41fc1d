// Drop-in replacement of the reference CLI (src/main.cu:15-638):
//
//   ./test -d <dev> -aat <0|1> A.mtx [-b B.mtx] [-reorder 1] [-reorder_algo tasa|original|rcm|degree|gray|random]
//          [-o C.mtx]
//
// Same flags, same value overwrite (value[i] = i % 10, src/main.cu:191-197,
// applied in the reference reader's CSR order: rows in file order, columns
// unsorted, duplicates kept), same product modes (A*A, A*A^T, A*B) and the
// same stdout report lines, so the reference's batch scripts (which only
// redirect stdout) keep working.  After the overwrite each row is sorted and
// duplicate entries summed (canonicalize_rows), the form the library takes;
// the reported nnz and nnzCub are the reference's, counted with duplicates.
// -o (not in the reference) writes C, restored to the input order, as a
// Matrix Market file.
// Everything runs through the library's C ABI (include/tilespgemm_b200.h).
// The closing check compares the result with cuSPARSE in FP64 -- row
// pointers, columns and values (relative 1e-12) -- where the reference ran
// cuSPARSE with FP32 descriptors on FP64 data and compared structure only
// (src/external/cusparse/spgemm_cusparse.h:162-173, :282).
// -reorder_algo tasa (the default, as in the reference) runs the library's
// tile-aware planner build_reorder_plan (src/reorder.h:2407).
#include <cuda_runtime.h>
#include <cusparse.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <vector>

#include "mtx_reader.h"
#include "tilespgemm_b200.h"

static double now_ms()
{
    struct timeval t;
    gettimeofday(&t, NULL);
    return t.tv_sec * 1000.0 + t.tv_usec / 1000.0;
}

static void to_smatrix(MtxCSR &c, SMatrix *s)
{
    memset(s, 0, sizeof(*s));
    s->m = c.m;
    s->n = c.n;
    s->nnz = c.nnz;
    s->isSymmetric = c.isSymmetric;
    s->rowpointer = (int *)malloc(sizeof(int) * (c.m + 1));
    s->columnindex = (int *)malloc(sizeof(int) * (c.nnz ? c.nnz : 1));
    s->value = (double *)malloc(sizeof(double) * (c.nnz ? c.nnz : 1));
    memcpy(s->rowpointer, c.rowptr.data(), sizeof(int) * (c.m + 1));
    memcpy(s->columnindex, c.colidx.data(), sizeof(int) * c.nnz);
    memcpy(s->value, c.val.data(), sizeof(double) * c.nnz);
}

static void transpose_csr(const SMatrix *a, SMatrix *t)
{
    memset(t, 0, sizeof(*t));
    t->m = a->n;
    t->n = a->m;
    t->nnz = a->nnz;
    t->rowpointer = (int *)calloc(a->n + 1, sizeof(int));
    t->columnindex = (int *)malloc(sizeof(int) * (a->nnz ? a->nnz : 1));
    t->value = (double *)malloc(sizeof(double) * (a->nnz ? a->nnz : 1));
    for (int p = 0; p < a->nnz; p++)
        t->rowpointer[a->columnindex[p] + 1]++;
    for (int j = 0; j < a->n; j++)
        t->rowpointer[j + 1] += t->rowpointer[j];
    std::vector<int> cur(t->rowpointer, t->rowpointer + a->n);
    for (int r = 0; r < a->m; r++)
        for (int p = a->rowpointer[r]; p < a->rowpointer[r + 1]; p++)
        {
            int q = cur[a->columnindex[p]]++;
            t->columnindex[q] = r;
            t->value[q] = a->value[p];
        }
}

// C = A*B with cuSPARSE (FP64) and comparison against the tiled result.
static void cusparse_check(const SMatrix *A, const SMatrix *B, const SMatrix *C, unsigned long long nnzCub)
{
    printf("\n--------------- SpGEMM (using cuSPARSE) ---------------\n");
    cusparseHandle_t h;
    if (cusparseCreate(&h) != CUSPARSE_STATUS_SUCCESS)
    {
        printf("cuSPARSE failed!\n");
        return;
    }
    int *dAr, *dAc, *dBr, *dBc, *dCr;
    double *dAv, *dBv;
    cudaMalloc(&dAr, sizeof(int) * (A->m + 1));
    cudaMalloc(&dAc, sizeof(int) * (A->nnz ? A->nnz : 1));
    cudaMalloc(&dAv, sizeof(double) * (A->nnz ? A->nnz : 1));
    cudaMalloc(&dBr, sizeof(int) * (B->m + 1));
    cudaMalloc(&dBc, sizeof(int) * (B->nnz ? B->nnz : 1));
    cudaMalloc(&dBv, sizeof(double) * (B->nnz ? B->nnz : 1));
    cudaMalloc(&dCr, sizeof(int) * (A->m + 1));
    cudaMemcpy(dAr, A->rowpointer, sizeof(int) * (A->m + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(dAc, A->columnindex, sizeof(int) * A->nnz, cudaMemcpyHostToDevice);
    cudaMemcpy(dAv, A->value, sizeof(double) * A->nnz, cudaMemcpyHostToDevice);
    cudaMemcpy(dBr, B->rowpointer, sizeof(int) * (B->m + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(dBc, B->columnindex, sizeof(int) * B->nnz, cudaMemcpyHostToDevice);
    cudaMemcpy(dBv, B->value, sizeof(double) * B->nnz, cudaMemcpyHostToDevice);
    cusparseSpMatDescr_t mA, mB, mC;
    cusparseCreateCsr(&mA, A->m, A->n, A->nnz, dAr, dAc, dAv, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                      CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F);
    cusparseCreateCsr(&mB, B->m, B->n, B->nnz, dBr, dBc, dBv, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                      CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F);
    cusparseCreateCsr(&mC, A->m, B->n, 0, dCr, NULL, NULL, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                      CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F);
    double alpha = 1.0, beta = 0.0;
    cusparseSpGEMMDescr_t d;
    cusparseSpGEMM_createDescr(&d);
    size_t b1 = 0, b2 = 0;
    void *w1 = NULL, *w2 = NULL;
    const cusparseOperation_t op = CUSPARSE_OPERATION_NON_TRANSPOSE;
    double t0 = now_ms();
    cusparseSpGEMM_workEstimation(h, op, op, &alpha, mA, mB, &beta, mC, CUDA_R_64F, CUSPARSE_SPGEMM_DEFAULT, d, &b1, NULL);
    cudaMalloc(&w1, b1 ? b1 : 1);
    cusparseSpGEMM_workEstimation(h, op, op, &alpha, mA, mB, &beta, mC, CUDA_R_64F, CUSPARSE_SPGEMM_DEFAULT, d, &b1, w1);
    cusparseSpGEMM_compute(h, op, op, &alpha, mA, mB, &beta, mC, CUDA_R_64F, CUSPARSE_SPGEMM_DEFAULT, d, &b2, NULL);
    cudaMalloc(&w2, b2 ? b2 : 1);
    cusparseStatus_t cs =
        cusparseSpGEMM_compute(h, op, op, &alpha, mA, mB, &beta, mC, CUDA_R_64F, CUSPARSE_SPGEMM_DEFAULT, d, &b2, w2);
    int64_t r, c, nz;
    cusparseSpMatGetSize(mC, &r, &c, &nz);
    int *dCc;
    double *dCv;
    cudaMalloc(&dCc, sizeof(int) * (nz ? nz : 1));
    cudaMalloc(&dCv, sizeof(double) * (nz ? nz : 1));
    cusparseCsrSetPointers(mC, dCr, dCc, dCv);
    cusparseSpGEMM_copy(h, op, op, &alpha, mA, mB, &beta, mC, CUDA_R_64F, CUSPARSE_SPGEMM_DEFAULT, d);
    cudaDeviceSynchronize();
    double t = now_ms() - t0;
    printf(" - cuda SpGEMM completed!\n\n");
    const int nnzC = (int)nz;
    printf("nnzC = %i, nnzCub = %lld, Compression rate = %4.2f\n", nnzC, nnzCub,
           nnzC ? (double)nnzCub / nnzC : 0.0);
    printf("CUDA  cuSPARSE SpGEMM runtime is %4.4f ms, GFlops = %4.4f\n", t, t > 0 ? 2.0 * nnzCub / (1e6 * t) : 0.0);
    if (cs != CUSPARSE_STATUS_SUCCESS || (nnzC <= 0 && C->nnz > 0))
    {
        printf("cuSPARSE failed!\n");
    }
    else
    {
        printf("\nValidating results...\n");
        if (nnzC != C->nnz)
            printf("[NOT PASSED] nnzC = %i, nnzC_golden = %i\n", nnzC, C->nnz);
        else
            printf("[PASSED] nnzC = %i\n", nnzC);
        std::vector<int> hr(A->m + 1), hc(nz ? nz : 1);
        std::vector<double> hv(nz ? nz : 1);
        cudaMemcpy(hr.data(), dCr, sizeof(int) * (A->m + 1), cudaMemcpyDeviceToHost);
        cudaMemcpy(hc.data(), dCc, sizeof(int) * nz, cudaMemcpyDeviceToHost);
        cudaMemcpy(hv.data(), dCv, sizeof(double) * nz, cudaMemcpyDeviceToHost);
        int err = 0;
        for (int i = 0; i <= A->m; i++)
            err += hr[i] != C->rowpointer[i];
        if (err)
            printf("[NOT PASSED] row_pointer, #err = %i\n", err);
        else
            printf("[PASSED] row_pointer\n");
        err = 0;
        const int nmin = nnzC < C->nnz ? nnzC : C->nnz;
        for (int j = 0; j < nmin; j++)
        {
            const double ref = hv[j], got = C->value[j];
            const double rel = fabs(got - ref) / (fabs(ref) > 1e-300 ? fabs(ref) : 1e-300);
            if (hc[j] != C->columnindex[j] || (got != ref && rel > 1e-12))
                err++;
        }
        err += nnzC > C->nnz ? nnzC - C->nnz : C->nnz - nnzC;
        if (err)
            printf("[NOT PASSED] column_index & value, #err = %i (%4.2f%% #nnz)\n", err,
                   nnzC ? 100.0 * err / nnzC : 0.0);
        else
            printf("[PASSED] column_index & value\n");
    }
    cusparseSpGEMM_destroyDescr(d);
    cusparseDestroySpMat(mA);
    cusparseDestroySpMat(mB);
    cusparseDestroySpMat(mC);
    cusparseDestroy(h);
    cudaFree(w1);
    cudaFree(w2);
    cudaFree(dAr);
    cudaFree(dAc);
    cudaFree(dAv);
    cudaFree(dBr);
    cudaFree(dBc);
    cudaFree(dBv);
    cudaFree(dCr);
    cudaFree(dCc);
    cudaFree(dCv);
    printf("---------------------------------------------------------------\n");
}

// Scalar products of A*B counted over the CSR as read (duplicates included),
// the reference's nnzCub (src/main.cu:392-397); B given by its row lengths.
static unsigned long long count_products(const SMatrix *A, const std::vector<long long> &brow)
{
    unsigned long long s = 0;
    for (int i = 0; i < A->nnz; i++)
        s += (unsigned long long)brow[A->columnindex[i]];
    return s;
}

static void canonicalize(SMatrix *s)
{
    canonicalize_rows(s->m, s->rowpointer, s->columnindex, s->value);
    s->nnz = s->rowpointer[s->m];
}

static int write_mtx(const char *path, const SMatrix *C)
{
    FILE *f = fopen(path, "w");
    if (!f)
        return -1;
    fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%d %d %d\n", C->m, C->n, C->nnz);
    for (int r = 0; r < C->m; r++)
        for (int p = C->rowpointer[r]; p < C->rowpointer[r + 1]; p++)
            fprintf(f, "%d %d %.17g\n", r + 1, C->columnindex[p] + 1, C->value[p]);
    return fclose(f);
}

static const char *problem_name(ReorderProblemKind k)
{
    return k == REORDER_PROBLEM_AA ? "AA" : k == REORDER_PROBLEM_AAT ? "AAT" : "AB";
}

int main(int argc, char **argv)
{
    if (argc < 6)
    {
        printf("Run the code by './test -d 0 -aat 0 matrixA.mtx [-b matrixB.mtx] [-reorder 1] [-reorder_algo tasa|degree|rcm|...]'.\n");
        return 0;
    }
    printf("--------------------------------!!!!!!!!------------------------------------\n");
    int device_id = 0, aat = 0, reorder = 0, argi = 1;
    const char *reorder_algo = "tasa";
    if (strcmp(argv[argi++], "-d") != 0)
        return 0;
    device_id = atoi(argv[argi++]);
    printf("device_id = %i\n", device_id);
    cudaSetDevice(device_id);
    char name[256] = {0};
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device_id);
    strncpy(name, prop.name, sizeof(name) - 1);
    int clk_khz = 0;
    cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, device_id);
    printf("---------------------------------------------------------------\n");
    printf("Device [ %i ] %s @ %4.2f MHz\n", device_id, name, clk_khz * 1e-3f);
    if (strcmp(argv[argi++], "-aat") != 0)
        return 0;
    aat = atoi(argv[argi++]);
    char *filename = NULL, *filename_b = NULL, *filename_c = NULL;
    while (argi < argc)
    {
        if (!strcmp(argv[argi], "-reorder") || !strcmp(argv[argi], "-b") || !strcmp(argv[argi], "-reorder_algo") ||
            !strcmp(argv[argi], "-o"))
        {
            const char *flag = argv[argi++];
            if (argi >= argc)
            {
                printf("Missing value for %s.\n", flag);
                return 0;
            }
            if (!strcmp(flag, "-reorder"))
                reorder = atoi(argv[argi]);
            else if (!strcmp(flag, "-b"))
                filename_b = argv[argi];
            else if (!strcmp(flag, "-o"))
                filename_c = argv[argi];
            else
                reorder_algo = argv[argi];
            argi++;
        }
        else
            filename = argv[argi++];
    }
    if (!filename)
    {
        printf("Run the code by './test -d 0 -aat 0 matrixA.mtx [-b matrixB.mtx] [-reorder 1] [-reorder_algo tasa|degree|rcm|...]'.\n");
        return 0;
    }
    const int ab_mode = filename_b != NULL;
    printf("MAT A: -------------- %s --------------\n", filename);
    if (ab_mode)
        printf("MAT B: -------------- %s --------------\n", filename_b);

    MtxCSR ca, cb;
    std::string err;
    double t1 = now_ms();
    if (read_matrix_market(filename, &ca, &err) != 0)
    {
        printf("cannot read %s: %s\n", filename, err.c_str());
        return 0;
    }
    double t2 = now_ms();
    SMatrix A0, B0, *A = &A0, *B = &B0;
    to_smatrix(ca, &A0);
    printf("input matrix A: ( %i, %i ) nnz = %i\n loadfile time    = %4.5f sec\n", A0.m, A0.n, A0.nnz,
           (t2 - t1) / 1000.0);
    if (!aat && !ab_mode && A0.m != A0.n)
    {
        printf("matrix squaring must have rowA == colA. Exit.\n");
        return 0;
    }
    ReorderProblemKind kind = REORDER_PROBLEM_AA;
    if (ab_mode)
    {
        if (aat)
        {
            printf("explicit A*B mode does not support -aat 1. Exit.\n");
            return 0;
        }
        t1 = now_ms();
        if (read_matrix_market(filename_b, &cb, &err) != 0)
        {
            printf("cannot read %s: %s\n", filename_b, err.c_str());
            return 0;
        }
        t2 = now_ms();
        to_smatrix(cb, &B0);
        printf("input matrix B: ( %i, %i ) nnz = %i\n loadfile time    = %4.5f sec\n", B0.m, B0.n, B0.nnz,
               (t2 - t1) / 1000.0);
        if (A0.n != B0.m)
        {
            printf("A*B requires colA == rowB. Exit.\n");
            return 0;
        }
        kind = REORDER_PROBLEM_AB;
    }
    printf("the tilesize = %d\n", TSG_BLOCK_SIZE);
    for (int i = 0; i < A0.nnz; i++)
        A0.value[i] = i % 10;
    if (ab_mode)
    {
        for (int i = 0; i < B0.nnz; i++)
            B0.value[i] = i % 10;
    }
    else if (aat && A0.m == A0.n && A0.isSymmetric)
    {
        printf("matrix AAT does not do symmetric matrix. Exit.\n");
        return 0;
    }
    // the reference's nnzCub, over the CSR as read (it does not change under
    // the reorderings: a sum over A's entries of B's row lengths)
    std::vector<long long> brow;
    if (ab_mode)
        for (int k = 0; k < B0.m; k++)
            brow.push_back(B0.rowpointer[k + 1] - B0.rowpointer[k]);
    else if (aat)
    {
        brow.assign((size_t)A0.n, 0); // rows of A^T: A's column counts
        for (int i = 0; i < A0.nnz; i++)
            brow[A0.columnindex[i]]++;
    }
    else
        for (int k = 0; k < A0.m; k++)
            brow.push_back(A0.rowpointer[k + 1] - A0.rowpointer[k]);
    const unsigned long long nnzCub_read = count_products(&A0, brow);
    canonicalize(&A0);
    if (ab_mode)
        canonicalize(&B0);
    else if (aat)
    {
        transpose_csr(&A0, &B0);
        kind = REORDER_PROBLEM_AAT;
    }
    else
    {
        B0 = A0; // B aliases A's CSR (src/main.cu:230-241)
    }

    ReorderInfo info;
    reorder_info_init(&info);
    SMatrix Ar, Br;
    memset(&Ar, 0, sizeof(Ar));
    memset(&Br, 0, sizeof(Br));
    int materialized = 0, shared_csr = 0;
    double ordergen_ms = 0.0;
    if (reorder)
    {
        printf("reorder enabled\n");
        printf("reorder problem = %s\n", problem_name(kind));
        printf("reorder algorithm = %s\n", reorder_algo);
        printf("reorder strategy = %s\n", strcmp(reorder_algo, "tasa") == 0 ? "TASA-Fast-Unified" : "External-Order");
        t1 = now_ms();
        int st;
        if (!strcmp(reorder_algo, "tasa"))
        {
            ReorderProblem problem;
            problem.kind = kind;
            problem.matrixA = &A0;
            problem.matrixB = kind == REORDER_PROBLEM_AA ? &A0 : &B0;
            st = build_reorder_plan(&problem, &info);
            if (st)
            {
                printf("reorder failed, status = %d. Exit.\n", st);
                return 0;
            }
        }
        else if (!strcmp(reorder_algo, "original"))
        {
            st = build_original_reorder_plan(kind, &A0, kind == REORDER_PROBLEM_AA ? &A0 : &B0, &info);
            if (st)
            {
                printf("original reorder plan failed, status = %d. Exit.\n", st);
                return 0;
            }
        }
        else
        {
            st = build_external_reorder_plan(kind, reorder_algo, filename, filename_b, &A0,
                                             kind == REORDER_PROBLEM_AA ? &A0 : &B0, &info, &ordergen_ms);
            if (st)
            {
                printf("external reorder failed, status = %d. Exit.\n", st);
                return 0;
            }
        }
        if (info.guard_degraded_to_identity)
        {
            shared_csr = kind == REORDER_PROBLEM_AA;
        }
        else
        {
            double tp = now_ms();
            if (apply_bipermutation_csr(&A0, &info.row_perm, &info.inner_perm, &Ar))
            {
                printf("reorder apply A failed, status = %d. Exit.\n", -1);
                return 0;
            }
            if (kind == REORDER_PROBLEM_AA && info.shared_symmetric_csr)
            {
                Br = Ar;
                shared_csr = 1;
            }
            else if (apply_bipermutation_csr(kind == REORDER_PROBLEM_AA ? &A0 : &B0, &info.inner_perm, &info.col_perm,
                                              &Br))
            {
                printf("reorder apply B failed, status = %d. Exit.\n", -1);
                return 0;
            }
            info.permute_time_ms = now_ms() - tp;
            A = &Ar;
            B = &Br;
            materialized = 1;
        }
        info.reorder_time_ms = now_ms() - t1;
        printf("reorder time = %.2f ms\n", info.reorder_time_ms);
        printf("reorder mode = %s\n", info.mode);
        printf("reorder signature time = %.2f ms\n", info.signature_time_ms);
        printf("reorder tile profile time = %.2f ms\n", info.tile_profile_time_ms);
        printf("reorder affinity time = %.2f ms\n", info.affinity_time_ms);
        printf("reorder sort time = %.2f ms\n", info.sort_time_ms);
        printf("reorder local refine time = %.2f ms\n", info.local_refine_time_ms);
        printf("reorder local refine window = %d\n", info.local_refine_window);
        printf("reorder proxy time = %.2f ms\n", info.proxy_time_ms);
        printf("reorder proxy samples = %d\n", info.proxy_sample_rows);
        printf("reorder ordergen time = %.2f ms\n", ordergen_ms);
        printf("reorder permute time = %.2f ms\n", info.permute_time_ms);
        printf("reorder preprocess time = %.2f ms\n", ordergen_ms + info.permute_time_ms);
        printf("reorder shared csr = %d\n", shared_csr);
        printf("risk reason = %s\n", info.risk_reason);
        printf("risk input tile ratio = %.4f\n", info.risk_input_tile_ratio);
        printf("risk C tile ratio = %.4f\n", info.risk_c_tile_ratio);
        if (info.guard_degraded_to_identity)
            printf("reorder uses conservative identity\n");
        printf("input tiles A before reorder = %lld\n", info.input_tiles_A_before);
        printf("input tiles A after reorder = %lld\n", info.input_tiles_A_after);
        printf("input tiles B before reorder = %lld\n", info.input_tiles_B_before);
        printf("input tiles B after reorder = %lld\n", info.input_tiles_B_after);
        printf("estimated C tiles before reorder = %lld\n", info.estimated_c_tiles_before);
        printf("estimated C tiles after reorder = %lld\n", info.estimated_c_tiles_after);
    }

    const unsigned long long nnzCub = nnzCub_read;
    printf("SpGEMM nnzCub = %lld\n", nnzCub);

    // tile format: A row-major (packed bytes), B column-major (its own copy
    // of the CSR arrays, which csr2tile_col_major leaves untouched)
    SMatrix At = *A, Bt = *B;
    t1 = now_ms();
    csr2tile_row_major(&At);
    t2 = now_ms();
    printf("CSR to Tile conversion uses %.2f ms\n", t2 - t1);
    double tile_bytes = (At.tilem + 1) * 4.0 + At.numtile * 4.0 + (At.numtile + 1) * 4.0 + At.nnz * 8.0 +
                        At.nnz * 1.0 + At.numtile * 16.0 + At.numtile * 16.0 * 2.0;
    printf("tile space overhead = %.2f MB\n", tile_bytes / 1024 / 1024);
    csr2tile_col_major(&Bt);

    // the driver's intersection bitmaps and densities (src/main.cu:430-465),
    // handed to tilespgemm like the reference does (which ignores them)
    unsigned int *bmA = NULL, *bmB = NULL;
    int bmlen = 0;
    if (tile_intersection_bitmaps(&At, &Bt, &bmA, &bmB, &bmlen) != 0)
    {
        printf("intersection bitmaps failed: %s. Exit.\n", tsg_last_error());
        return 0;
    }
    const double densA = (double)At.numtile / ((double)At.tilem * (double)At.tilen);
    const double densB = (double)Bt.numtile / ((double)Bt.tilem * (double)Bt.tilen);
    SMatrix C;
    memset(&C, 0, sizeof(C));
    unsigned long long nnzC = 0;
    double cr = 0, ttile = 0, gf = 0, s1 = 0, s2 = 0, s3 = 0, sm = 0;
    tilespgemm(&At, &Bt, &C, bmA, bmB, bmlen, densA, densB, nnzCub, &nnzC, &cr, &ttile, &gf, filename, &s1, &s2,
               &s3, &sm);
    free(bmA);
    free(bmB);

    printf("-------------------------------check----------------------------------------\n");
    tile2csr(&C);
    printf("tile to CSR conversion complete!\n");
    if (materialized)
    {
        t1 = now_ms();
        int st = restore_bipermutation_csr(&C, &info.row_perm, &info.col_perm);
        if (st)
        {
            printf("restore reorder result failed, status = %d. Exit.\n", st);
            return 0;
        }
        printf("restore reorder result uses %.2f ms\n", now_ms() - t1);
    }
    if (filename_c && write_mtx(filename_c, &C) != 0)
        printf("cannot write %s\n", filename_c);
    cusparse_check(&A0, &B0, &C, nnzCub);
    matrix_destroy(&At);
    matrix_destroy(&Bt);
    free(Bt.tile_rowidx);
    free(Bt.csc_tile_ptr);
    free(Bt.csc_tile_rowidx);
    free(At.tile_rowidx);
    matrix_destroy(&C);
    free(C.tile_rowidx);
    free(C.rowpointer);
    free(C.columnindex);
    free(C.value);
    if (reorder)
        reorder_info_destroy(&info);
    return 0;
}
