/*
 * Reference CPU code, compiled from the reference's own sources -- TEST
 * INFRASTRUCTURE ONLY (oracle/Makefile builds it into oracle/_ref/ when the
 * reference tree is present).  Nothing here is restated: the headers of
 * for-the-juan/RW-SpGEMM are included as they are and wrapped in extern "C"
 * entry points for ctypes.  The only change made around them is the one the
 * reference's own CPU oracle needs to run at all: spgemm_cpu reads A's packed
 * (row<<4)|col byte as a column (src/spgemm-cpu.h:231,:324), so the wrapper
 * hands it a copy of A with the bytes unpacked (col & 0xf).
 */
#include "common.h"
#include "utils.h"
#include "csr2tile.h"
#include "tile2csr.h"
#include "spgemm-cpu.h"
#include "spgemm_serialref_spa_new.h"

extern "C" {

void ref_csr2tile_row_major(SMatrix *m) { csr2tile_row_major(m); }

void ref_csr2tile_col_major(SMatrix *m) { csr2tile_col_major(m); }

void ref_tile2csr(SMatrix *m) { tile2csr(m); }

void ref_spgemm_cpu(SMatrix *A, SMatrix *B, SMatrix *C)
{
    unsigned char *packed = A->tile_csr_Col;
    unsigned char *plain = (unsigned char *)malloc(A->nnz > 0 ? A->nnz : 1);
    for (int i = 0; i < A->nnz; i++)
        plain[i] = packed[i] & 0xf;
    A->tile_csr_Col = plain;
    spgemm_cpu(A, B, C);
    A->tile_csr_Col = packed;
    free(plain);
}

/* Symbolic SPA: row pointers (pass 1) and column indices (pass 2). */
int ref_spgemm_spa_rowptr(int mA, int nA, int nnzA, const int *rpA, const int *ciA,
                          int mB, int nB, int nnzB, const int *rpB, const int *ciB,
                          int *rpC)
{
    int nnzC = 0;
    spgemm_spa(rpA, ciA, NULL, mA, nA, nnzA, rpB, ciB, NULL, mB, nB, nnzB,
               rpC, NULL, NULL, mA, nB, &nnzC, 1);
    return nnzC;
}

void ref_spgemm_spa_cols(int mA, int nA, int nnzA, const int *rpA, const int *ciA,
                         int mB, int nB, int nnzB, const int *rpB, const int *ciB,
                         int *rpC, int *ciC)
{
    int nnzC = 0;
    spgemm_spa(rpA, ciA, NULL, mA, nA, nnzA, rpB, ciB, NULL, mB, nB, nnzB,
               rpC, ciC, NULL, mA, nB, &nnzC, 0);
}

void ref_free(void *p) { free(p); }

int ref_omp_max_threads(void) { return omp_get_max_threads(); }
}
