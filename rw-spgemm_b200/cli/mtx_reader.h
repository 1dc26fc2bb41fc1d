// Matrix Market reader for the drop-in CLI.
//
// Semantics of the reference's mmio_allinone (src/mmio_highlevel.h:593-759):
// coordinate files only; symmetric and hermitian files are mirrored (off-
// diagonal entries stored twice); pattern entries read as 1.0, integer as
// their value, complex as the real part; duplicates are kept.  One difference,
// required by the GPU conversion: each row is sorted by column (stable).  For
// the usual column-major-sorted files the mirrored rows already come out
// sorted, so the CSR is identical to the reference reader's.
#pragma once

#include <string>
#include <vector>

struct MtxCSR
{
    int m = 0, n = 0, nnz = 0;
    int isSymmetric = 0;
    std::vector<int> rowptr, colidx;
    std::vector<double> val;
};

// Returns 0 on success, a negative code on failure (message in err).
int read_matrix_market(const char *path, MtxCSR *out, std::string *err);
