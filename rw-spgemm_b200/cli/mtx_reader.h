// Matrix Market reader for the drop-in CLI.
//
// Semantics of the reference's mmio_allinone (src/mmio_highlevel.h:593-759):
// coordinate files only; symmetric and hermitian files are mirrored (off-
// diagonal entries stored twice); pattern entries read as 1.0, integer as
// their value, complex as the real part.  The CSR comes out in the same order
// as the reference's: entries grouped by row in file order (a mirrored entry
// goes to its row when its original is read), columns within a row NOT
// sorted and duplicates kept.  canonicalize_rows then gives the form the
// library takes (each row sorted by column, duplicates summed).
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

// In place: every row sorted by column (stable) and entries of one column
// merged into one whose value is their sum, added in their order in the row.
// The reference keeps duplicates and its kernels add every entry's products
// into C, which gives the same sums in exact arithmetic (and bit for bit for
// its CLI's integer values, value[i] = i % 10).  Returns the number of
// entries removed.
long long canonicalize_rows(int m, int *rowptr, int *colidx, double *val);
