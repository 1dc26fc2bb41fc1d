/*
 * The reference's reorder-plan estimators, compiled from its own sources --
 * TEST INFRASTRUCTURE ONLY (oracle/Makefile builds it into oracle/_ref/ when
 * the reference tree is given).  Nothing here is restated: src/reorder.h and
 * src/external_reorder.h of for-the-juan/RW-SpGEMM are included as they are
 * (they need nvcc for their thrust kernels) and their host functions wrapped
 * in extern "C" entry points for ctypes: the sampled input-tile and C-tile
 * estimates (src/reorder.h:785-975), the plan's estimate fill
 * (src/external_reorder.h:143-171), the original-order plan (:173-202) and
 * the tile-aware planner build_reorder_plan (src/reorder.h:2407-2428; its
 * general-matrix plans run thrust kernels, so they need a GPU).
 */
#include "common.h"
#include "reorder.h"
#include "external_reorder.h"

extern "C" {

long long ref_est_input_tiles(const SMatrix *m, const AxisPermutation *row, const AxisPermutation *col)
{
    return estimate_input_tile_count_biperm(m, row, col);
}

long long ref_est_c_tiles(const SMatrix *m, const AxisPermutation *row, const AxisPermutation *inner,
                          const AxisPermutation *col)
{
    return estimate_symbolic_c_tile_count(m, row, inner, col);
}

long long ref_est_c_tiles_ab(const SMatrix *a, const SMatrix *b, const AxisPermutation *row,
                             const AxisPermutation *inner, const AxisPermutation *col)
{
    return estimate_symbolic_c_tile_count_ab(a, b, row, inner, col);
}

void ref_fill_reorder_estimates(int kind, const SMatrix *a, const SMatrix *b, ReorderInfo *info)
{
    fill_reorder_estimates((ReorderProblemKind)kind, a, b, info);
}

int ref_build_original_reorder_plan(int kind, const SMatrix *a, const SMatrix *b, ReorderInfo *info)
{
    return build_original_reorder_plan((ReorderProblemKind)kind, a, b, info);
}

int ref_build_reorder_plan(int kind, const SMatrix *a, const SMatrix *b, ReorderInfo *info)
{
    ReorderProblem problem;
    problem.kind = (ReorderProblemKind)kind;
    problem.matrixA = a;
    problem.matrixB = b;
    return build_reorder_plan(&problem, info);
}

void ref_reorder_info_init(ReorderInfo *info) { reorder_info_init(info); }

void ref_reorder_info_destroy(ReorderInfo *info) { reorder_info_destroy(info); }
}
