"""Regenerates the golden fixtures in this directory from the REFERENCE's own
CPU code (for-the-juan/RW-SpGEMM src/csr2tile.h, src/tile2csr.h,
src/spgemm-cpu.h, src/spgemm_serialref_spa_new.h), compiled from its sources
by oracle/Makefile into oracle/_ref/libtsgref.so.

Run where the reference tree exists:  python tests/golden/make_golden.py
Outputs (committed, small):
  cases.npz          per-case CSR inputs and the reference's outputs
  known_answers.json scalar facts for the benchmark-sized inputs
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
from conftest import load_oracle, load_package  # noqa: E402

TILE_KEYS = ["tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col",
             "tile_csr_Value", "mask"]


def small_cases(g):
    return {
        "lap8": g.overwrite_values_mod10(g.laplacian_2d(8)),
        "lap37x29": g.laplacian_2d(37, 29),
        "band100": g.banded(100, 5, seed=4),
        "rmat7": g.rmat(7, 6, seed=11),
        "pois_rect": g.random_poisson(45, 61, 5.0, seed=9),
        "pois_sq": g.random_poisson(96, None, 4.0, seed=2),
    }


def main():
    o = load_oracle()
    o.build()
    if not o.ref_available():
        raise SystemExit("reference build missing: oracle/_ref/libtsgref.so")
    load_package()
    import rw_spgemm_b200.generators as g

    arrays = {}
    for name, mat in small_cases(g).items():
        m, n, rp, ci, v = mat
        arrays[f"{name}/m"] = np.array([m, n], dtype=np.int64)
        arrays[f"{name}/rowptr"] = rp
        arrays[f"{name}/colidx"] = ci
        arrays[f"{name}/val"] = v
        A = o.ref_csr2tile_row_major(mat)
        for k in TILE_KEYS:
            arrays[f"{name}/A/{k}"] = A[k]
        B = o.ref_csr2tile_col_major(mat)
        for k in TILE_KEYS + ["csc_tile_ptr", "csc_tile_rowidx"]:
            arrays[f"{name}/B/{k}"] = B[k]
        if m == n:
            srp, sci = o.ref_spgemm_spa(mat, mat)
            arrays[f"{name}/C/rowptr"] = srp
            arrays[f"{name}/C/colidx"] = sci
            if n % 16 == 0:  # spgemm_cpu's count pass is only consistent for n % 16 == 0
                C = o.ref_spgemm_cpu(A, B)
                for k in ["tile_ptr", "tile_columnidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col",
                          "tile_csr_Value"]:
                    arrays[f"{name}/Ct/{k}"] = C[k]
                rp2, ci2, v2 = o.ref_tile2csr(C)
                arrays[f"{name}/C/val"] = v2
    np.savez_compressed(HERE / "cases.npz", **arrays)

    facts = {"generator": "rw-spgemm_b200/generators.py", "source": "reference CPU code via oracle/_ref"}
    for name, mat in [("laplacian_64x64", g.laplacian_2d(64)), ("laplacian_256x256", g.laplacian_2d(256)),
                      ("stencil27_64", g.stencil_27pt_3d(64, seed=0))]:
        m, n, rp, ci, v = mat
        A = o.ref_csr2tile_row_major(mat)
        srp, sci = o.ref_spgemm_spa(mat, mat)
        f = {"n": int(n), "nnzA": int(ci.size), "tilesA": int(A["numtile"]), "nnzC": int(srp[-1]),
             "products": int(o.count_products(mat, mat))}
        if name.startswith("laplacian"):
            C = o.ref_spgemm_cpu(A, o.ref_csr2tile_col_major(mat))
            f["tilesC"] = int(C["numtile"])
            f["tilesC_nonempty"] = int(np.count_nonzero(np.diff(C["tile_nnz"])))
            crp, cci, cv = o.ref_tile2csr(C)
            f["row0_cols"] = cci[crp[0]:crp[1]].tolist()
            f["row0_vals"] = cv[crp[0]:crp[1]].tolist()
        else:
            B = o.ref_csr2tile_col_major(mat)
            f["tilesC"] = int(o.spgemm_tiled(o.csr2tile_row_major(mat), o.csr2tile_col_major(mat))["numtile"])
            f["tilesB_colmajor"] = int(B["numtile"])
        facts[name] = f
    (HERE / "known_answers.json").write_text(json.dumps(facts, indent=1) + "\n")
    print(json.dumps(facts, indent=1))


if __name__ == "__main__":
    main()
