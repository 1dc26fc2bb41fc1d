"""Regenerates tests/golden/orders.npz from the REFERENCE's own ordering code
(for-the-juan/RW-SpGEMM reorder_algorithm/common/order_utils.py: native_original,
native_degree, native_rcm, and native_random under TASA_RANDOM_SEED 1 and 7),
run in this container on small Matrix Market files written from the library's
generators.

Run where the reference tree exists:
    python tests/golden/make_golden_orders.py <reference tree>
"""
from __future__ import annotations

import importlib.util
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
if len(sys.argv) != 2:
    sys.exit("usage: make_golden_orders.py <reference tree (holds reorder_algorithm/common/order_utils.py)>")
REF_UTILS = Path(sys.argv[1]) / "reorder_algorithm" / "common" / "order_utils.py"
if not REF_UTILS.is_file():
    sys.exit(f"{REF_UTILS} not found")
sys.path.insert(0, str(HERE.parent))
from conftest import load_package  # noqa: E402


def write_mtx(path, mat, symmetric_lower=False):
    m, n, rp, ci, v = mat
    rows = np.repeat(np.arange(m), np.diff(rp))
    keep = rows >= ci if symmetric_lower else np.ones(ci.size, bool)
    kind = "symmetric" if symmetric_lower else "general"
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {kind}\n{m} {n} {int(keep.sum())}\n")
        order = np.lexsort((rows[keep], ci[keep]))  # column-major, as SuiteSparse files
        for r, c, x in zip(rows[keep][order], ci[keep][order], v[keep][order]):
            f.write(f"{r + 1} {c + 1} {x!r}\n")


def cases(g):
    return {
        "lap12": (g.laplacian_2d(12, 10), True),
        "st27_6": (g.stencil_27pt_3d(6, seed=1), True),
        "pois_sym": (g.permute_symmetric(g.banded(90, 3, seed=3), g.random_symmetric_permutation(90, 5)), True),
        "pois": (g.random_poisson(120, None, 3.0, seed=6), False),
        "rmat7": (g.rmat(7, 4, seed=2), False),
    }


def main():
    spec = importlib.util.spec_from_file_location("ref_order_utils", REF_UTILS)
    ou = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ou)
    load_package()
    import rw_spgemm_b200.generators as g

    out = {}
    with tempfile.TemporaryDirectory() as td:
        for name, (mat, sym) in cases(g).items():
            mtx = Path(td) / f"{name}.mtx"
            write_mtx(mtx, mat, symmetric_lower=sym)
            m, n, rp, ci, v = mat
            out[f"{name}/m"] = np.array([m, n])
            out[f"{name}/rowptr"], out[f"{name}/colidx"], out[f"{name}/val"] = rp, ci, v
            for kind in ("original", "degree", "rcm"):
                of = Path(td) / f"{name}.{kind}"
                rc = ou.run_native(kind, ["order_gen", str(mtx), str(of)])
                assert rc == 0, (name, kind, rc)
                out[f"{name}/{kind}"] = np.loadtxt(of, dtype=np.int64).astype(np.int32).reshape(-1)
            for seed in (1, 7):
                os.environ["TASA_RANDOM_SEED"] = str(seed)
                of = Path(td) / f"{name}.random{seed}"
                rc = ou.run_native("random", ["order_gen", str(mtx), str(of)])
                assert rc in (0, None), (name, "random", rc)
                out[f"{name}/random{seed}"] = np.loadtxt(of, dtype=np.int64).astype(np.int32).reshape(-1)
    np.savez_compressed(HERE / "orders.npz", **out)
    print("wrote", HERE / "orders.npz", sorted({k.split('/')[0] for k in out}))


if __name__ == "__main__":
    main()
