"""The drop-in CLI (rw-spgemm_b200/bin/test) with the reference's flags:
reports the same lines and passes its FP64 cuSPARSE cross-check."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "rw-spgemm_b200" / "bin" / "test"


def write_mtx(path, mat, symmetric_lower=False):
    m, n, rp, ci, v = mat
    rows = np.repeat(np.arange(m), np.diff(rp))
    keep = rows >= ci if symmetric_lower else np.ones(ci.size, bool)
    kind = "symmetric" if symmetric_lower else "general"
    order = np.lexsort((rows[keep], ci[keep]))
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {kind}\n% test\n{m} {n} {int(keep.sum())}\n")
        for r, c, x in zip(rows[keep][order], ci[keep][order], v[keep][order]):
            f.write(f"{r + 1} {c + 1} {x!r}\n")


def run(args):
    out = subprocess.run([str(BIN)] + args, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    return out.stdout


def expect_passed(text, nnzC):
    assert f"nnzC = {nnzC}\n" in text
    assert "[PASSED] nnzC" in text and "[PASSED] row_pointer" in text and "[PASSED] column_index & value" in text
    assert re.search(r"CUDA  TileSpGEMM runtime is [\d.]+ ms, gflops = [\d.]+", text)


def test_cli_aa_aat_ab(tmp_path, gen, oracle):
    a = gen.laplacian_2d(50, 37)
    pa = tmp_path / "lap.mtx"
    write_mtx(pa, a, symmetric_lower=True)
    G = oracle.gustavson(a, a)
    expect_passed(run(["-d", "0", "-aat", "0", str(pa)]), G[3].size)
    # A*A^T needs a non-symmetric file
    r = gen.random_poisson(300, 200, 5.0, seed=3)
    pr = tmp_path / "r.mtx"
    write_mtx(pr, r)
    txt = run(["-d", "0", "-aat", "1", str(pr)])
    expect_passed(txt, oracle.gustavson(r, gen.transpose(r))[3].size)
    b = gen.random_poisson(200, 150, 4.0, seed=5)
    pb = tmp_path / "b.mtx"
    write_mtx(pb, b)
    expect_passed(run(["-d", "0", "-aat", "0", str(pr), "-b", str(pb)]), oracle.gustavson(r, b)[3].size)
    assert "matrix AAT does not do symmetric matrix. Exit." in run(["-d", "0", "-aat", "1", str(pa)])


@pytest.mark.parametrize("algo", ["original", "rcm", "degree", "gray", "random"])
def test_cli_reorder(tmp_path, gen, oracle, algo):
    base = gen.stencil_27pt_3d(8, seed=1)
    a = gen.permute_symmetric(base, gen.random_symmetric_permutation(512, 3))
    p = tmp_path / "st.mtx"
    write_mtx(p, a, symmetric_lower=True)
    txt = run(["-d", "0", "-aat", "0", str(p), "-reorder", "1", "-reorder_algo", algo])
    assert f"reorder algorithm = {algo}" in txt and "estimated C tiles after reorder" in txt
    expect_passed(txt, oracle.gustavson(a, a)[3].size)


def test_cli_usage_and_tasa(tmp_path, gen):
    assert "Run the code by" in run(["-d", "0"])
    p = tmp_path / "x.mtx"
    write_mtx(p, gen.laplacian_2d(6), symmetric_lower=True)
    assert "reorder failed" in run(["-d", "0", "-aat", "0", str(p), "-reorder", "1"])
