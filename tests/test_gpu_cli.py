"""The drop-in CLI (rw-spgemm_b200/bin/test) with the reference's flags:
reports the same lines and passes its FP64 cuSPARSE cross-check; values are
overwritten (i % 10) in the reference reader's order and duplicate entries
computed as the reference computes them."""
import os
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


def run(args, env=None):
    out = subprocess.run([str(BIN)] + args, capture_output=True, text=True, timeout=300,
                         env=dict(os.environ, **(env or {})))
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
    args = ["-d", "0", "-aat", "0", str(p), "-reorder", "1", "-reorder_algo", algo]
    if algo == "random":
        # as the reference's adapter: refused unless TASA_ENABLE_UNSAFE_RANDOM=1
        txt = run(args, env={"TASA_ENABLE_UNSAFE_RANDOM": "0"})
        assert "external reorder missing dependency: random" in txt
        assert "external reorder failed, status = -20. Exit." in txt
    txt = run(args, env={"TASA_ENABLE_UNSAFE_RANDOM": "1"})
    assert f"reorder algorithm = {algo}" in txt and "estimated C tiles after reorder" in txt
    expect_passed(txt, oracle.gustavson(a, a)[3].size)


def write_scrambled(path, entries, m, n, symmetric=False):
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {'symmetric' if symmetric else 'general'}\n"
                f"{m} {n} {len(entries)}\n")
        for r, c in entries:
            f.write(f"{r + 1} {c + 1} 0.5\n")


def reference_read(entries, m, n, symmetric=False):
    """The reference reader's CSR (src/mmio_highlevel.h:593-759: rows grouped
    in file order, a mirrored entry placed when its original is read,
    columns unsorted, duplicates kept) with the CLI's value[i] = i % 10
    (src/main.cu:191-197), then each row sorted and duplicates summed --
    the matrix the reference's product computes with."""
    rows = [[] for _ in range(m)]
    for r, c in entries:
        rows[r].append(c)
        if symmetric and r != c:
            rows[c].append(r)
    val, p = [], 0
    out_rp, out_ci, out_v = [0], [], []
    for r in range(m):
        acc = {}
        for c in rows[r]:
            acc[c] = acc.get(c, 0.0) + float(p % 10)
            p += 1
        for c in sorted(acc):
            out_ci.append(c)
            out_v.append(acc[c])
        out_rp.append(len(out_ci))
    return (m, n, np.array(out_rp, np.int32), np.array(out_ci, np.int32), np.array(out_v)), p


def read_c(path):
    with open(path) as f:
        f.readline()
        m, n, nnz = (int(x) for x in f.readline().split())
        a = np.loadtxt(f, ndmin=2) if nnz else np.zeros((0, 3))
    rows = a[:, 0].astype(np.int64) - 1
    rp = np.zeros(m + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    return np.cumsum(rp), a[:, 1].astype(np.int32) - 1, a[:, 2]


def _scrambled_entries(rng, m, n, count, dups, lower=False):
    ents = set()
    while len(ents) < count:
        r, c = int(rng.integers(0, m)), int(rng.integers(0, n))
        if lower and c > r:
            r, c = c, r
        ents.add((r, c))
    ents = sorted(ents)
    ents += [ents[int(i)] for i in rng.integers(0, len(ents), dups)]   # duplicate entries
    rng.shuffle(ents)                                                  # file order not sorted
    return [tuple(e) for e in ents]


@pytest.mark.parametrize("mode", ["AA", "AA-symmetric", "AAT", "AB", "AB-reorder", "AAT-reorder"])
def test_cli_values_in_file_order_with_duplicates(tmp_path, oracle, mode):
    rng = np.random.default_rng(sum(map(ord, mode)))
    n = 300
    sym = mode == "AA-symmetric"
    ea = _scrambled_entries(rng, n, n, 1500, 40, lower=sym)
    pa = tmp_path / "a.mtx"
    write_scrambled(pa, ea, n, n, symmetric=sym)
    A, nnz_read = reference_read(ea, n, n, symmetric=sym)
    args = ["-d", "0", "-aat", "1" if mode.startswith("AAT") else "0", str(pa), "-o", str(tmp_path / "c.mtx")]
    if mode.startswith("AB"):
        eb = _scrambled_entries(rng, n, n, 1200, 30)
        pb = tmp_path / "b.mtx"
        write_scrambled(pb, eb, n, n)
        B, _ = reference_read(eb, n, n)
        args += ["-b", str(pb)]
    elif mode.startswith("AAT"):
        import scipy.sparse as sp
        T = sp.csr_matrix((A[4], A[3], A[2]), shape=(n, n)).T.tocsr()
        T.sort_indices()
        B = (n, n, T.indptr.astype(np.int32), T.indices.astype(np.int32), T.data)
    else:
        B = A
    if mode.endswith("reorder"):
        args += ["-reorder", "1", "-reorder_algo", "rcm" if mode.startswith("AB") else "degree"]
    txt = run(args)
    assert f"nnz = {nnz_read}\n" in txt                     # counted as read, duplicates included
    G = oracle.gustavson(A, B)
    expect_passed(txt, G[3].size)
    rp, ci, v = read_c(tmp_path / "c.mtx")
    np.testing.assert_array_equal(rp, G[2])
    np.testing.assert_array_equal(ci, G[3])
    np.testing.assert_array_equal(v, G[4])                   # small integers: exact


def test_cli_usage_and_tasa(tmp_path, gen, oracle):
    assert "Run the code by" in run(["-d", "0"])
    p = tmp_path / "x.mtx"
    lap = gen.laplacian_2d(6)
    write_mtx(p, lap, symmetric_lower=True)
    txt = run(["-d", "0", "-aat", "0", str(p), "-reorder", "1"])        # tasa: the reference's default
    assert "reorder algorithm = tasa" in txt and "reorder strategy = TASA-Fast-Unified" in txt
    assert "reorder mode = identity_narrow_tiles" in txt and "reorder uses conservative identity" in txt
    expect_passed(txt, oracle.gustavson(lap, lap)[3].size)
    # a general (unsymmetric) file: the signature plan on the GPU, A*A and A*B
    g = gen.random_poisson(700, 700, 6.0, seed=2)
    b = gen.random_poisson(700, 500, 4.0, seed=3)
    pg, pb = tmp_path / "g.mtx", tmp_path / "b.mtx"
    write_mtx(pg, g)
    write_mtx(pb, b)
    txt = run(["-d", "0", "-aat", "0", str(pg), "-reorder", "1", "-reorder_algo", "tasa"])
    assert re.search(r"reorder mode = (active_general|conservative_identity)\n", txt)
    expect_passed(txt, oracle.gustavson(g, g)[3].size)
    txt = run(["-d", "0", "-aat", "0", str(pg), "-b", str(pb), "-reorder", "1"])
    assert re.search(r"reorder mode = (active_ab|conservative_identity)\n", txt)
    expect_passed(txt, oracle.gustavson(g, b)[3].size)
