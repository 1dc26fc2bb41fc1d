"""Seeded synthetic sparse matrices (CSR, int32 indices, FP64 values, rows
sorted, no duplicates) standing in for the SuiteSparse inputs of the
reference's experiments.

Every generator returns ``(m, n, rowptr, colidx, val)`` as numpy arrays.
"""
from __future__ import annotations

import numpy as np


def _coo_to_csr(m, n, rows, cols, vals):
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = np.asarray(vals, dtype=np.float64)[order]
    keep = np.ones(key.size, dtype=bool)
    keep[1:] = key[1:] != key[:-1]  # duplicates merged: first value kept
    key = key[keep]
    vals = vals[keep]
    r = (key // n).astype(np.int64)
    c = (key % n).astype(np.int32)
    rowptr = np.zeros(m + 1, dtype=np.int64)
    np.add.at(rowptr, r + 1, 1)
    rowptr = np.cumsum(rowptr).astype(np.int32)
    return m, n, rowptr, c, vals


def laplacian_2d(nx: int, ny: int | None = None):
    """5-point Laplacian on an nx x ny grid: 4 on the diagonal, -1 off it."""
    ny = nx if ny is None else ny
    n = nx * ny
    idx = np.arange(n, dtype=np.int64)
    x, y = idx % nx, idx // nx
    rows, cols, vals = [idx], [idx], [np.full(n, 4.0)]
    for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        ok = (x + dx >= 0) & (x + dx < nx) & (y + dy >= 0) & (y + dy < ny)
        rows.append(idx[ok])
        cols.append(idx[ok] + dx + dy * nx)
        vals.append(np.full(int(ok.sum()), -1.0))
    return _coo_to_csr(n, n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def stencil_27pt_3d(nx: int, seed: int = 0, low: float = 0.5, high: float = 1.5):
    """27-point stencil on an nx^3 grid, values uniform(low, high)."""
    n = nx ** 3
    idx = np.arange(n, dtype=np.int64)
    x, y, z = idx % nx, (idx // nx) % nx, idx // (nx * nx)
    rows, cols = [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ok = ((x + dx >= 0) & (x + dx < nx) & (y + dy >= 0) & (y + dy < nx)
                      & (z + dz >= 0) & (z + dz < nx))
                rows.append(idx[ok])
                cols.append(idx[ok] + dx + dy * nx + dz * nx * nx)
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    m, n_, rp, ci, _ = _coo_to_csr(n, n, rows, cols, np.zeros(rows.size))
    rng = np.random.default_rng(seed)
    return m, n_, rp, ci, rng.uniform(low, high, ci.size)


def rmat(scale: int, edge_factor: int, a=0.57, b=0.19, c=0.19, seed: int = 1,
         low: float = -1.0, high: float = 1.0):
    """R-MAT graph: 2^scale vertices, edge_factor * 2^scale edges drawn by
    per-level quadrant choice with probabilities (a, b, c, 1-a-b-c);
    duplicates merged; values uniform(low, high)."""
    n = 1 << scale
    ne = edge_factor * n
    rng = np.random.default_rng(seed)
    rows = np.zeros(ne, dtype=np.int64)
    cols = np.zeros(ne, dtype=np.int64)
    ab, abc = a + b, a + b + c
    for level in range(scale):
        u = rng.random(ne)
        bit = 1 << (scale - 1 - level)
        down = u >= ab            # quadrants c, d
        right = ((u >= a) & (u < ab)) | (u >= abc)   # quadrants b, d
        rows += down * bit
        cols += right * bit
    m, n_, rp, ci, _ = _coo_to_csr(n, n, rows, cols, np.zeros(ne))
    return m, n_, rp, ci, rng.uniform(low, high, ci.size)


def banded(n: int, half_bandwidth: int, seed: int = 0, low=-1.0, high=1.0):
    """Full band |i-j| <= half_bandwidth, values uniform(low, high); built
    directly in CSR order."""
    i = np.arange(n, dtype=np.int64)
    start = np.maximum(i - half_bandwidth, 0)
    stop = np.minimum(i + half_bandwidth, n - 1)
    lens = stop - start + 1
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=rp[1:])
    pos = np.arange(int(rp[-1]), dtype=np.int64)
    ci = (np.repeat(start - rp[:-1], lens) + pos).astype(np.int32)
    rng = np.random.default_rng(seed)
    return n, n, rp.astype(np.int32), ci, rng.uniform(low, high, ci.size)


def random_poisson(m: int, n: int | None = None, lam: float = 8.0, seed: int = 0, low=-1.0, high=1.0):
    """Each row draws Poisson(lam) uniform random columns (duplicates merged)."""
    n = m if n is None else n
    rng = np.random.default_rng(seed)
    per = rng.poisson(lam, m)
    rows = np.repeat(np.arange(m, dtype=np.int64), per)
    cols = rng.integers(0, n, rows.size)
    mm, nn, rp, ci, _ = _coo_to_csr(m, n, rows, cols, np.zeros(rows.size))
    return mm, nn, rp, ci, rng.uniform(low, high, ci.size)


def random_symmetric_permutation(n: int, seed: int = 7):
    """new -> old permutation (numpy default_rng(seed).permutation)."""
    return np.random.default_rng(seed).permutation(n).astype(np.int32)


def permute_symmetric(mat, order):
    """P A P^T for a new->old order; rows re-sorted."""
    m, n, rp, ci, v = mat
    order = np.asarray(order, dtype=np.int64)
    new_of_old = np.empty(n, dtype=np.int64)
    new_of_old[order] = np.arange(n)
    lens = np.diff(rp)
    rows_old = np.repeat(np.arange(m), lens)
    return _coo_to_csr(m, n, new_of_old[rows_old], new_of_old[ci], v)


def transpose(mat):
    m, n, rp, ci, v = mat
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(rp))
    return _coo_to_csr(n, m, ci, rows, v)


def overwrite_values_mod10(mat):
    """value[i] = i % 10 by CSR position, as the reference CLI does before
    computing (src/main.cu:191-197)."""
    m, n, rp, ci, _ = mat
    return m, n, rp, ci, (np.arange(ci.size) % 10).astype(np.float64)


def products(matA, matB) -> int:
    """nnzCub: sum over A's nonzeros (i, k) of nnz(B row k) (src/main.cu:392-397)."""
    _, _, _, ci, _ = matA
    _, _, rpB, _, _ = matB
    return int(np.diff(rpB.astype(np.int64))[ci].sum())


def batched_products(count: int = 512, seed: int = 0, n_min: int = 1024, n_max: int = 65536,
                     hb_min: int = 8, hb_max: int = 64, lam: float = 8.0):
    """Independent square products C_i = A_i * B_i: n_i log-uniform in
    [n_min, n_max]; each of A_i, B_i banded (half-bandwidth uniform in
    [hb_min, hb_max]) or random with Poisson(lam) nonzeros per row; values
    uniform(-1, 1); a fixed seed per product."""
    out = []
    for n, sides in _batched_specs(count, seed, n_min, n_max, hb_min, hb_max):
        out.append(tuple(banded(n, p, seed=s) if kind == "banded" else random_poisson(n, None, lam, seed=s)
                         for kind, p, s in sides))
    return out


def _batched_specs(count, seed, n_min, n_max, hb_min, hb_max):
    """(n, [(kind, half-bandwidth, seed) for A, B]) of every product of
    batched_products, drawn from one generator in a fixed order."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        sides = []
        for side in range(2):
            s = int(rng.integers(0, 2**31 - 1))
            if rng.random() < 0.5:
                sides.append(("banded", int(rng.integers(hb_min, hb_max + 1)), s))
            else:
                sides.append(("poisson", 0, s))
        specs.append((n, sides))
    return specs


def batched_product_classes(count: int = 512, seed: int = 0, n_min: int = 1024, n_max: int = 65536,
                            hb_min: int = 8, hb_max: int = 64):
    """Class of each product of batched_products(count, seed, ...):
    "banded*banded", "poisson*poisson" (sparse C tiles, hypersparse for large
    n) or "mixed"."""
    out = []
    for _, sides in _batched_specs(count, seed, n_min, n_max, hb_min, hb_max):
        kinds = {k for k, _, _ in sides}
        out.append("mixed" if len(kinds) == 2 else f"{sides[0][0]}*{sides[0][0]}")
    return out


def served_pool(seed: int = 0):
    """The served mix's matrices, by key: 40 small ones from the batched
    generators ("s0".."s39", n 1k-16k, banded or Poisson(8)) and R-MAT scale
    14 (edge factor 8, 16), 15 (8, 16) and 16 (8) ("r14_0", ...)."""
    rng = np.random.default_rng(seed)
    pool = {}
    for i in range(40):
        n = int(round(np.exp(rng.uniform(np.log(1024), np.log(16384)))))
        s = int(rng.integers(0, 2**31 - 1))
        pool[f"s{i}"] = (banded(n, int(rng.integers(8, 65)), seed=s) if rng.random() < 0.5
                         else random_poisson(n, None, 8.0, seed=s))
    for sc, efs in ((14, (8, 16)), (15, (8, 16)), (16, (8,))):
        for i, ef in enumerate(efs):
            pool[f"r{sc}_{i}"] = rmat(sc, ef, seed=2 * (sc - 14) + i + 1)
    return pool


def served_jobs(pool, count: int, seed: int = 1):
    """`count` jobs (kind, a_key, b_key) over served_pool(): 85% small
    matrices, 10% R-MAT scale 14, 4% scale 15, 1% scale 16; half A*A^T (b_key
    None), half A*B with B a same-class matrix of matching size (A itself
    when there is none)."""
    rng = np.random.default_rng(seed)
    classes = {"small": [k for k in pool if k[0] == "s"]}
    for sc in (14, 15, 16):
        classes[sc] = [k for k in pool if k.startswith(f"r{sc}_")]
    jobs = []
    for _ in range(count):
        u = rng.random()
        cls = "small" if u < 0.85 else 14 if u < 0.95 else 15 if u < 0.99 else 16
        a = classes[cls][int(rng.integers(0, len(classes[cls])))]
        if rng.random() < 0.5:
            jobs.append(("AAT", a, None))
        else:
            same = [k for k in classes[cls] if pool[k][0] == pool[a][1]] or [a]
            jobs.append(("AB", a, same[int(rng.integers(0, len(same)))]))
    return jobs
