"""GPU parity at the sizes bench.py runs, against the CPU oracle.

* R-MAT scale 20 (edge factor 16), C = A*A and C = A*A^T, computed in the
  bench's row blocks: every block's nnz(C) equals the oracle's row counts
  summed over its rows, and three sub-blocks (the first tile rows, the
  heaviest tile row -- hub rows -- and the last tile rows) equal the oracle
  entry by entry (structure bit-exact, values bit-identical).
* The 27-point 64^3 stencil after the bench's random symmetric permutation,
  under every GPU ordering: the product computed in the new order and
  restored equals the product of the permuted matrix (structure bit-exact,
  values within REL_TOL: the inner index order changes with the ordering),
  and that equals the natural-order product under the permutation.
* The bench's 512-product batch: every product bit-identical to the
  one-product path, and 32 of them to the oracle.
* The bench's served mix, R-MAT scale 14-16 jobs included: every result
  bit-identical to the one-product path, sampled ones to the oracle.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
NTHREADS = max(1, os.cpu_count() or 1)
C_KEYS = ["tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col", "mask",
          "tile_csr_Value"]


@pytest.fixture(scope="module")
def blocks_mod(tsg):
    import rw_spgemm_b200.blocks as b
    return b


def _csr_equal(got, want, exact_values=True):
    np.testing.assert_array_equal(np.asarray(got[0]), np.asarray(want[2]))
    np.testing.assert_array_equal(np.asarray(got[1]), np.asarray(want[3]))
    gv, wv = np.asarray(got[2], np.float64), np.asarray(want[4], np.float64)
    if exact_values:
        assert np.array_equal(gv.view(np.uint64), wv.view(np.uint64)), "values not bit-identical"
    else:
        rel = np.abs(gv - wv) / np.maximum(np.abs(wv), np.finfo(np.float64).tiny)
        rel[gv == wv] = 0.0
        assert float(rel.max(initial=0.0)) <= REL_TOL


@pytest.mark.parametrize("kind", ["A*A", "A*A^T"])
def test_rmat20_row_blocks_against_oracle(tsg, ctx, gen, oracle, blocks_mod, kind):
    A = gen.rmat(20, 16, seed=1)
    B = A if kind == "A*A" else gen.transpose(A)
    counts, total = oracle.gustavson_row_nnz(A, B, nthreads=NTHREADS)
    row_csum = np.concatenate([[0], np.cumsum(counts, dtype=np.int64)])
    TB = tsg.csr_host_to_tiled(ctx, B, tsg.TSG_TILED_CSC_VIEW)
    tileprod = blocks_mod.tile_row_products(A, B)
    blocks = blocks_mod.row_blocks(tileprod, 1.5e9)  # the bench's blocks
    assert len(blocks) >= 3
    m = A[0]
    got_total = 0
    for b0, b1 in blocks:
        TA = tsg.csr_host_to_tiled(ctx, blocks_mod.block_rows(A, b0, b1), tsg.TSG_TILED_PACKED_COL)
        C, info = tsg.spgemm(ctx, TA, TB)
        want = int(row_csum[min(b1 * 16, m)] - row_csum[b0 * 16])
        assert info["nnz_C"] == want, f"block {b0}-{b1}"
        got_total += info["nnz_C"]
        C.free()
        TA.free()
    assert got_total == total
    # entry by entry: first tile rows, the heaviest tile row, last tile rows
    heavy = int(np.argmax(tileprod))
    for t0, t1 in ((0, 4), (heavy, heavy + 1), (len(tileprod) - 4, len(tileprod))):
        sub = blocks_mod.block_rows(A, t0, t1)
        TA = tsg.csr_host_to_tiled(ctx, sub, tsg.TSG_TILED_PACKED_COL)
        C, info = tsg.spgemm(ctx, TA, TB)
        got = [x.cpu().numpy() for x in tsg.tiled_to_csr(ctx, C)]
        C.free()
        TA.free()
        _csr_equal(got, oracle.gustavson(sub, B, nthreads=NTHREADS))
    TB.free()


def _permute_result(C, new_of_old):
    """The CSR C of a product permuted: row/column i -> new_of_old[i]."""
    m, n, rp, ci, v = C
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(rp))
    r2, c2 = new_of_old[rows], new_of_old[ci]
    order = np.lexsort((c2, r2))
    rp2 = np.zeros(m + 1, np.int64)
    np.add.at(rp2, r2 + 1, 1)
    return m, n, np.cumsum(rp2).astype(np.int32), c2[order].astype(np.int32), np.asarray(v)[order]


def test_permuted_stencil64_every_ordering_restores_the_product(tsg, ctx, gen):
    import torch
    base = gen.stencil_27pt_3d(64, seed=0)
    perm = gen.random_symmetric_permutation(base[0], 7)   # new -> old, as the bench
    mat = gen.permute_symmetric(base, perm)
    m, n, rp, ci, v = mat
    # natural-order product, moved under the permutation
    Cb, _ = tsg.spgemm_csr_host(ctx, base)
    new_of_old = np.empty(m, np.int64)
    new_of_old[perm] = np.arange(m)
    want = _permute_result((m, n) + tuple(Cb[2:]), new_of_old)
    C0, _ = tsg.spgemm_csr_host(ctx, mat)
    _csr_equal(C0[2:], want, exact_values=False)
    dev = torch.device("cuda", 0)
    d_rp, d_ci = (torch.from_numpy(np.ascontiguousarray(x, np.int32)).to(dev) for x in (rp, ci))
    tiles_before = None
    for kind in ("original", "rcm", "degree", "gray", "random"):
        p = tsg.order(ctx, kind, m, n, d_rp, d_ci, seed=1).cpu().numpy()
        assert np.array_equal(np.sort(p), np.arange(m))
        Cp, info = tsg.spgemm_csr_host(ctx, tsg.apply_bipermutation_csr(mat, p, p))
        C = tsg.restore_bipermutation_csr(Cp, p, p)
        _csr_equal(C[2:], (m, n) + tuple(C0[2:]), exact_values=(kind == "original"))
        if kind == "original":
            tiles_before = info["numtile_C"]
        elif kind == "rcm":
            assert info["numtile_C"] < tiles_before / 50  # RCM restores the band


def test_batched_512_against_single_path_and_oracle(tsg, ctx, gen, oracle):
    mats = gen.batched_products(512, seed=0)
    pairs = [(tsg.csr_host_to_tiled(ctx, a, tsg.TSG_TILED_CSC_VIEW), tsg.csr_host_to_tiled(ctx, b, tsg.TSG_TILED_CSC_VIEW))
             for a, b in mats]
    batch = tsg.Batch(ctx, pairs, "spa", 8, 512, graph=True)
    batch.run()
    tiles, nnz = batch.sync()
    sampled = set(np.random.default_rng(4).choice(len(mats), 32, replace=False).tolist())
    t_sum = n_sum = 0
    for p, (A, B) in enumerate(pairs):
        got = batch.product(p).download()
        C, info = tsg.spgemm(ctx, A, B)
        want = C.download()
        for k in C_KEYS:
            assert np.array_equal(np.asarray(got[k]).view(np.uint8), np.asarray(want[k]).view(np.uint8)), \
                f"product {p}: {k} differs from the one-product path"
        if p in sampled:
            _csr_equal([x.cpu().numpy() for x in tsg.tiled_to_csr(ctx, C)],
                       oracle.gustavson(mats[p][0], mats[p][1], nthreads=NTHREADS))
        t_sum += want["numtile"]
        n_sum += want["nnz"]
        C.free()
    assert tiles == t_sum and nnz == n_sum
    batch.close()
    for A, B in pairs:
        A.free()
        B.free()


def test_served_mix_with_rmat_jobs(tsg, ctx, gen, oracle):
    import rw_spgemm_b200.serve as srv_mod
    pool = gen.served_pool()
    jobs = gen.served_jobs(pool, 240, seed=5)
    assert sum(1 for _, a, _ in jobs if a.startswith("r16")) >= 1  # the heaviest class is in the mix
    srv = srv_mod.SpGEMMServer(0, mem_cap=40 << 30, slots=2, max_batch=64)
    for key, m in pool.items():
        srv.register(key, m)
    srv.start()
    futs = [srv.submit(kind, a, b) for kind, a, b in jobs]
    res = [f.result(timeout=600) for f in futs]
    srv.close()
    checked = set()
    for i, ((kind, a, b), C) in enumerate(zip(jobs, res)):
        key = (kind, a, b)
        if key in checked:
            continue  # same operands: the same one-product result
        checked.add(key)
        Bm = gen.transpose(pool[a]) if kind == "AAT" else pool[b]
        alone, _ = tsg.spgemm_csr_host(ctx, pool[a], Bm)
        for x, y in zip(C[2:], alone[2:]):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8)), f"job {i} {key}"
        if len(checked) % 8 == 1:
            _csr_equal([np.asarray(x) for x in C[2:]], oracle.gustavson(pool[a], Bm, nthreads=NTHREADS))
