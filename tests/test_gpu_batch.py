"""Batched products in one persistent launch: every product equals the
oracle (bit for bit) and the one-product path, under both schedules, and
graph replays reproduce the same bits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
C_KEYS = ["tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col", "mask",
          "tile_csr_Value"]


def _tiled(tsg, ctx, mat, flags):
    import torch
    d = torch.device("cuda", 0)
    m, n, rp, ci, v = mat
    t = [torch.from_numpy(np.ascontiguousarray(x)).to(d) for x in (rp.astype(np.int32), ci.astype(np.int32),
                                                                    v.astype(np.float64))]
    torch.cuda.synchronize()
    T = tsg.csr_to_tiled(ctx, m, n, *t, flags)
    T._keep = t
    return T


def _pairs(gen):
    rng = np.random.default_rng(5)
    mats = []
    for i in range(14):
        m, k, n = (int(x) for x in rng.integers(1, 400, 3))
        mats.append((gen.random_poisson(m, k, float(rng.uniform(0.5, 10)), seed=i),
                     gen.random_poisson(k, n, float(rng.uniform(0.5, 10)), seed=100 + i)))
    mats.append((gen.banded(300, 40, seed=1), gen.banded(300, 20, seed=2)))   # dense / full tiles
    mats.append((gen.rmat(10, 8, seed=3), gen.rmat(10, 8, seed=4)))          # hubs
    mats.append((gen.laplacian_2d(30), gen.laplacian_2d(30)))
    mats.append(((5, 6, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0)),
                 gen.random_poisson(6, 9, 2.0, seed=9)))                    # empty A
    # hypersparse: wide C tile rows with few products (whole-row path)
    mats.append((gen.random_poisson(8192, 8192, 4.0, seed=10), gen.random_poisson(8192, 8192, 4.0, seed=11)))
    mats.append((gen.random_poisson(3000, 4000, 2.0, seed=12), gen.random_poisson(4000, 9000, 3.0, seed=13)))
    return mats


@pytest.mark.parametrize("cfg", [("rows", 16, 1024), ("rows", 8, 256), ("rows", 32, 2048), ("tiles", 8, 256),
                                 ("elems", 8, 256), ("spa", 8, 512)])
def test_batch_matches_oracle_and_single_path(tsg, ctx, oracle, gen, cfg):
    mats = _pairs(gen)
    pairs = [(_tiled(tsg, ctx, a, tsg.TSG_TILED_PACKED_COL), _tiled(tsg, ctx, b, tsg.TSG_TILED_CSC_VIEW))
             for a, b in mats]
    batch = tsg.Batch(ctx, pairs, *cfg)
    batch.run()
    tiles, nnz = batch.sync()
    first = []
    for p, (a, b) in enumerate(mats):
        got = batch.product(p).download()
        want = oracle.spgemm_tiled(oracle.csr2tile_row_major(a), oracle.csr2tile_col_major(b))
        for k in C_KEYS:
            np.testing.assert_array_equal(np.asarray(got[k]).view(np.uint8), np.asarray(want[k]).view(np.uint8),
                                          err_msg=f"product {p} {k}")
        first.append(got)
    assert tiles == sum(f["numtile"] for f in first) and nnz == sum(f["nnz"] for f in first)
    # replay: same bits
    batch.run()
    batch.sync()
    for p in range(len(mats)):
        again = batch.product(p).download()
        for k in C_KEYS:
            np.testing.assert_array_equal(np.asarray(again[k]).view(np.uint8), np.asarray(first[p][k]).view(np.uint8))
    info = batch.info()
    assert info["launches"] == 2 and info["grid"] > 0
    batch.close()


def test_batch_uses_graph(tsg, ctx, gen):
    mats = _pairs(gen)[:3]
    pairs = [(_tiled(tsg, ctx, a, 1), _tiled(tsg, ctx, b, 2)) for a, b in mats]
    batch = tsg.Batch(ctx, pairs)
    assert batch.info()["graph"], "the persistent launch was not captured in a CUDA graph"
    batch.close()


def test_product_bounds_bound_the_result(tsg, ctx, oracle, gen):
    for a, b in _pairs(gen)[:6]:
        A, B = _tiled(tsg, ctx, a, 1), _tiled(tsg, ctx, b, 2)
        prods, pairs = tsg.product_bounds(ctx, A, B)
        assert prods == oracle.count_products(a, b)
        C, info = tsg.spgemm(ctx, A, B)
        assert info["nnz_C"] <= prods and info["numtile_C"] <= pairs


def test_product_bounds_of_many_products_in_one_call(tsg, ctx, oracle, gen):
    mats = _pairs(gen)
    pairs = [(_tiled(tsg, ctx, a, 1), _tiled(tsg, ctx, b, 2)) for a, b in mats]
    many = tsg.product_bounds_many(ctx, pairs, c_tiles=True)
    assert [m[:2] for m in many] == tsg.product_bounds_many(ctx, pairs)
    for (a, b), (A, B), (prods, tpairs, ctiles) in zip(mats, pairs, many):
        assert (prods, tpairs) == tsg.product_bounds(ctx, A, B)
        assert prods == oracle.count_products(a, b)
        C, info = tsg.spgemm(ctx, A, B)
        assert ctiles == info["numtile_C"]      # step 1's count is exact
    assert tsg.product_bounds_many(ctx, []) == []


def test_batch_planned_from_given_bounds(tsg, ctx, gen):
    """tsg_batch_create_bounded with tsg_product_bounds_many's bounds gives
    the same bits and arena as the self-bounding create; a C-tile bound
    below the true count makes the batch report TSG_ERR_OVERFLOW (the
    kernel's own capacity check skips that product)."""
    mats = _pairs(gen)
    pairs = [(_tiled(tsg, ctx, a, tsg.TSG_TILED_PACKED_COL), _tiled(tsg, ctx, b, tsg.TSG_TILED_CSC_VIEW))
             for a, b in mats]
    bounds = [(pr, ct) for pr, _, ct in tsg.product_bounds_many(ctx, pairs, c_tiles=True)]
    ref = tsg.Batch(ctx, pairs, "spa", 8, 512, graph=False)
    ref.run()
    ref.sync()
    got = tsg.Batch(ctx, pairs, "spa", 8, 512, graph=False, bounds=bounds)
    assert got.info()["arena_bytes"] == ref.info()["arena_bytes"]
    got.run()
    got.sync()
    for p in range(len(mats)):
        a, b = ref.product(p).download(), got.product(p).download()
        for k in C_KEYS:
            np.testing.assert_array_equal(np.asarray(b[k]).view(np.uint8), np.asarray(a[k]).view(np.uint8))
    got.close()
    p_big = max(range(len(bounds)), key=lambda i: bounds[i][1])
    short = list(bounds)
    short[p_big] = (bounds[p_big][0], bounds[p_big][1] - 1)
    bad = tsg.Batch(ctx, pairs, "spa", 8, 512, graph=False, bounds=short)
    bad.run()
    with pytest.raises(tsg.TsgError, match="exceeded its bound"):
        bad.sync()
    bad.close()
    ref.close()
    with pytest.raises(ValueError):
        tsg.Batch(ctx, pairs, bounds=bounds[:-1])


def test_batch_phase_times(tsg, ctx, gen):
    mats = _pairs(gen)[:6]
    pairs = [(_tiled(tsg, ctx, a, 1), _tiled(tsg, ctx, b, 2)) for a, b in mats]
    batch = tsg.Batch(ctx, pairs)
    batch.run()
    batch.sync()
    ph = batch.phase_ms()
    assert len(ph) == 7 and all(v >= 0.0 for v in ph.values())
    assert 0.0 < sum(ph.values()) < 10_000.0
    batch.close()


@pytest.mark.parametrize("graph", [False, True])
def test_batch_barrier_bound_gives_up_and_the_batch_recovers(tsg, ctx, oracle, gen, graph):
    """A grid-barrier wait bound of zero makes the waiting blocks give up: the
    run reports TSG_ERR_TIMEOUT through sync (no GPU fault, the context stays
    usable), and the same batch with a normal bound then computes every
    product exactly."""
    mats = _pairs(gen)[:8]
    pairs = [(_tiled(tsg, ctx, a, tsg.TSG_TILED_PACKED_COL), _tiled(tsg, ctx, b, tsg.TSG_TILED_CSC_VIEW))
             for a, b in mats]
    batch = tsg.Batch(ctx, pairs, "spa", 8, 512, graph=graph)
    batch.set_wait_limit(0.0)
    batch.run()
    with pytest.raises(tsg.TsgError) as ei:
        batch.sync()
    assert ei.value.status == -7  # TSG_ERR_TIMEOUT
    batch.set_wait_limit(10.0)
    batch.run()
    batch.sync()
    for p, (a, b) in enumerate(mats):
        got = batch.product(p).download()
        want = oracle.spgemm_tiled(oracle.csr2tile_row_major(a), oracle.csr2tile_col_major(b))
        for k in C_KEYS:
            np.testing.assert_array_equal(np.asarray(got[k]).view(np.uint8), np.asarray(want[k]).view(np.uint8),
                                          err_msg=f"product {p} {k}")
    batch.close()
