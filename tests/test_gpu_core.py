"""GPU parity of the core path against the CPU oracle, through the C ABI.

Bar: tile structure, masks, row offsets, per-tile nnz, column bytes and CSR
structure are bit-exact; FP64 values must be within relative error 1e-12 per
entry (REL_TOL below) -- and because the GPU accumulates each output entry in
the oracle's order with separately rounded multiply and add, the tests also
assert they are bit-identical.
"""
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
GOLD = Path(__file__).resolve().parent / "golden"
TILE_KEYS = ["tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col",
             "tile_csr_Value", "mask"]
C_KEYS = ["tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col", "mask"]


def golden_cases():
    z = np.load(GOLD / "cases.npz")
    names = sorted({k.split("/")[0] for k in z.files})
    return {nm: (z, (int(z[f"{nm}/m"][0]), int(z[f"{nm}/m"][1]), z[f"{nm}/rowptr"], z[f"{nm}/colidx"],
                     z[f"{nm}/val"])) for nm in names}


CASES = golden_cases()


def assert_values(got, want):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape
    den = np.maximum(np.abs(want), np.finfo(np.float64).tiny)
    rel = np.abs(got - want) / den
    rel[(got == want)] = 0.0
    assert float(rel.max(initial=0.0)) <= REL_TOL
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), "values not bit-identical to the oracle"


def assert_tiles(got, want, keys):
    for k in keys:
        if k == "tile_csr_Value":
            assert_values(got[k], want[k])
        else:
            np.testing.assert_array_equal(got[k], want[k], err_msg=k)


# ---------------------------------------------------------------------------
# conversion
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_csr2tile_matches_reference_fixture(tsg, name):
    z, mat = CASES[name]
    A = tsg.csr2tile_row_major(mat)
    for k in TILE_KEYS:
        np.testing.assert_array_equal(A[k], z[f"{name}/A/{k}"], err_msg=f"row-major {k}")
    B = tsg.csr2tile_col_major(mat)
    for k in TILE_KEYS + ["csc_tile_ptr", "csc_tile_rowidx"]:
        np.testing.assert_array_equal(B[k], z[f"{name}/B/{k}"], err_msg=f"col-major {k}")


def test_conversion_random_and_edges(tsg, gen, oracle):
    mats = [gen.random_poisson(int(m), int(n), lam, seed=s) for s, (m, n, lam) in
            enumerate([(1, 1, 1.0), (17, 33, 3.0), (250, 97, 6.0), (512, 512, 12.0), (1000, 40, 30.0)])]
    mats.append(gen.banded(300, 40, seed=1))              # full 16x16 tiles
    mats.append((5, 7, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0)))  # empty
    mats.append(gen.rmat(10, 8, seed=3))                  # skewed rows
    for mat in mats:
        assert_tiles(tsg.csr2tile_row_major(mat), oracle.csr2tile_row_major(mat), TILE_KEYS)
        B, Bo = tsg.csr2tile_col_major(mat), oracle.csr2tile_col_major(mat)
        assert_tiles(B, Bo, TILE_KEYS + ["csc_tile_ptr", "csc_tile_rowidx"])


# ---------------------------------------------------------------------------
# SpGEMM
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_tilespgemm_matches_oracle(tsg, oracle, name):
    """Drop-in path: host column-major B is converted to the internal layout."""
    z, mat = CASES[name]
    if mat[0] != mat[1]:
        pytest.skip("rectangular")
    A = {k: z[f"{name}/A/{k}"] for k in TILE_KEYS}
    B = {k: z[f"{name}/B/{k}"] for k in TILE_KEYS + ["csc_tile_ptr", "csc_tile_rowidx"]}
    for d in (A, B):
        d.update(m=mat[0], n=mat[1], nnz=mat[3].size, tilem=(mat[0] + 15) // 16, tilen=(mat[1] + 15) // 16,
                 numtile=d["tile_columnidx"].size)
    C, t = tsg.tilespgemm(A, B, nnzCub=oracle.count_products(mat, mat))
    Co = oracle.spgemm_tiled(A, B)
    assert_tiles(C, Co, C_KEYS + ["tile_csr_Value"])
    rp, ci, v = tsg.tile2csr(C)
    np.testing.assert_array_equal(rp, z[f"{name}/C/rowptr"])
    np.testing.assert_array_equal(ci, z[f"{name}/C/colidx"])
    if f"{name}/C/val" in z.files:
        assert_values(v, z[f"{name}/C/val"])


def _handle_product(tsg, ctx, matA, matB):
    import torch
    dev = torch.device("cuda", 0)

    def up(mat):
        m, n, rp, ci, v = mat
        return (torch.from_numpy(np.ascontiguousarray(rp, np.int32)).to(dev),
                torch.from_numpy(np.ascontiguousarray(ci, np.int32)).to(dev),
                torch.from_numpy(np.ascontiguousarray(v, np.float64)).to(dev))

    torch.cuda.synchronize()
    a = up(matA)
    b = up(matB)
    torch.cuda.synchronize()
    A = tsg.csr_to_tiled(ctx, matA[0], matA[1], *a, tsg.TSG_TILED_PACKED_COL)
    B = tsg.csr_to_tiled(ctx, matB[0], matB[1], *b, tsg.TSG_TILED_CSC_VIEW)
    C, info = tsg.spgemm(ctx, A, B)
    return A, B, C, info


SCHEDULES = [("tiles", 8, 512, True), ("elems", 8, 512, True), ("elems", 8, 512, False), ("tiles", 8, 512, False),
             ("spa", 8, 512, True), ("spa", 8, 512, False),
             ("rows", 8, 256, False), ("rows", 16, 1024, False), ("rows", 32, 2048, False)]


@pytest.fixture(params=SCHEDULES, ids=lambda p: f"{p[0]}{p[1]}-{p[2]}{'-fused' if p[3] else ''}")
def sched(request, ctx):
    ctx.set_schedule(*request.param[:3])
    ctx.set_fusion(request.param[3])
    yield request.param
    ctx.set_schedule("spa", 8, 512)
    ctx.set_fusion(True)


@pytest.mark.parametrize("seed", range(6))
def test_handle_spgemm_random_rectangular(tsg, ctx, sched, oracle, gen, seed):
    rng = np.random.default_rng(100 + seed)
    m, k, n = (int(x) for x in rng.integers(1, 700, 3))
    matA = gen.random_poisson(m, k, float(rng.uniform(0.5, 14)), seed=seed)
    matB = gen.random_poisson(k, n, float(rng.uniform(0.5, 14)), seed=seed + 50)
    A, B, C, info = _handle_product(tsg, ctx, matA, matB)
    Co = oracle.spgemm_tiled(oracle.csr2tile_row_major(matA), oracle.csr2tile_col_major(matB))
    assert_tiles(C.download(), Co, C_KEYS + ["tile_csr_Value"])
    assert info["numtile_C"] == Co["numtile"] and info["nnz_C"] == Co["nnz"]


def test_aat_and_dense_tiles(tsg, ctx, sched, oracle, gen):
    cases = [(gen.random_poisson(300, 200, 9.0, seed=4), None),
             (gen.banded(257, 48, seed=5), None),             # full (256) and dense (225-255) C tiles
             (gen.rmat(11, 16, seed=7), None)]                # hub rows
    for matA, _ in cases:
        matB = gen.transpose(matA) if matA[0] != matA[1] else matA
        for B in ([matB, gen.transpose(matA)] if matA[0] == matA[1] else [matB]):
            A_, B_, C, info = _handle_product(tsg, ctx, matA, B)
            Co = oracle.spgemm_tiled(oracle.csr2tile_row_major(matA), oracle.csr2tile_col_major(B))
            assert_tiles(C.download(), Co, C_KEYS + ["tile_csr_Value"])


def test_many_pairs_per_c_tile(tsg, ctx, sched, oracle, gen):
    """C tiles with ~100 matched tile pairs (long A rows and B columns): every
    product still folds in k order."""
    matA = gen.random_poisson(1600, 1600, 120.0, seed=8)
    matB = gen.random_poisson(1600, 1500, 30.0, seed=9)
    A_, B_, C, info = _handle_product(tsg, ctx, matA, matB)
    rp, ci, v = (x.cpu().numpy() for x in tsg.tiled_to_csr(ctx, C))
    G = oracle.gustavson(matA, matB)
    np.testing.assert_array_equal(rp, G[2])
    np.testing.assert_array_equal(ci, G[3])
    assert np.array_equal(v.view(np.uint64), G[4].view(np.uint64))


def _hyper_rows(matA, matB, Co):
    """Per A tile row: True where the fused step 1/2 pass marks it
    hypersparse -- more than 128 C tiles, C tile columns spanning less than
    16,384, and exact scalar products (sum over A's entries of B's row
    length) below 4 per C tile."""
    m, _, rpA, ciA, _ = matA
    tilem = (m + 15) // 16
    rowsA = np.repeat(np.arange(m), np.diff(rpA)) // 16
    prods = np.bincount(rowsA, weights=np.diff(matB[2])[ciA], minlength=tilem)
    tp, col = np.asarray(Co["tile_ptr"]), np.asarray(Co["tile_columnidx"])
    nt = np.diff(tp)
    span = np.zeros(tilem, np.int64)
    has = nt > 0
    span[has] = col[tp[1:][has] - 1] - col[tp[:-1][has]]
    return (nt > 128) & (span < 16384) & (prods < 4 * nt)


def test_hypersparse_rows(tsg, ctx, sched, oracle, gen):
    """Random operands so sparse that nearly every tile column of a C tile row
    exists while few of those tiles receive a product: the whole-row
    hypersparse path (masks ORed in global memory, values summed in k order
    in place).  Covers rectangular shapes, empty rows of A and B and rows
    spanning ~12,000 tile columns (n = 200,000); the last case's C rows span
    more than 16,384 tile columns (n = 300,000) and take the segment path
    instead."""
    cases = [(gen.random_poisson(8192, 8192, 4.0, seed=31), gen.random_poisson(8192, 8192, 4.0, seed=32), True),
             (gen.random_poisson(6000, 5000, 0.4, seed=33), gen.random_poisson(5000, 7000, 6.0, seed=34), True),
             (gen.random_poisson(2048, 4096, 3.0, seed=37), gen.random_poisson(4096, 200000, 3.0, seed=38), True),
             (gen.random_poisson(4096, 8192, 3.0, seed=35), gen.random_poisson(8192, 300000, 3.0, seed=36), False)]
    for matA, matB, hyper in cases:
        A_, B_, C, info = _handle_product(tsg, ctx, matA, matB)
        Co = oracle.spgemm_tiled(oracle.csr2tile_row_major(matA), oracle.csr2tile_col_major(matB))
        assert_tiles(C.download(), Co, C_KEYS + ["tile_csr_Value"])
        frac = _hyper_rows(matA, matB, Co).mean()
        assert (frac > 0.9) if hyper else (frac < 0.1)


_ORACLE_CACHE = {}


def test_long_rows_in_large_blocks(tsg, ctx, sched, oracle, gen):
    """A product whose mean C tile row is ~2,048 tiles: the SPA steps take
    blocks of 2,048 tiles, and the 4,096-tile rows (not hypersparse: ~6
    products per tile) are cut into chunks owned by different blocks; every
    other tile row is empty."""
    if "long_rows" not in _ORACLE_CACHE:  # the same inputs for every schedule
        m0, n0, rp, ci, v = gen.random_poisson(2048, 65536, 40.0, seed=41)
        keep = (np.arange(m0) // 16) % 2 == 0
        lens = np.where(keep, np.diff(rp), 0)
        sel = np.repeat(keep, np.diff(rp))
        matA = (m0, n0, np.concatenate([[0], np.cumsum(lens)]).astype(rp.dtype), ci[sel], v[sel])
        matB = gen.random_poisson(65536, 65536, 40.0, seed=42)
        _ORACLE_CACHE["long_rows"] = (matA, matB, oracle.spgemm_tiled(oracle.csr2tile_row_major(matA),
                                                                      oracle.csr2tile_col_major(matB)))
    matA, matB, Co = _ORACLE_CACHE["long_rows"]
    A_, B_, C, info = _handle_product(tsg, ctx, matA, matB)
    assert_tiles(C.download(), Co, C_KEYS + ["tile_csr_Value"])
    nt = np.diff(np.asarray(Co["tile_ptr"]))
    assert Co["numtile"] // len(nt) >= 2048 and nt.max() > 2048
    assert not _hyper_rows(matA, matB, Co).any()  # SPA rows, not hypersparse


def test_laplacian_256_known_answers(tsg, ctx, sched, oracle, gen):
    facts = json.loads((GOLD / "known_answers.json").read_text())["laplacian_256x256"]
    mat = gen.laplacian_2d(256)
    A, B, C, info = _handle_product(tsg, ctx, mat, mat)
    assert info["numtile_C"] == facts["tilesC"] and info["nnz_C"] == facts["nnzC"]
    Cd = C.download()
    assert int(np.count_nonzero(np.diff(Cd["tile_nnz"]))) == facts["tilesC_nonempty"]
    Co = oracle.spgemm_tiled(oracle.csr2tile_row_major(mat), oracle.csr2tile_col_major(mat))
    assert_tiles(Cd, Co, C_KEYS + ["tile_csr_Value"])
    rp, ci, v = (x.cpu().numpy() for x in tsg.tiled_to_csr(ctx, C))
    assert ci[rp[0]:rp[1]].tolist() == facts["row0_cols"]
    assert v[rp[0]:rp[1]].tolist() == facts["row0_vals"]


def test_stencil27_full_size_against_gustavson(tsg, ctx, sched, oracle, gen):
    """27-point stencil 64^3 (n=262,144): structure and every value against the
    element-level oracle; the known answers pin the counts."""
    facts = json.loads((GOLD / "known_answers.json").read_text())["stencil27_64"]
    mat = gen.stencil_27pt_3d(64, seed=0)
    A, B, C, info = _handle_product(tsg, ctx, mat, mat)
    assert A.numtile == facts["tilesA"]
    assert info["numtile_C"] == facts["tilesC"] and info["nnz_C"] == facts["nnzC"]
    rp, ci, v = (x.cpu().numpy() for x in tsg.tiled_to_csr(ctx, C))
    G = oracle.gustavson(mat, mat, nthreads=8)
    np.testing.assert_array_equal(rp, G[2])
    np.testing.assert_array_equal(ci, G[3])
    assert_values(v, G[4])


def test_spgemm_is_deterministic(tsg, ctx, sched, gen):
    mat = gen.rmat(12, 8, seed=2)
    _, _, C1, _ = _handle_product(tsg, ctx, mat, mat)
    _, _, C2, _ = _handle_product(tsg, ctx, mat, mat)
    d1, d2 = C1.download(), C2.download()
    for k in C_KEYS + ["tile_csr_Value"]:
        assert np.array_equal(np.asarray(d1[k]).view(np.uint8), np.asarray(d2[k]).view(np.uint8))


# ---------------------------------------------------------------------------
# tile -> CSR and end to end
# ---------------------------------------------------------------------------
def test_tile2csr_dropin_matches_oracle(tsg, oracle, gen):
    for mat in [gen.laplacian_2d(37, 29), gen.random_poisson(200, 300, 7.0, seed=8)]:
        T = oracle.csr2tile_row_major(mat)
        T["tile_csr_Col"] = T["tile_csr_Col"] & 15  # plain bytes, as C tiles carry
        rp, ci, v = tsg.tile2csr(T)
        np.testing.assert_array_equal(rp, mat[2])
        np.testing.assert_array_equal(ci, mat[3])
        assert_values(v, mat[4])


def test_end_to_end_host_call(tsg, ctx, oracle, gen):
    for matA, matB in [(gen.laplacian_2d(100), None),
                       (gen.random_poisson(333, 444, 5.0, seed=1), gen.random_poisson(444, 222, 5.0, seed=2))]:
        C, info = tsg.spgemm_csr_host(ctx, matA, matB)
        G = oracle.gustavson(matA, matA if matB is None else matB)
        np.testing.assert_array_equal(C[2], G[2])
        np.testing.assert_array_equal(C[3], G[3])
        assert_values(C[4], G[4])


# ---------------------------------------------------------------------------
# input errors come back as status codes, never as a device fault
# ---------------------------------------------------------------------------
def test_malformed_csr_is_rejected(tsg, ctx):
    import torch
    dev = torch.device("cuda", 0)
    rp = torch.tensor([0, 2, 3], dtype=torch.int32, device=dev)
    unsorted = torch.tensor([5, 1, 0], dtype=torch.int32, device=dev)
    out_of_range = torch.tensor([1, 9, 0], dtype=torch.int32, device=dev)
    v = torch.ones(3, dtype=torch.float64, device=dev)
    for ci in (unsorted, out_of_range):
        with pytest.raises(tsg.TsgError) as e:
            tsg.csr_to_tiled(ctx, 2, 8, rp, ci, v, tsg.TSG_TILED_PACKED_COL)
        assert e.value.status == -4


def test_two_phase_end_to_end_into_caller_buffers(tsg, ctx, oracle, gen):
    out = tsg.HostResultBuffers(10, 10)
    for matA, matB in [(gen.laplacian_2d(60), None), (gen.random_poisson(200, 150, 5.0, seed=3),
                                                       gen.random_poisson(150, 90, 5.0, seed=4))]:
        C, info = tsg.spgemm_csr_host_into(ctx, matA, matB, out)
        G = oracle.gustavson(matA, matA if matB is None else matB)
        np.testing.assert_array_equal(C[2], G[2])
        np.testing.assert_array_equal(C[3], G[3])
        assert_values(C[4], G[4])


def test_row_blocks_of_a_give_the_whole_product(tsg, ctx, gen):
    """C computed from blocks of A's tile rows (the large-product driver)
    equals C computed at once, bit for bit."""
    import torch
    A = gen.rmat(12, 8, seed=21)
    B = gen.transpose(A)
    m, n, rp, ci, v = A
    TB = tsg.csr_host_to_tiled(ctx, B, tsg.TSG_TILED_CSC_VIEW)
    TA = tsg.csr_host_to_tiled(ctx, A, tsg.TSG_TILED_PACKED_COL)
    C, _ = tsg.spgemm(ctx, TA, TB)
    whole = [x.cpu().numpy() for x in tsg.tiled_to_csr(ctx, C)]
    parts = []
    for r0 in range(0, m, 16 * 37):  # blocks of 37 tile rows
        r1 = min(r0 + 16 * 37, m)
        blk = (r1 - r0, n, (rp[r0:r1 + 1] - rp[r0]).astype(np.int32), ci[rp[r0]:rp[r1]], v[rp[r0]:rp[r1]])
        Tb = tsg.csr_host_to_tiled(ctx, blk, tsg.TSG_TILED_PACKED_COL)
        Cb, _ = tsg.spgemm(ctx, Tb, TB)
        parts.append([x.cpu().numpy() for x in tsg.tiled_to_csr(ctx, Cb)])
    rp_all = np.concatenate([[0]] + [p[0][1:] + sum(q[0][-1] for q in parts[:i]) for i, p in enumerate(parts)])
    np.testing.assert_array_equal(rp_all, whole[0])
    np.testing.assert_array_equal(np.concatenate([p[1] for p in parts]), whole[1])
    assert np.array_equal(np.concatenate([p[2] for p in parts]).view(np.uint64), whole[2].view(np.uint64))


@pytest.mark.parametrize("name", sorted(CASES))
def test_intersection_bitmaps_match_the_drivers(tsg, oracle, name):
    """tile_intersection_bitmaps equals the reference driver's loops
    (src/main.cu:430-465) on the golden fixtures' tiles, and on a product
    whose tile counts are not multiples of 32."""
    z, mat = CASES[name]
    if mat[0] != mat[1]:
        pytest.skip("rectangular: A*A is not defined")
    A = {k: z[f"{name}/A/{k}"] for k in TILE_KEYS}
    B = {k: z[f"{name}/B/{k}"] for k in TILE_KEYS + ["csc_tile_ptr", "csc_tile_rowidx"]}
    for d in (A, B):
        d.update(m=mat[0], n=mat[1], nnz=mat[3].size, tilem=(mat[0] + 15) // 16, tilen=(mat[1] + 15) // 16,
                 numtile=d["tile_columnidx"].size)
    got = tsg.tile_intersection_bitmaps(A, B)
    want = oracle.intersection_bitmaps(A, B)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)


def test_intersection_bitmaps_rectangular(tsg, oracle, gen):
    a, b = gen.random_poisson(900, 1000, 4.0, seed=61), gen.random_poisson(1000, 777, 5.0, seed=62)
    A, B = tsg.csr2tile_row_major(a), tsg.csr2tile_col_major(b)
    got = tsg.tile_intersection_bitmaps(A, B)
    want = oracle.intersection_bitmaps(A, B)
    assert got[0].shape == (A["tilem"], (A["tilen"] + 31) // 32) and got[1].shape == (B["tilen"], (A["tilen"] + 31) // 32)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)
