"""The tile-aware reorder planner (build_reorder_plan, src/reorder.h:2407)
for A*A of symmetric matrices -- host code in the reference and here, so the
reference's own planner, compiled from its sources into oracle/_ref, runs
beside it on the CPU.  Every plan path is covered: identity for narrow tile
rows, reverse Cuthill-McKee with windowed refinement (n <= 50,000), windowed
16-row packing (n > 50,000), the risk guard's fall-back to identity, the
TASA_FORCE_ACTIVE and TASA_AB_SHARED_SYM switches and the error codes.  The
three permutations, the estimates, ratios, flags, window, mode and reason
must equal the reference's exactly (the planner's timings are not
compared).  General matrices, A*B and A*A^T run their signatures on the GPU
(tests/test_gpu_tasa.py)."""
import ctypes

import numpy as np
import pytest

from conftest import load_oracle, load_package


def _sym(mat):
    import scipy.sparse as sp
    m, n, rp, ci, v = mat
    a = sp.csr_matrix((np.ones(len(ci)), ci, rp), shape=(m, n))
    s = ((a + a.T) > 0).astype(np.float64).tocsr()
    s.sort_indices()
    return m, n, s.indptr.astype(np.int32), s.indices.astype(np.int32), np.asarray(s.data)


@pytest.fixture(scope="module")
def ref():
    o = load_oracle()
    if not o.ref_reorder_available():
        pytest.skip("oracle/_ref/libtsgref_reorder.so not built (reference tree absent when oracle/Makefile ran)")
    return o


@pytest.fixture(scope="module")
def gen():
    load_package()
    import rw_spgemm_b200.generators as g
    return g


def _same(got, want):
    o = load_oracle()
    for f in o.PLAN_FIELDS + ("mode", "risk_reason"):
        assert got[f] == want[f], (f, got[f], want[f])
    for ax in ("row_perm", "inner_perm", "col_perm"):
        np.testing.assert_array_equal(got[ax], want[ax], err_msg=ax)


CASES = {
    "laplacian_100x100": ("identity_narrow_tiles", lambda g: g.laplacian_2d(100)),
    "poisson_8000": ("active_symmetric", lambda g: _sym(g.random_poisson(8000, 8000, 8.0, seed=3))),
    "rmat_13": ("active_symmetric", lambda g: _sym(g.rmat(13, 8, seed=1))),
    "banded_20000_permuted": ("active_symmetric", lambda g: g.permute_symmetric(
        g.banded(20000, 40, seed=2), g.random_symmetric_permutation(20000, seed=3))),
    "stencil27_40_permuted": ("active_symmetric", lambda g: g.permute_symmetric(
        g.stencil_27pt_3d(40), g.random_symmetric_permutation(64000, seed=7))),
    "poisson_60000": ("active_symmetric", lambda g: _sym(g.random_poisson(60000, 60000, 4.0, seed=5))),
    # the guard: a band the reverse Cuthill-McKee order does not improve
    "banded_8000_no_gain": ("conservative_identity", lambda g: g.banded(8000, 300, seed=1)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_symmetric_plan_equals_the_references(ref, gen, name):
    mode, make = CASES[name]
    tsg = load_package()
    M = make(gen)
    st, want = ref.ref_build_reorder_plan("AA", M, symmetric=True)
    assert st == 0 and want["mode"] == mode
    got = tsg.build_reorder_plan("AA", "tasa", M, symmetric=True)
    _same(got, want)
    n = M[0]
    window = 0 if mode == "identity_narrow_tiles" else (32 if n <= 50000 else 64)
    assert got["local_refine_window"] == window
    if mode == "conservative_identity":
        assert got["risk_reason"] == "small_no_tile_gain" and got["guard_degraded_to_identity"] == 1
        np.testing.assert_array_equal(got["row_perm"], np.arange(n))
    for ax in ("row_perm", "inner_perm", "col_perm"):
        assert sorted(got[ax].tolist()) == list(range(n))
    np.testing.assert_array_equal(got["row_perm"], got["col_perm"])     # one order on every axis


def test_forced_plans_and_the_shared_symmetric_a_times_b(ref, gen, monkeypatch):
    tsg = load_package()
    M = _sym(gen.random_poisson(4000, 4000, 2.0, seed=9))
    monkeypatch.setenv("TASA_FORCE_ACTIVE", "1")
    st, want = ref.ref_build_reorder_plan("AA", M, symmetric=True)
    assert st == 0 and want["risk_reason"] == "accepted_force"
    _same(tsg.build_reorder_plan("AA", "tasa", M, symmetric=True), want)
    monkeypatch.setenv("TASA_FORCE_ACTIVE", "")
    monkeypatch.setenv("TASA_AB_SHARED_SYM", "1")
    A, B = _sym(gen.random_poisson(8000, 8000, 8.0, seed=3)), _sym(gen.random_poisson(8000, 8000, 6.0, seed=4))
    st, want = ref.ref_build_reorder_plan("AB", A, B, symmetric=True)
    assert st == 0 and want["mode"] == "conservative_identity" and want["risk_reason"] == "small_no_tile_gain"
    _same(tsg.build_reorder_plan("AB", "tasa", A, B, symmetric=True), want)


def test_non_square_a_times_a_is_refused_like_the_reference(ref, gen):
    tsg = load_package()
    M = gen.random_poisson(100, 120, 3.0, seed=1)
    st, _ = ref.ref_build_reorder_plan("AA", M, symmetric=True)
    with pytest.raises(tsg.TsgError) as e:
        tsg.build_reorder_plan("AA", "tasa", M, symmetric=True)
    assert st == -1 and e.value.status == -1


def test_reorder_info_init_equals_the_references(ref):
    tsg = load_package()
    L = tsg.lib()
    mine = tsg.ReorderInfo()
    L.reorder_info_init(ctypes.byref(mine))
    theirs = ref.OReorderInfo()
    ref.rrlib().ref_reorder_info_init(ctypes.byref(theirs))
    for f in ref.PLAN_FIELDS:
        assert getattr(mine, f) == getattr(theirs, f), f
    assert mine.mode == theirs.mode and mine.risk_reason == theirs.risk_reason
