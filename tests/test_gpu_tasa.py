"""The tile-aware reorder planner's signature plans (general A*A, A*B,
A*A^T; src/reorder.h:2046-2204): the library computes the row and column
tile signatures on the GPU and sorts every axis by five stable radix passes;
the reference's own planner, compiled from its sources (oracle/_ref, thrust
kernels), runs on the same GPU beside it.  Permutations, estimates, ratios,
flags, mode and reason must be equal; the applied plan's product is
bit-identical to the oracle's on the permuted operands and, restored, equal
to the unpermuted product up to the rounding of the reordered sums."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(oracle):
    if not oracle.ref_reorder_available():
        pytest.skip("oracle/_ref/libtsgref_reorder.so not built")
    return oracle


def _same(o, got, want):
    for f in o.PLAN_FIELDS + ("mode", "risk_reason"):
        assert got[f] == want[f], (f, got[f], want[f])
    for ax in ("row_perm", "inner_perm", "col_perm"):
        np.testing.assert_array_equal(got[ax], want[ax], err_msg=ax)


def _cases(gen):
    st = gen.permute_symmetric(gen.stencil_27pt_3d(20, seed=1), gen.random_symmetric_permutation(8000, seed=2))
    rm = gen.rmat(13, 8, seed=3)
    pa = gen.random_poisson(3000, 2000, 5.0, seed=4)
    pb = gen.random_poisson(2000, 2500, 3.0, seed=5)
    bd = gen.banded(2000, 30, seed=6)
    big = gen.random_poisson(70000, 70000, 3.0, seed=7)
    empty_rows = gen.random_poisson(1000, 1000, 0.3, seed=8)           # many empty rows and columns
    return [("AA", st, None), ("AA", rm, None), ("AA", big, None), ("AA", empty_rows, None),
            ("AB", pa, pb), ("AB", pa, bd), ("AB", bd, pb), ("AAT", pa, gen.transpose(pa)),
            ("AAT", rm, gen.transpose(rm))]


def test_signature_plans_equal_the_references(tsg, ref, gen):
    modes = set()
    for kind, A, B in _cases(gen):
        st, want = ref.ref_build_reorder_plan(kind, A, B, symmetric=False)
        assert st == 0, kind
        got = tsg.build_reorder_plan(kind, "tasa", A, B, symmetric=False)
        _same(ref, got, want)
        modes.add(want["mode"])
    assert modes & {"active_general", "active_ab", "active_aat"}, modes


def test_forced_signature_plan_gives_the_same_product(tsg, ctx, ref, gen, oracle, monkeypatch):
    monkeypatch.setenv("TASA_FORCE_ACTIVE", "1")
    A = gen.rmat(12, 8, seed=9)
    st, want = ref.ref_build_reorder_plan("AA", A, None, symmetric=False)
    got = tsg.build_reorder_plan("AA", "tasa", A, None, symmetric=False)
    assert st == 0 and got["risk_reason"] == "accepted_force"
    _same(ref, got, want)
    Ar = tsg.apply_bipermutation_csr(A, got["row_perm"], got["inner_perm"])
    Br = tsg.apply_bipermutation_csr(A, got["inner_perm"], got["col_perm"])
    C, _ = tsg.spgemm_csr_host(ctx, Ar, Br)
    perm_c = oracle.gustavson(Ar, Br)          # the permuted product: bit for bit
    for k in (2, 3):
        np.testing.assert_array_equal(C[k], perm_c[k])
    assert np.array_equal(np.asarray(C[4]).view(np.uint64), np.asarray(perm_c[4]).view(np.uint64))
    m, n, rp, ci, v = tsg.restore_bipermutation_csr(C, got["row_perm"], got["col_perm"])
    want_c = oracle.gustavson(A, A)
    np.testing.assert_array_equal(rp, want_c[2])
    np.testing.assert_array_equal(ci, want_c[3])
    # the inner order changes each sum's order: equal up to rounding of
    # sums of U(-1,1) products (absolute, as entries near zero cancel)
    np.testing.assert_allclose(v, want_c[4], rtol=1e-12, atol=1e-14)
