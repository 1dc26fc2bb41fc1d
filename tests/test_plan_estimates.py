"""Reorder-plan tile-count estimates on the host (no GPU): the reference
samples 24 evenly strided tile rows and scales (src/reorder.h:785-975,
src/external_reorder.h:143-171).  The library's estimates, the oracle's
restatement and -- when oracle/_ref holds it -- the reference's own code,
compiled from its sources, agree exactly, for A*A, A*A^T and A*B problems
under original, random and ordering-like permutations, and the library's
original-order plan equals the reference's field for field."""
import ctypes

import numpy as np
import pytest

from conftest import load_oracle, load_package


@pytest.fixture(scope="module")
def cases():
    load_package()
    import rw_spgemm_b200.generators as gen
    rng = np.random.default_rng(17)
    out = []
    st = gen.permute_symmetric(gen.stencil_27pt_3d(12, seed=1), gen.random_symmetric_permutation(1728, 5))
    rm = gen.rmat(11, 8, seed=4)                           # hub rows
    pb = gen.random_poisson(1000, 1000, 5.0, seed=6)
    bd = gen.banded(1000, 7, seed=7)
    for A, B, kind in ((st, None, "AA"), (rm, None, "AA"), (st, gen.transpose(st), "AAT"),
                       (rm, gen.transpose(rm), "AAT"), (pb, bd, "AB"), (bd, pb, "AB")):
        n = A[0]
        ident = np.arange(n)
        deg = np.argsort(-np.diff(A[2]), kind="stable")   # an ordering-like permutation
        for rp_, cp_ in ((ident, ident), (rng.permutation(n), None), (deg, None)):
            cp_ = rp_ if cp_ is None and kind != "AB" else (cp_ if cp_ is not None else rng.permutation(n))
            out.append((kind, A, B, rp_, rp_, cp_))
    return out


def test_library_estimates_equal_the_oracle_restatement(cases):
    tsg, o = load_package(), load_oracle()
    for kind, A, B, r, i, c in cases:
        got = tsg.reorder_estimates(kind, A, B, r, i, c)
        want = o.reorder_estimates(kind, A, B if B is not None else A, r, i, c)
        assert got == want, (kind, got, want)


def test_oracle_restatement_equals_the_reference_estimators(cases):
    o = load_oracle()
    if not o.ref_reorder_available():
        pytest.skip("oracle/_ref/libtsgref_reorder.so not built (reference tree absent when oracle/Makefile ran)")
    for kind, A, B, r, i, c in cases:
        assert o.reorder_estimates(kind, A, B if B is not None else A, r, i, c) == \
            o.ref_reorder_estimates(kind, A, B, r, i, c), kind


@pytest.mark.parametrize("kind", ["AA", "AAT", "AB"])
def test_original_plan_equals_the_references(cases, kind):
    tsg, o = load_package(), load_oracle()
    if not o.ref_reorder_available():
        pytest.skip("oracle/_ref/libtsgref_reorder.so not built")
    A, B = next((A, B) for k, A, B, *_ in cases if k == kind)
    plan = tsg.build_reorder_plan(kind, "original", A, B)
    R = o.rrlib()
    hA = o._CSRHold(A)
    hB = o._CSRHold(B) if B is not None else hA
    info = o.OReorderInfo()
    R.ref_reorder_info_init(ctypes.byref(info))
    assert R.ref_build_original_reorder_plan({"AA": 0, "AAT": 1, "AB": 2}[kind], ctypes.byref(hA.om),
                                             ctypes.byref(hB.om), ctypes.byref(info)) == 0
    for f in o.ESTIMATE_FIELDS + ("shared_symmetric_csr", "guard_degraded_to_identity", "enabled", "n"):
        assert plan[f] == getattr(info, f), f
    assert plan["mode"] == info.mode.decode() and plan["risk_reason"] == info.risk_reason.decode()
