"""tsg_spgemm_csr_host_into: C computed into caller host buffers, the copy of
C's CSR overlapping the numeric step chunk by chunk.  Every result must equal
the oracle (bit for bit) and the two-phase call, whatever the chunking, the
step-3 kernel (SPA in chunks, or the tile kernel first) and the sizes."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gustavson_equal(oracle, matA, matB, got):
    G = oracle.gustavson(matA, matB)
    m, n, rp, ci, v = got
    np.testing.assert_array_equal(rp, G[2])
    np.testing.assert_array_equal(ci, G[3])
    assert np.array_equal(np.asarray(v).view(np.uint64), G[4].view(np.uint64))


@pytest.fixture
def pinned_out(tsg):
    return tsg.HostResultBuffers(1, 1)


def _cases(gen):
    band = gen.banded(4000, 40, seed=3)
    return [
        ("stencil 32^3 (several chunks, SPA)", gen.stencil_27pt_3d(32, seed=1), None),
        ("hypersparse A*B (two chunks)", gen.random_poisson(60000, 30000, 6.0, seed=2),
         gen.random_poisson(30000, 25000, 6.0, seed=4)),
        ("dense tiles (tile kernel first)", band, band),
        ("R-MAT 12 A*A^T", gen.rmat(12, 16, seed=5), "T"),
    ]


@pytest.mark.parametrize("sched", [("spa", 8, 512), ("tiles", 8, 512), ("rows", 16, 1024)])
def test_overlapped_call_matches_oracle_and_two_phase(tsg, ctx, oracle, gen, pinned_out, sched):
    ctx.set_schedule(*sched)
    try:
        for name, A, B in _cases(gen):
            if isinstance(B, str):
                B = gen.transpose(A)
            got, info = tsg.spgemm_csr_host_overlap(ctx, A, B, pinned_out)
            _gustavson_equal(oracle, A, B if B is not None else A, got)
            two = tsg.HostResultBuffers(A[0], 1)
            ref, _ = tsg.spgemm_csr_host_into(ctx, A, B, two)
            for x, y in zip(got[2:], ref[2:]):
                assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8)), name
            assert info["nnz_C"] == got[3].size
    finally:
        ctx.set_schedule("spa", 8, 512)


def test_capacity_is_reported_and_nothing_written(tsg, ctx, gen):
    A = gen.stencil_27pt_3d(12, seed=0)
    m, n, rp, ci, v = (A[0], A[1], np.ascontiguousarray(A[2], np.int32), np.ascontiguousarray(A[3], np.int32),
                       np.ascontiguousarray(A[4], np.float64))
    c_rp = np.zeros(m + 1, np.int32)
    c_ci = np.full(8, -7, np.int32)
    c_v = np.full(8, -7.0)
    nnz = ctypes.c_int(0)
    info = tsg.TsgInfo()
    st = tsg.lib().tsg_spgemm_csr_host_into(ctx.handle, m, n, n, ci.size, rp.ctypes.data, ci.ctypes.data,
                                            v.ctypes.data, ci.size, rp.ctypes.data, ci.ctypes.data, v.ctypes.data,
                                            c_rp.ctypes.data, c_ci.ctypes.data, c_v.ctypes.data, 8,
                                            ctypes.byref(nnz), ctypes.byref(info))
    assert st == tsg.TSG_ERR_OVERFLOW
    assert nnz.value > 8
    assert (c_ci == -7).all() and (c_v == -7.0).all()
    # grown buffers: the same call succeeds
    out = tsg.HostResultBuffers(m, nnz.value)
    got, _ = tsg.spgemm_csr_host_overlap(ctx, A, None, out)
    assert got[3].size == nnz.value and got[2][-1] == nnz.value


def test_empty_and_tiny_products(tsg, ctx, oracle, gen, pinned_out):
    empty = (5, 6, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0))
    B = gen.random_poisson(6, 9, 2.0, seed=9)
    got, info = tsg.spgemm_csr_host_overlap(ctx, empty, B, pinned_out)
    assert info["nnz_C"] == 0 and (got[2] == 0).all() and got[3].size == 0
    one = (1, 1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([3.0]))
    got, _ = tsg.spgemm_csr_host_overlap(ctx, one, None, pinned_out)
    assert list(got[2]) == [0, 1] and list(got[3]) == [0] and got[4][0] == 9.0
    small = gen.random_poisson(37, 41, 3.0, seed=1)
    small_b = gen.random_poisson(41, 29, 3.0, seed=2)
    got, _ = tsg.spgemm_csr_host_overlap(ctx, small, small_b, pinned_out)
    _gustavson_equal(oracle, small, small_b, got)
