"""tsg_tiled_to_csr_noalloc: tiles -> CSR with its scan scratch in a fixed
device array (no allocation), called through the C ABI.  Its output must
equal tsg_tiled_to_csr's on the same tiled C, on two calls in a row (the
second reuses the scratch the first wrote), the context's allocation count
must not move across a call, an empty C must give rowptr = [0], and a C
larger than the scratch covers must be rejected before any work.  The file
name keeps it last in collection; it also passes run alone."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ROWS = 4096 * 8192


def _noalloc(tsg, ctx, C, rp, ci, v):
    L = tsg.lib()
    f = L.tsg_tiled_to_csr_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(tsg.TsgTiled), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    ptr = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None else None)  # noqa: E731
    return f(ctx.handle, ctypes.byref(C.s), ptr(rp), ptr(ci), ptr(v))


def _product(tsg, ctx, gen, case):
    if case == "poisson_small":
        A = gen.random_poisson(3000, None, 6.0, seed=11)
    elif case == "stencil_multi_block":
        A = gen.stencil_27pt_3d(40)  # 64,000 rows: 8 scan blocks
    elif case == "million_rows":
        A = gen.banded(1000000, 1, seed=6)  # 123 scan blocks: the partial scan spans several warps
    else:
        A = gen.banded(100003, 9, seed=4)  # ragged last block and tile row
    return _tiled_square(tsg, ctx, A)


def _tiled_square(tsg, ctx, A):
    import torch
    m, n, rp, ci, v = A
    d = torch.device("cuda", torch.cuda.current_device())
    T = tsg.csr_to_tiled(ctx, m, n, torch.from_numpy(rp).to(d), torch.from_numpy(ci).to(d),
                         torch.from_numpy(v).to(d), tsg.TSG_TILED_CSC_VIEW)
    C, _ = tsg.spgemm(ctx, T, T)
    T.free()
    return C


@pytest.mark.parametrize("case", ["poisson_small", "stencil_multi_block", "banded_ragged", "million_rows"])
def test_noalloc_matches_tiled_to_csr_twice(tsg, ctx, gen, case):
    import torch
    C = _product(tsg, ctx, gen, case)
    rp0, ci0, v0 = tsg.tiled_to_csr(ctx, C)
    m, nnz = C.s.m, C.s.nnz
    d = rp0.device
    for call in range(2):
        rp = torch.full((m + 1,), -7, dtype=torch.int32, device=d)
        ci = torch.full((max(nnz, 1),), -7, dtype=torch.int32, device=d)
        v = torch.full((max(nnz, 1),), float("nan"), dtype=torch.float64, device=d)
        torch.cuda.synchronize()
        before = ctx.allocations()
        assert _noalloc(tsg, ctx, C, rp, ci, v) == 0, tsg.lib().tsg_last_error()
        assert ctx.allocations() == before, "the no-alloc conversion allocated"
        ctx.synchronize()
        # integer structure bit-exact; values are copies (tolerance 0)
        assert torch.equal(rp, rp0), f"rowptr differs on call {call}"
        assert torch.equal(ci[:nnz], ci0), f"colidx differs on call {call}"
        assert np.array_equal(v[:nnz].cpu().numpy().view(np.uint64), v0.cpu().numpy().view(np.uint64))
    C.free()


def test_noalloc_rejects_more_rows_than_the_scratch_covers(tsg, ctx):
    import torch
    big = tsg.TsgTiled()
    big.m = MAX_ROWS + 1
    big.n = 16
    big.tilem = (big.m + 15) // 16
    big.tilen = 1
    d = torch.device("cuda", torch.cuda.current_device())
    rp = torch.empty(1, dtype=torch.int32, device=d)
    C = type("T", (), {"s": big})()
    st = _noalloc(tsg, ctx, C, rp, rp, rp)
    assert st == -1
    assert b"scratch" in tsg.lib().tsg_last_error()


def test_noalloc_empty_c(tsg, ctx):
    import torch
    empty = tsg.TsgTiled()
    empty.m = 0
    empty.n = 5
    empty.tilem = 0
    empty.tilen = 1
    d = torch.device("cuda", torch.cuda.current_device())
    rp = torch.full((1,), -7, dtype=torch.int32, device=d)
    C = type("T", (), {"s": empty})()
    before = ctx.allocations()
    assert _noalloc(tsg, ctx, C, rp, None, None) == 0, tsg.lib().tsg_last_error()
    assert ctx.allocations() == before
    ctx.synchronize()
    assert int(rp[0]) == 0
