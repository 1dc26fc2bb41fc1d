"""Row-partitioned product on the GPU: each rank's tile-row range of A
(partition by predicted products, B whole) multiplied block by block on the
device, the pieces of all ranks of a 4-rank world computed one after the
other on this GPU (ranks never wait on each other: the only collective is
the offsets all-gather after the product, covered on CPU by
tests/test_shard.py), assembled and compared with the oracle -- structure
bit-exact, values bit-identical."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
NTHREADS = max(1, os.cpu_count() or 1)


@pytest.mark.parametrize("scale,ef,kind", [(14, 16, "AA"), (15, 8, "AAT")])
def test_pieces_of_a_4_rank_world_assemble_to_the_product(tsg, ctx, gen, oracle, scale, ef, kind):
    import rw_spgemm_b200.shard as sh
    A = gen.rmat(scale, ef, seed=2)
    B = A if kind == "AA" else gen.transpose(A)

    def multiply(sub, Bm):
        C, _ = tsg.spgemm_csr_host(ctx, sub, Bm)
        return C[2], C[3], C[4]

    world = 4
    pieces = [sh.compute_piece(A, B, r, world, multiply, budget=5e6) for r in range(world)]
    assert sum(p.rows for p in pieces) == A[0]
    whole = sh.assemble(pieces)
    want = oracle.gustavson(A, B, nthreads=NTHREADS)
    np.testing.assert_array_equal(whole[2], want[2])
    np.testing.assert_array_equal(whole[3], want[3])
    assert np.array_equal(np.asarray(whole[4]).view(np.uint64), np.asarray(want[4]).view(np.uint64))
