"""Row-partitioned product over ranks, on CPU: two gloo ranks split A's
tile rows by predicted products (B replicated), each computes its piece
block by block, one all-gather places the pieces, and the pieces
concatenated equal the single-rank product.  The exact CPU multiply of the
oracle stands in for the device product of each block (the GPU runs it in
tests/test_gpu_shard.py); what is checked here is the partition, the block
walk, the offsets and the assembly."""
import os
import pickle
import socket
from pathlib import Path

import numpy as np
import pytest

from conftest import load_oracle, load_package

CASES = [(11, 8, "AA"), (12, 16, "AAT")]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _mats(scale, ef, kind):
    load_package()
    import rw_spgemm_b200.generators as g
    A = g.rmat(scale, ef, seed=3)
    return A, (A if kind == "AA" else g.transpose(A))


def _multiply(sub, B):
    C = load_oracle().gustavson(sub, B)
    return C[2], C[3], C[4]


def _worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        load_package()
        import rw_spgemm_b200.shard as sh
        for scale, ef, kind in CASES:
            A, B = _mats(scale, ef, kind)
            # a small block budget: several blocks per rank
            piece = sh.place(sh.compute_piece(A, B, rank, world, _multiply, budget=2e5), dist)
            got = [None] * world
            dist.all_gather_object(got, piece)
            if rank == 0:
                Path(out_dir, f"{scale}_{ef}_{kind}").write_bytes(pickle.dumps(got))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def pieces(tmp_path_factory):
    import torch.multiprocessing as mp
    out = tmp_path_factory.mktemp("shard")
    mp.spawn(_worker, args=(2, _free_port(), str(out)), nprocs=2, join=True)
    load_package()
    import rw_spgemm_b200.shard  # noqa: F401  (the pickled pieces' class)
    return {c: pickle.loads((out / f"{c[0]}_{c[1]}_{c[2]}").read_bytes()) for c in CASES}


@pytest.mark.parametrize("case", CASES)
def test_ranges_cover_every_tile_row_once_and_balance(pieces, case):
    load_package()
    import rw_spgemm_b200.blocks as blocks
    A, B = _mats(*case)
    ps = pieces[case]
    tilem = (A[0] + 15) // 16
    covered = np.zeros(tilem, np.int64)
    for p in ps:
        covered[p.t0:p.t1] += 1
    assert np.all(covered == 1)
    assert [p.t1 for p in ps[:-1]] == [p.t0 for p in ps[1:]]
    tp = blocks.tile_row_products(A, B)
    shares = np.array([p.products for p in ps], np.float64)
    assert shares.sum() == tp.sum()
    assert shares.max() <= 1.10 * tp.sum() / len(ps)  # within 10% of an equal share


@pytest.mark.parametrize("case", CASES)
def test_pieces_concatenate_to_the_single_rank_product(pieces, case):
    load_package()
    import rw_spgemm_b200.shard as sh
    A, B = _mats(*case)
    ps = pieces[case]
    # offsets from the all-gather agree with the pieces themselves
    row0 = nnz0 = 0
    for p in ps:
        assert (p.row0, p.nnz0) == (row0, nnz0)
        assert p.per_rank == [(q.rows, q.nnz) for q in ps]
        row0 += p.rows
        nnz0 += p.nnz
    assert all(p.nnz_total == nnz0 for p in ps) and row0 == A[0]
    whole = sh.assemble(ps)
    want = load_oracle().gustavson(A, B)
    assert whole[0] == want[0] and whole[1] == want[1]
    np.testing.assert_array_equal(whole[2], want[2])
    np.testing.assert_array_equal(whole[3], want[3])
    assert np.array_equal(np.asarray(whole[4]).view(np.uint64), np.asarray(want[4]).view(np.uint64))


def test_single_rank_piece_is_the_whole_product():
    load_package()
    import rw_spgemm_b200.shard as sh
    A, B = _mats(11, 8, "AA")
    p = sh.place(sh.compute_piece(A, B, 0, 1, _multiply, budget=1e5))
    assert (p.t0, p.t1, p.row0, p.nnz0) == (0, (A[0] + 15) // 16, 0, 0)
    want = load_oracle().gustavson(A, B)
    np.testing.assert_array_equal(p.rowptr, want[2])
    assert p.nnz_total == int(want[2][-1])
