"""The N > 1 plumbing of bench.py on CPU: world-size-2 gloo process group,
max over ranks of the step time, the replica throughput, and the reference
arm's other ranks leaving without work."""
import importlib.util
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b = _bench()
        dist.barrier()
        got = b.max_over_ranks(10.0 + rank, dist, "cpu")
        Path(out_dir, f"rank{rank}").write_text(repr(got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    assert [float((tmp_path / f"rank{r}").read_text()) for r in range(2)] == [11.0, 11.0]


def test_replica_throughput_and_single_process():
    b = _bench()
    assert b.max_over_ranks(3.5) == 3.5
    # 2 ranks x 1e9 products in 10 ms = 400 GFLOP/s for the whole job
    assert b.replica_gflops(1e9, 2, 10.0) == pytest.approx(400.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0
    assert out.stdout.strip() == ""
