"""Continuous-batching server: every job's result equals the oracle, is the
same (bit for bit) alone and inside a mix of concurrently arriving jobs, and
memory admission rejects a job that cannot fit while the others complete."""
import random
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def srv_mod(tsg):
    import rw_spgemm_b200.serve as s
    return s


def _matrices(gen):
    mats = {}
    for i in range(5):
        mats[f"p{i}"] = gen.random_poisson(400 + 97 * i, None, 5.0 + i, seed=i)
    mats["b0"] = gen.banded(700, 12, seed=1)
    mats["l0"] = gen.laplacian_2d(25, 28)
    mats["r0"] = gen.rmat(10, 8, seed=5)
    return mats


def _jobs(mats, rng, n):
    keys = [k for k in mats]
    out = []
    for _ in range(n):
        a = rng.choice(keys)
        if rng.random() < 0.5:
            out.append(("AAT", a, None))
        else:
            cands = [k for k in keys if mats[k][0] == mats[a][1]]
            out.append(("AB", a, rng.choice(cands)))
    return out


def _run(srv_mod, mats, jobs, slots=2, max_batch=16, gap=0.0005, mem_cap=8 << 30):
    srv = srv_mod.SpGEMMServer(0, mem_cap=mem_cap, slots=slots, max_batch=max_batch)
    for k, m in mats.items():
        srv.register(k, m)
    srv.start()
    futs = []
    for kind, a, b in jobs:
        futs.append(srv.submit(kind, a, b))
        if gap:
            time.sleep(random.random() * gap)
    res = [f.result(timeout=120) for f in futs]
    stats = srv.stats()
    srv.close()
    return res, stats


def test_server_results_match_oracle_and_are_identical_alone(srv_mod, gen, oracle):
    mats = _matrices(gen)
    rng = random.Random(3)
    jobs = _jobs(mats, rng, 40)
    mixed, stats = _run(srv_mod, mats, jobs)
    assert stats["jobs"] == 40 and stats["p99_ms"] >= stats["p50_ms"] > 0
    for (kind, a, b), C in zip(jobs, mixed):
        B = gen.transpose(mats[a]) if kind == "AAT" else mats[b]
        G = oracle.gustavson(mats[a], B)
        np.testing.assert_array_equal(np.asarray(C[2]), G[2])
        np.testing.assert_array_equal(np.asarray(C[3]), G[3])
        assert np.array_equal(np.asarray(C[4]).view(np.uint64), G[4].view(np.uint64))
    # the same jobs alone, one at a time, in a fresh server
    for idx in (0, 7, 19, 33):
        alone, _ = _run(srv_mod, mats, [jobs[idx]], slots=1, max_batch=1, gap=0)
        for x, y in zip(alone[0][2:], mixed[idx][2:]):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))


def test_admission_rejects_what_cannot_fit(srv_mod, gen):
    mats = {"small": gen.random_poisson(300, None, 3.0, seed=1), "big": gen.banded(20000, 60, seed=2)}
    srv = srv_mod.SpGEMMServer(0, mem_cap=24 << 20, slots=2, max_batch=8)
    for k, m in mats.items():
        srv.register(k, m)
    srv.start()
    f_big = srv.submit("AB", "big", "big")
    f_small = [srv.submit("AAT", "small") for _ in range(5)]
    with pytest.raises(MemoryError):
        f_big.result(timeout=60)
    for f in f_small:
        f.result(timeout=60)
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_concurrent_submitters(srv_mod, gen):
    mats = _matrices(gen)
    srv = srv_mod.SpGEMMServer(0, mem_cap=8 << 30, slots=3, max_batch=8)
    for k, m in mats.items():
        srv.register(k, m)
    srv.start()
    futs, lock = [], threading.Lock()

    def client(seed):
        rng = random.Random(seed)
        for kind, a, b in _jobs(mats, rng, 15):
            f = srv.submit(kind, a, b)
            with lock:
                futs.append(f)

    ts = [threading.Thread(target=client, args=(s,)) for s in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for f in futs:
        f.result(timeout=120)
    st = srv.stats()
    srv.close()
    assert st["jobs"] == 60 and st["batches"] >= 2


def test_device_delivery_matches_host_delivery(srv_mod, gen):
    mats = _matrices(gen)
    jobs = _jobs(mats, random.Random(11), 12)
    res = {}
    for mode in ("host", "device"):
        srv = srv_mod.SpGEMMServer(0, mem_cap=8 << 30, slots=2, max_batch=8, deliver=mode)
        for k, m in mats.items():
            srv.register(k, m)
        srv.start()
        futs = [srv.submit(kind, a, b) for kind, a, b in jobs]
        res[mode] = [f.result(timeout=120) for f in futs]
        srv.close()
    for h, d in zip(res["host"], res["device"]):
        assert h[0] == d[0] and h[1] == d[1]
        for x, y in zip(h[2:], d[2:]):
            assert np.array_equal(np.asarray(x).view(np.uint8), y.cpu().numpy().view(np.uint8))


def test_operand_bytes_match_the_pool(tsg, ctx, gen):
    """The admission's operand size (tsg_tiled_device_bytes) is what the
    library holds: the pool's bytes in use grow by it (within the pool's own
    rounding) when a B-role operand -- tiles, column view, column masks, row
    view -- is made resident; the tile-data-only count is far below it."""
    import torch
    mat = gen.rmat(17, 16, seed=4)
    torch.cuda.synchronize()
    ctx.synchronize()
    before = ctx.pool_used()
    T = tsg.csr_host_to_tiled(ctx, mat, tsg.TSG_TILED_CSC_VIEW)
    ctx.synchronize()
    grown = ctx.pool_used() - before
    dev = T.device_bytes
    tile_data_only = (T.s.tilem + 1) * 4 + T.numtile * 68 + T.nnz * 9 + (T.s.tilen + 1) * 4
    print(f"pool grew {grown} bytes, device_bytes {dev}, tile data only {tile_data_only}")
    assert abs(grown - dev) <= 0.02 * dev + (1 << 20)
    assert tile_data_only < 0.75 * dev
    T.free()
    ctx.synchronize()


def test_auto_schedule_server_matches_the_fixed_one(srv_mod, gen):
    mats = _matrices(gen)
    jobs = _jobs(mats, random.Random(3), 40)
    fixed, _ = _run(srv_mod, mats, jobs, gap=0.0)
    srv = srv_mod.SpGEMMServer(0, mem_cap=8 << 30, slots=2, max_batch=16, schedule="auto")
    for k, m in mats.items():
        srv.register(k, m)
    srv.start()
    res = [f.result(timeout=300) for f in [srv.submit(*j) for j in jobs]]
    st = srv.stats()
    srv.close()
    assert st["tuned"], "no batch was tuned"
    for a, b in zip(res, fixed):
        for x, y in zip(a[2:], b[2:]):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
