"""The server's admission and batching policy, on the host: jobs are taken in
arrival order; a batch closes once its jobs' predicted scalar products reach
the work budget (a single larger job still runs, alone); a job waits while
resident operands + arenas in flight + its predicted bytes would exceed the
memory cap (evicting unpinned operands first), and a job that could never fit
(its predicted bytes plus its own operands above the cap) is rejected with
MemoryError.  The device parts (operand upload, bounds,
batches) are stand-ins; the GPU tests cover them."""
import collections
import threading

import pytest


@pytest.fixture
def serve_mod(tsg):
    import rw_spgemm_b200.serve as s
    return s


class FakeCache:
    def __init__(self, sizes):
        self.sizes = dict(sizes)   # key -> resident bytes once loaded
        self.tiles = collections.OrderedDict()
        self.bytes = 0
        self.evicted = []

    def get(self, key, host_mat):
        if key not in self.tiles:
            self.tiles[key] = key
            self.bytes += self.sizes[key]
        self.tiles.move_to_end(key)
        return key

    def size_of(self, key):
        return self.sizes[key]

    def evict_until(self, limit, pinned_keys):
        for key in list(self.tiles):
            if self.bytes <= limit:
                break
            if key in pinned_keys:
                continue
            self.tiles.pop(key)
            self.bytes -= self.sizes[key]
            self.evicted.append(key)


class FakeBatch:
    def __init__(self, ctx, pairs, *sched, graph=False, dense=0, bounds=None):
        self.pairs = list(pairs)
        self.bounds = bounds
        self.sched = tuple(sched) + (dense,)

    def info(self):
        return {"arena_bytes": 0}

    def run(self):
        pass


class FakeSlot:
    def __init__(self):
        self.ctx = None
        self.batch = None
        self.pending = None
        self.jobs = []
        self.arena = 0
        self.t_launch = 0.0


def make_server(serve_mod, monkeypatch, mem_cap, budget, sizes, predict):
    monkeypatch.setattr(serve_mod, "Batch", FakeBatch)
    srv = serve_mod.SpGEMMServer.__new__(serve_mod.SpGEMMServer)
    srv.deliver, srv.device, srv.mem_cap, srv.max_batch = "device", 0, mem_cap, 64
    srv.batch_products, srv.schedule = float(budget), ("spa", 8, 512)
    srv.tuner, srv.tuned = None, {}
    srv.matrices = {k: None for k in sizes}
    srv.slots = [FakeSlot(), FakeSlot()]
    srv.cache = FakeCache(sizes)
    srv.queue = collections.deque()
    srv.lock = threading.Condition()
    srv.running, srv.thread, srv.next_id = False, None, 0
    srv.done, srv.batches, srv.rejected = [], 0, 0
    srv.host_s = collections.defaultdict(float)
    srv.preds = {}
    srv.classes, srv.lookahead = {}, 256
    srv._predict = lambda A, B: tuple(predict[(A, B)]) + (1,) * (3 - len(predict[(A, B)]))
    srv._predict_many = lambda ops: [srv._predict(A, B) for A, B in ops]
    return srv


def batch_jobs(slot):
    return [j.jid for j in slot.jobs]


def test_work_budget_closes_batches_in_arrival_order(serve_mod, monkeypatch):
    predict = {("a", "b"): (10, 60), ("c", "d"): (10, 60), ("e", "f"): (10, 10), ("g", "h"): (10, 500)}
    srv = make_server(serve_mod, monkeypatch, 10_000, 100, {k: 1 for k in "abcdefgh"}, predict)
    for a, b in [("a", "b"), ("c", "d"), ("e", "f"), ("g", "h")]:
        srv.submit("AB", a, b)
    s0, s1 = srv.slots
    assert srv._form_batch(s0) and batch_jobs(s0) == [0]          # 60 + 60 > 100: job 1 opens the next
    assert srv._form_batch(s1) and batch_jobs(s1) == [1, 2]       # 60 + 10 <= 100; + 500 > 100
    s0.batch = None
    assert srv._form_batch(s0) and batch_jobs(s0) == [3]          # above the budget, alone
    assert srv.batches == 3 and not srv.queue


def test_memory_cap_defers_evicts_and_rejects(serve_mod, monkeypatch):
    sizes = {"a": 300, "b": 300, "x": 300, "y": 300, "p": 10, "q": 10, "u": 450, "v": 450}
    predict = {("a", "b"): (200, 5), ("x", "y"): (300, 5), ("p", "q"): (5000, 5), ("u", "v"): (200, 5)}
    srv = make_server(serve_mod, monkeypatch, 1000, 1e9, sizes, predict)
    f_big = srv.submit("AB", "p", "q")      # predicted 5000 bytes > cap: rejected
    f_ops = srv.submit("AB", "u", "v")      # 200 predicted + 900 of its own operands > cap: rejected
    srv.submit("AB", "a", "b")
    srv.submit("AB", "x", "y")
    s0, s1 = srv.slots
    assert srv._form_batch(s0)
    assert srv.rejected == 2
    assert isinstance(f_big.exception(timeout=0), MemoryError) and isinstance(f_ops.exception(timeout=0), MemoryError)
    # a, b (600 resident) + 200 predicted fit; x, y would need 600 + 600 + 200 + 300: waits
    assert batch_jobs(s0) == [2]
    assert [j.jid for j in srv.queue] == [3]
    # with the first batch still in flight its operands stay pinned: x, y still cannot fit
    assert not srv._form_batch(s1)
    assert "a" not in srv.cache.evicted and "b" not in srv.cache.evicted
    # once it finishes, a and b may be evicted to make room, and the job is admitted
    s0.batch, s0.jobs, s0.arena = None, [], 0
    assert srv._form_batch(s1) and batch_jobs(s1) == [3]
    assert set(srv.cache.evicted) >= {"a", "b"} and srv.cache.bytes + 300 <= 1000


class FakeTuner:
    def __init__(self):
        self.calls = []

    def tune_batch(self, ctx, pairs, reps=2, use_cache=True):
        self.calls.append(len(pairs))
        return ("rows", 16, 1024, 0) if len(self.calls) == 1 else ("spa", 8, 512, 128)


def test_auto_schedule_tunes_once_per_density_class(serve_mod, monkeypatch):
    # (bytes, products, C-tile bound): densities 1 and 1 (class 1), then 100 (class 6)
    predict = {("a", "b"): (10, 50, 50), ("c", "d"): (10, 40, 40), ("e", "f"): (10, 8000, 80)}
    srv = make_server(serve_mod, monkeypatch, 10_000, 60, {k: 1 for k in "abcdef"}, predict)
    srv.schedule, srv.tuner = "auto", FakeTuner()
    s0, s1 = srv.slots
    srv.submit("AB", "a", "b")
    assert srv._form_batch(s0) and s0.batch.sched == ("rows", 16, 1024, 0)
    s0.batch = None
    srv.submit("AB", "c", "d")
    assert srv._form_batch(s0) and s0.batch.sched == ("rows", 16, 1024, 0)   # same class: no new tuning
    assert srv.tuner.calls == [1]
    srv.submit("AB", "e", "f")
    assert srv._form_batch(s1) and s1.batch.sched == ("spa", 8, 512, 128)    # new class: tuned
    assert srv.tuner.calls == [1, 1] and set(srv.tuned) == {1, 6}


def test_operand_bytes_are_the_librarys_allocation(serve_mod):
    class T:
        device_bytes = 12345
    assert serve_mod.OperandCache.tiled_bytes(T()) == 12345


def test_queue_head_with_resident_operands_is_predicted_in_one_call(serve_mod, monkeypatch):
    predict = {("a", "b"): (10, 5), ("c", "d"): (10, 5), ("a", "d"): (10, 5), ("e", "f"): (10, 5)}
    srv = make_server(serve_mod, monkeypatch, 10_000, 1e9, {k: 1 for k in "abcdef"}, predict)
    calls = {"many": [], "one": 0}
    one = srv._predict

    def many(ops):
        calls["many"].append(list(ops))
        return [one(A, B) for A, B in ops]

    def single(A, B):
        calls["one"] += 1
        return one(A, B)
    srv._predict_many, srv._predict = many, single
    for k in "abcd":
        srv.cache.get(k, None)
    for a, b in [("a", "b"), ("c", "d"), ("a", "d"), ("e", "f")]:
        srv.submit("AB", a, b)
    assert srv._form_batch(srv.slots[0]) and batch_jobs(srv.slots[0]) == [0, 1, 2, 3]
    # the three jobs on resident operands in one call, the one that uploads alone
    assert calls["many"] == [[("a", "b"), ("c", "d"), ("a", "d")]] and calls["one"] == 1


def test_batches_are_planned_from_cached_predictions(serve_mod, monkeypatch):
    predict = {("a", "b"): (10, 7, 3), ("c", "d"): (10, 9, 4)}
    srv = make_server(serve_mod, monkeypatch, 10_000, 1e9, {k: 1 for k in "abcd"}, predict)
    n = {"one": 0}
    one = srv._predict

    def counted(A, B):
        n["one"] += 1
        return one(A, B)
    srv._predict = counted
    for a, b in [("a", "b"), ("c", "d"), ("a", "b")]:
        srv.submit("AB", a, b)
    s0, s1 = srv.slots
    assert srv._form_batch(s0) and batch_jobs(s0) == [0, 1, 2]
    # (products, C tiles) per job go to the batch; the repeated pair was predicted once
    assert s0.batch.bounds == [(7, 3), (9, 4), (7, 3)] and n["one"] == 2
    srv.submit("AB", "c", "d")
    assert srv._form_batch(s1) and n["one"] == 2


def test_replacing_an_operand_drops_what_came_from_it(serve_mod, monkeypatch):
    predict = {("a", "b"): (10, 7, 3), ("a", ("a", "T")): (10, 7, 3)}
    srv = make_server(serve_mod, monkeypatch, 10_000, 1e9, {"a": 1, "b": 1, ("a", "T"): 1}, predict)
    srv.matrices = {"a": (1, 1, [0, 0], [], []), "b": None}
    srv.preds = {("a", "b"): (1, 2, 3), ("b", "b"): (4, 5, 6)}
    srv.matrices[("a", "T")] = "old transpose"
    srv.cache.drop = lambda keys: srv.cache.evicted.extend(sorted(map(str, keys)))
    srv.submit("AB", "b", "b")
    srv.register("a", (2, 2, [0, 0, 0], [], []))
    assert ("a", "T") not in srv.matrices and srv.preds == {("b", "b"): (4, 5, 6)}
    assert srv.cache.evicted == ["('a', 'T')", "a"]
    with pytest.raises(RuntimeError):
        srv.register("b", "another")


def test_batches_hold_one_skew_class_and_others_keep_their_places(serve_mod, monkeypatch):
    predict = {(a, a): (10, 40) for a in "abcde"}
    srv = make_server(serve_mod, monkeypatch, 10_000, 100, {k: 1 for k in "abcde"}, predict)
    srv.classes = {"a": 0, "b": 3, "c": 0, "d": 3, "e": 0}
    for a in "abcde":
        srv.submit("AB", a, a)
    s0, s1 = srv.slots
    assert srv._form_batch(s0) and batch_jobs(s0) == [0, 2]        # class 0; 40 + 40 + 40 > 100: e waits
    assert [j.jid for j in srv.queue] == [1, 3, 4]
    assert srv._form_batch(s1) and batch_jobs(s1) == [1, 3]        # class 3
    s0.batch = None
    assert srv._form_batch(s0) and batch_jobs(s0) == [4] and not srv.queue
    srv.lookahead = 1
    for a in "bab":
        srv.submit("AB", a, a)
    s0.batch = None
    assert srv._form_batch(s0) and batch_jobs(s0) == [5]            # looks past one job only
    assert [j.jid for j in srv.queue] == [6, 7]


def test_skew_class_of_a_matrix(serve_mod):
    import numpy as np
    serve = serve_mod
    flat = (4, 4, np.array([0, 2, 4, 6, 8]), np.zeros(8, np.int32), np.ones(8))
    hub = (4, 4, np.array([0, 13, 14, 15, 16]), np.zeros(16, np.int32), np.ones(16))
    empty = (3, 3, np.zeros(4, np.int64), np.zeros(0, np.int32), np.zeros(0))
    assert serve.skew_class(flat) == 0 and serve.skew_class(hub) == 1 and serve.skew_class(empty) == 0


def test_host_delivery_copies_every_result_out_of_the_staging_buffer(serve_mod, monkeypatch):
    """Host delivery hands each job numpy arrays of its own, copied out of
    the slot's reusable staging buffer in pieces on the host pool's threads
    (pieces of at most 16 MB: the values of the second job span several)."""
    import torch
    import numpy as np
    srv = make_server(serve_mod, monkeypatch, 10_000, 1e9, {}, {})
    srv.deliver = "host"
    rng = np.random.default_rng(4)
    shapes = [(5, 3, 7), (1000, 900, 5_000_000), (0, 4, 0)]     # (m, n, nnz)
    layout, total, want = [], 0, []
    jobs = []
    for jid, (m, n, nnz) in enumerate(shapes):
        job = serve_mod.Job(jid, "AB", "a", "b")
        jobs.append(job)
        v_off = total
        rp_off = v_off + 8 * nnz
        ci_off = rp_off + 4 * (m + 1)
        total = (ci_off + 4 * nnz + 7) & ~7
        layout.append((job, None, m, n, nnz, v_off, rp_off, ci_off))
        want.append((np.arange(m + 1, dtype=np.int32) * 3, rng.integers(0, 1 << 30, nnz).astype(np.int32),
                     rng.standard_normal(nnz)))
    staging = torch.zeros(total + 8, dtype=torch.uint8)
    raw = staging.numpy()
    for (job, _, m, n, nnz, v_off, rp_off, ci_off), (rp, ci, v) in zip(layout, want):
        raw[rp_off:rp_off + rp.nbytes] = rp.view(np.uint8)
        raw[ci_off:ci_off + ci.nbytes] = ci.view(np.uint8)
        raw[v_off:v_off + v.nbytes] = v.view(np.uint8)

    class Closing:
        def close(self):
            pass
    slot = FakeSlot()
    slot.staging, slot.pending, slot.batch, slot.jobs = staging, (layout, None), Closing(), jobs
    srv._deliver(slot)
    raw[:] = 0                                              # the staging buffer is reused by the next batch
    for job, (m, n, nnz), (rp, ci, v) in zip(jobs, shapes, want):
        got = job.future.result(timeout=0)
        assert got[0] == m and got[1] == n and job.result_nnz == nnz
        np.testing.assert_array_equal(got[2], rp)
        np.testing.assert_array_equal(got[3], ci)
        assert np.array_equal(got[4].view(np.uint64), v.view(np.uint64))
    assert slot.pending is None and slot.batch is None
    srv._pool.shutdown()
