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
    def __init__(self, ctx, pairs, *sched, graph=False, dense=0):
        self.pairs = list(pairs)
        self.sched = tuple(sched) + (dense,)

    def info(self):
        return {"arena_bytes": 0}

    def run(self):
        pass


class FakeSlot:
    def __init__(self):
        self.ctx = None
        self.batch = None
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
    srv._predict = lambda A, B: tuple(predict[(A, B)]) + (1,) * (3 - len(predict[(A, B)]))
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
