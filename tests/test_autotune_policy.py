"""The autotuner's host logic: every candidate is timed, the fastest kept and
set on the context, the choice cached by the batch-feature key (a second call
does not time again) and persisted to / reloaded from its JSON file.  The
product itself is a stand-in; the GPU tests time the real kernels."""
import pytest


@pytest.fixture
def at(tsg):
    import rw_spgemm_b200.autotune as a
    return a


class FakeC:
    def free(self):
        pass


class FakeCtx:
    def __init__(self):
        self.schedule = None
        self.timing = False

    def set_timing(self, on):
        self.timing = on

    def set_schedule(self, *cand):
        self.schedule = tuple(cand)


def test_tune_single_picks_caches_and_persists(at, monkeypatch, tmp_path):
    cost = {("spa", 8, 512, 0): 3.0, ("spa", 8, 512, 32): 3.5, ("spa", 8, 512, 128): 2.5, ("spa", 8, 512, 257): 2.9,
            ("elems", 8, 512, 0): 5.0, ("tiles", 8, 512, 0): 4.0, ("rows", 16, 1024, 0): 1.5,
            ("rows", 8, 256, 0): 2.0, ("rows", 32, 2048, 0): 9.0}
    runs = []

    def fake_spgemm(ctx, A, B):
        runs.append(ctx.schedule)
        return FakeC(), {"ms_total": cost[ctx.schedule]}

    monkeypatch.setattr(at, "spgemm", fake_spgemm)
    monkeypatch.setattr(at, "product_bounds", lambda ctx, A, B: (10_000, 400))
    path = tmp_path / "tune.json"
    tuner = at.Autotuner(str(path))
    ctx = FakeCtx()
    choice = tuner.tune_single(ctx, "A", "B", reps=1)
    assert choice == ("rows", 16, 1024, 0) and ctx.schedule == choice
    assert set(runs) == set(cost) and len(runs) == 2 * len(cost)          # reps + 1 runs per candidate
    assert tuner.last_timings == cost and ctx.timing is False
    # cached: no timing on the second call, and a fresh tuner reads the file
    runs.clear()
    assert tuner.tune_single(ctx, "A", "B") == choice and not runs
    again = at.Autotuner(str(path))
    assert again.tune_single(FakeCtx(), "A", "B") == choice and not runs
    assert at.summarize(cost)["rows-16-1024"] == 1.5 and at.summarize(cost)["spa-8-512-d128"] == 2.5
    assert at.normalize(("spa", 8, 512)) == ("spa", 8, 512, 0)


def test_batch_key_separates_sizes(at, monkeypatch):
    sizes = {"small": (1_000, 100), "big": (10_000_000, 100_000)}
    monkeypatch.setattr(at, "product_bounds", lambda ctx, A, B: sizes[A])
    assert at.batch_key(None, [("small", None)]) != at.batch_key(None, [("big", None)])
    assert at.batch_key(None, [("small", None)] * 4) != at.batch_key(None, [("small", None)])
