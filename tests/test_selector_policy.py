"""The selector's host logic: the model's pick when the matrix lies inside
the training range, the exhaustive search (also the yardstick of the model's
regret) when there is no model or the features fall outside it; regret is
the relative slowdown against the best configuration.  Features, timings and
the network's forward pass are stand-ins here; the GPU tests run them."""
import numpy as np
import pytest


@pytest.fixture
def sel(tsg):
    import rw_spgemm_b200.selector as s
    return s


class FakeModel:
    def __init__(self, scores, inside=True):
        self.scores, self.inside = np.asarray(scores, np.float32), inside

    def in_range(self, f):
        return self.inside

    def predict(self, f):
        return self.scores[None, :]


def test_choose_model_or_exhaustive(sel, monkeypatch):
    n = len(sel.CONFIGS)
    times = np.linspace(5.0, 1.0, n)  # the last configuration is the fastest
    timed = []
    monkeypatch.setattr(sel, "features", lambda ctx, mat, device=0: np.zeros(4, np.float32))

    def fake_time(ctx, mat, device=0):
        timed.append(mat)
        return None, times, None

    monkeypatch.setattr(sel, "time_configs", fake_time)
    scores = np.arange(n, dtype=np.float32)            # the model prefers the first
    c = sel.choose(FakeModel(scores), None, "m")
    assert c.source == "model" and c.config == sel.CONFIGS[0] and not timed
    c = sel.choose(FakeModel(scores, inside=False), None, "m")
    assert c.source == "exhaustive" and c.config == sel.CONFIGS[n - 1] and timed == ["m"]
    c = sel.choose(None, None, "m2")
    assert c.source == "exhaustive" and c.config == sel.CONFIGS[n - 1] and timed == ["m", "m2"]


def test_in_range_uses_the_training_span(sel):
    m = sel.MLP.__new__(sel.MLP)
    m.lo, m.hi = np.array([0.0, 10.0]), np.array([1.0, 20.0])
    assert m.in_range(np.array([0.5, 15.0]))
    assert m.in_range(np.array([1.4, 24.0]))            # within half a span outside
    assert not m.in_range(np.array([1.6, 15.0]))
    m.lo = None
    assert not m.in_range(np.array([0.5, 15.0]))         # untrained


def test_regret(sel):
    t = np.array([[1.0, 2.0, 4.0], [3.0, 1.5, 6.0]])
    mean, med, worst = sel.regret(t, np.array([0, 1]))
    assert mean == 0.0 and med == 0.0 and worst == 0.0
    mean, med, worst = sel.regret(t, np.array([1, 2]))
    assert worst == pytest.approx(3.0) and mean == pytest.approx((1.0 + 3.0) / 2)
