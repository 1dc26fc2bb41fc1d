"""The selector's hand-written MLP kernels against the CPU oracle (forward,
gradients, Adam), and the learned choice against exhaustive search."""
import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def mlp_oracle():
    spec = importlib.util.spec_from_file_location("mlp_oracle", ROOT / "oracle" / "mlp_oracle.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def sel(tsg):
    import rw_spgemm_b200.selector as s
    return s


def test_mlp_forward_gradients_and_adam_match_oracle(ctx, sel):
    import torch
    mo = mlp_oracle()
    F, H, O, B = 23, 64, 15, 48
    net = sel.MLP(ctx, F, H, O, seed=3)
    rng = np.random.default_rng(1)
    X = rng.normal(size=(B, F)).astype(np.float32)
    T = rng.normal(size=(B, O)).astype(np.float32)
    M = (rng.random((B, O)) < 0.8).astype(np.float32)
    d = torch.device("cuda", 0)
    Xd, Td, Md = (torch.from_numpy(a).to(d) for a in (X, T, M))
    w0 = net.params().astype(np.float64)
    _, _, y_ref = mo.forward(w0, X.astype(np.float64), F, H, O)
    y = net.forward(Xd).cpu().numpy()
    np.testing.assert_allclose(y, y_ref, rtol=1e-4, atol=1e-4)
    loss = net.step(Xd, Td, Md, lr=0.0)                 # gradients only
    ref_loss, ref_g = mo.loss_and_grads(w0, X, T, M, F, H, O)
    g = net.params(which=1).astype(np.float64)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, ref_loss)
    np.testing.assert_allclose(g, ref_g, rtol=2e-3, atol=2e-5)
    net.step(Xd, Td, Md, lr=1e-2)                       # one Adam step
    w1, _, _ = mo.adam(w0, ref_g, np.zeros_like(w0), np.zeros_like(w0), 1, 1e-2)
    np.testing.assert_allclose(net.params(), w1, rtol=1e-3, atol=1e-5)
    net.close()


def test_mlp_training_reduces_loss(ctx, sel):
    rng = np.random.default_rng(2)
    feats = rng.normal(size=(256, 23)).astype(np.float32)
    W = rng.normal(size=(23, 15))
    targets = np.exp(np.tanh(feats @ W) * 0.5)
    net = sel.MLP(ctx, seed=5)
    losses = net.fit(feats, targets, epochs=60, lr=3e-3)
    assert losses[-1] < 0.3 * losses[0]
    net.close()


def test_selector_beats_fixed_choice_on_held_out(ctx, sel, gen):
    """Trains on method-generated timings of small matrices and checks the
    model's mean regret against the exhaustive best on held-out matrices is
    within 10% (the selector's target), and no worse than the method
    without the model (original order, default accumulator)."""
    mats = sel.training_matrices(gen, 80, seed=11)
    data = [sel.time_configs(ctx, m, repeats=2) for m in mats]
    feats = np.stack([d[0] for d in data])
    times = np.stack([d[1] for d in data])
    tr, te = slice(0, 64), slice(64, 80)
    net = sel.MLP(ctx, seed=7)
    net.fit(feats[tr], times[tr], epochs=300, lr=2e-3)
    picks = np.argmin(net.predict(feats[te]), axis=1)
    r_model = sel.regret(times[te], picks)[0]
    r_plain = sel.regret(times[te], np.zeros(times[te].shape[0], dtype=int))[0]
    print(f"held-out mean regret: model {r_model:.4f}, without the model {r_plain:.4f}")
    assert r_model <= 0.10
    assert r_model <= r_plain
    ch = sel.choose(None, ctx, mats[0])
    assert ch.source == "exhaustive" and ch.config in sel.CONFIGS
    net.close()
