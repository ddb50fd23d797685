"""CPU checks of the learned-settings MLP: the numpy oracle against finite
differences, the weight layout / output maps, and the committed training data."""
import json
import os

import numpy as np

from jxpamg_all_b200.learn import datagen, model
from oracle import mlp

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(os.path.dirname(HERE), "jxpamg_all_b200", "learn", "data")


def _rand_weights(rng):
    mu = rng.standard_normal(16) * 0.1
    sg = rng.uniform(0.5, 2.0, 16)
    w = model.init_weights(rng, mu, sg).astype(np.float64)
    w[model.OFF_B1:] += rng.standard_normal(model.N_WEIGHTS - model.OFF_B1) * 0.1
    return w


def test_layout_matches_library_constants():
    assert model.N_WEIGHTS == mlp.N_WEIGHTS == 16 + 16 + 64 * 16 + 64 + 3 * 64 + 3
    rng = np.random.default_rng(0)
    w = _rand_weights(rng).astype(np.float32)
    p = model.unpack(w)
    assert np.array_equal(model.pack(p["mu"], p["sigma"], p["W1"], p["b1"], p["W2"], p["b2"]), w)


def test_output_maps_invert():
    th, lo, hi = np.array([0.25, 0.5, 0.7]), np.array([0.1, 0.3, 0.5]), np.array([1.2, 1.1, 1.2])
    y = model.to_logits(th, lo, hi)
    assert np.allclose(model.theta_of(y[:, 0]), th)
    assert np.allclose(model.lower_of(y[:, 1]), lo)
    assert np.allclose(model.upper_of(y[:, 2]), hi)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    w = _rand_weights(rng)
    X = rng.standard_normal((7, 16))
    T = rng.standard_normal((7, 3))
    loss, g = mlp.loss_grad(w, X, T)
    assert np.all(g[:model.OFF_W1] == 0.0)
    idx = rng.choice(np.arange(model.OFF_W1, model.N_WEIGHTS), 60, replace=False)
    h = 1e-6
    for k in idx:
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (mlp.loss_grad(wp, X, T)[0] - mlp.loss_grad(wm, X, T)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), k


def test_adam_reduces_loss_and_keeps_normalisation():
    rng = np.random.default_rng(2)
    w = _rand_weights(rng)
    X = rng.standard_normal((32, 16))
    T = np.tanh(X[:, :3])
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    l0 = mlp.loss_grad(w, X, T)[0]
    for step in range(1, 201):
        _, g = mlp.loss_grad(w, X, T)
        w2, m, v = mlp.adam_step(w, g, m, v, 1e-2, 0.9, 0.999, 1e-8, step)
        assert np.array_equal(w2[:model.OFF_W1], w[:model.OFF_W1])
        w = w2
    assert mlp.loss_grad(w, X, T)[0] < 0.5 * l0


def test_weights_inc_roundtrip(tmp_path):
    rng = np.random.default_rng(3)
    w = _rand_weights(rng).astype(np.float32)
    p = tmp_path / "w.inc"
    model.write_weights_inc(str(p), w, "test")
    txt = p.read_text()
    body = txt[txt.index("{") + 1:txt.rindex("}")]
    vals = np.array([float(t.strip().rstrip("f")) for t in body.replace("\n", "").split(",") if t.strip()],
                    np.float32)
    assert np.array_equal(vals, w)


def test_committed_training_data():
    d = np.load(os.path.join(DATA, "runs.npz"))
    runs = {k: d[k] for k in d.files}
    S, C = runs["cost"].shape
    assert C == len(datagen.CANDIDATES) and S >= 100
    assert np.allclose(runs["candidates"], np.asarray(datagen.CANDIDATES))
    assert S * (C + 1) >= 2000  # solves behind the training set
    X, T = datagen.dataset(runs)
    assert X.shape[1] == 16 and T.shape[1] == 3 and X.shape[0] > S
    assert np.all(np.isfinite(X)) and np.all(np.isfinite(T))
    th = model.theta_of(T[:, 0])
    assert np.all(np.min(np.abs(th[:, None] - np.array([0.25, 0.5, 0.7])[None]), axis=1) < 1e-3)
    rep = json.load(open(os.path.join(DATA, "training_report.json")))
    assert rep["systems"] == S and rep["samples"] == X.shape[0]
    # the best candidate of each system beats the plain smoothers on average (what there is to learn)
    assert rep["train_mean_best_cost_ratio_vs_plain"] < 0.95


def test_library_weights_are_the_trained_ones():
    inc = os.path.join(os.path.dirname(HERE), "jxpamg_all_b200", "csrc", "learned_weights.inc")
    txt = open(inc).read()
    assert "Trained on" in txt
