"""The learned-settings MLP kernels against the numpy oracle, and what the
trained network gains over the same mixed-precision method without it."""
import ctypes

import numpy as np
import pytest
import torch

from jxpamg_all_b200 import lib
from jxpamg_all_b200.learn import datagen, model
from oracle import mlp

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _weights(seed):
    rng = np.random.default_rng(seed)
    w = model.init_weights(rng, rng.standard_normal(16) * 0.1, rng.uniform(0.5, 2, 16))
    w[model.OFF_B1:] += (rng.standard_normal(model.N_WEIGHTS - model.OFF_B1) * 0.1).astype(np.float32)
    return w.astype(np.float32)


def test_forward_matches_oracle():
    so = lib.load()
    rng = np.random.default_rng(0)
    w = _weights(0)
    X = rng.standard_normal((50, 16)).astype(np.float32)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    wd, xd = d(w), d(X)
    Y = torch.zeros(50, 3, device="cuda")
    H = torch.zeros(50, 64, device="cuda")
    lib.check(so.jxcpr_mlp_forward(_p(wd), _p(xd), 50, _p(H), _p(Y), ctypes.c_void_p(0)))
    Yo, Ho, _ = mlp.forward(w, X)
    assert np.allclose(Y.cpu().numpy(), Yo, rtol=1e-5, atol=1e-5)
    assert np.allclose(H.cpu().numpy(), Ho, rtol=1e-5, atol=1e-5)
    # the host forward the setup uses agrees with the device kernel
    y1 = np.zeros(3, np.float32)
    lib.check(so.jxcpr_mlp_forward_host(w.ctypes.data_as(ctypes.c_void_p), X[3].ctypes.data_as(ctypes.c_void_p),
                                        y1.ctypes.data_as(ctypes.c_void_p)))
    assert np.allclose(y1, Yo[3], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("B", [1, 37, 400])
def test_gradient_matches_oracle(B):
    so = lib.load()
    rng = np.random.default_rng(B)
    w = _weights(B)
    X = rng.standard_normal((B, 16)).astype(np.float32)
    T = rng.standard_normal((B, 3)).astype(np.float32)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    wd, xd, td = d(w), d(X), d(T)
    g = torch.zeros(model.N_WEIGHTS, device="cuda")
    loss = torch.zeros(1, device="cuda")
    work = torch.zeros(B * 134, device="cuda")
    lib.check(so.jxcpr_mlp_loss_grad(_p(wd), _p(xd), _p(td), B, _p(g), _p(loss), _p(work), ctypes.c_void_p(0)))
    torch.cuda.synchronize()
    lo, go = mlp.loss_grad(w, X, T)
    assert abs(loss.item() - lo) <= 1e-5 * max(1.0, lo)
    gd = g.cpu().numpy()
    assert np.all(gd[:model.OFF_W1] == 0)
    assert np.allclose(gd, go, rtol=1e-4, atol=1e-5 * np.max(np.abs(go)))


def test_adam_matches_oracle():
    so = lib.load()
    rng = np.random.default_rng(5)
    w = _weights(5)
    g = rng.standard_normal(model.N_WEIGHTS).astype(np.float32)
    m = (rng.standard_normal(model.N_WEIGHTS) * 0.01).astype(np.float32)
    v = np.abs(rng.standard_normal(model.N_WEIGHTS) * 0.01).astype(np.float32)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    wd, gd, md, vd = d(w), d(g), d(m), d(v)
    lib.check(so.jxcpr_mlp_adam(_p(wd), _p(gd), _p(md), _p(vd), ctypes.c_float(3e-3), ctypes.c_float(0.9),
                                ctypes.c_float(0.999), ctypes.c_float(1e-8), 7, ctypes.c_void_p(0)))
    torch.cuda.synchronize()
    # the kernel receives the hyper-parameters as float32: give the oracle the same values
    f = lambda x: float(np.float32(x))  # noqa: E731
    wo, mo, vo = mlp.adam_step(w, g, m, v, f(3e-3), f(0.9), f(0.999), f(1e-8), 7)
    assert np.allclose(wd.cpu().numpy(), wo, rtol=1e-5, atol=1e-6)
    assert np.allclose(md.cpu().numpy(), mo, rtol=1e-5, atol=1e-8)
    assert np.allclose(vd.cpu().numpy(), vo, rtol=1e-5, atol=1e-10)


def test_training_loop_reduces_loss():
    from jxpamg_all_b200.learn.train import train_mlp

    rng = np.random.default_rng(9)
    X = rng.standard_normal((200, 16)).astype(np.float32)
    T = np.stack([np.tanh(X[:, 0]), 0.5 * X[:, 1], np.sin(X[:, 2])], axis=1).astype(np.float32)
    w, hist = train_mlp(X, T, steps=300, lr=1e-2, log=lambda *_: None)
    assert hist[-1][1] < 0.3 * hist[0][1]
    assert np.array_equal(w[:32], np.concatenate([X.mean(0), X.std(0) + 1e-3]).astype(np.float32))


# held-out systems (never in the training runs): config-0-like grids, three-phase grids (the config-4
# family's method), full config-1 geometries with other seeds
HELD_OUT = ([5000 + i for i in range(8)] + [datagen.THREE_BASE + 5000 + i for i in range(6)] +
            [100000 + i for i in range(4)])


def test_trained_network_gain_over_default_chebyshev():
    """What the network adds: on held-out two- and three-phase systems, the learned settings (strength
    thresholds and Chebyshev intervals per level, with the probe / stall fallback) against the same
    mixed path with the default thresholds and Chebyshev intervals (fast_smoother 1), by the modelled cost
    (iterations x modelled bytes per iteration).  The learned settings must cost less on average by more
    than 3 % (the training report of the compiled weights: 0.968)."""
    ratios, used = [], 0
    for idx in HELD_OUT:
        s = datagen.system_variant(idx)
        base = datagen.variant_options(idx)
        dev = datagen.upload(s)
        learned = datagen.solve_case(s, dev, dict(base, fast_smoother=2))
        cheb = datagen.solve_case(s, dev, dict(base, fast_smoother=1, record_features=1))
        assert learned["converged"] and cheb["converged"]
        ratios.append(learned["cost"] / cheb["cost"])
        used += learned["learned"]["learned_used"]
        st = learned["learned"]
        assert 0 < st["factor_learned"] < 1 and 0 < st["factor_plain"] < 1
    mean = float(np.mean(ratios))
    print(f"learned / default Chebyshev modelled cost on held-out systems: {np.round(ratios, 3)} mean {mean:.3f}, "
          f"learned settings kept on {used} of {len(ratios)}")
    assert mean < 0.97


def test_rejected_learned_settings_fall_back_to_the_plain_method():
    """A system of the batch workload on which the learned strength thresholds build a poor
    hierarchy (without the fallback the learned mode needs 300-400 iterations where the plain
    method needs 29).  Either the setup probe rejects the learned settings or the solve stalls
    against the probe's prediction; both replace them by the plain preconditioner (default
    thresholds, plain smoothers), so the solve stays within a small multiple of the plain one."""
    from jxpamg_all_b200 import synth
    from jxpamg_all_b200.solver import CprGmres

    g = synth.batch_grids()
    s = synth.reservoir_system(*g[45], 45)
    base = dict(decouple=1, max_iter=400, smoother_order=1, coarse_exact=0, precision=1, flexible=1)
    P = CprGmres(**dict(base, fast_smoother=0)).setup(s.ia, s.ja, s.a, s.block_size)
    _, it_plain, _, conv_p = P.solve(s.b)
    L = CprGmres(**dict(base, fast_smoother=2)).setup(s.ia, s.ja, s.a, s.block_size)
    x, it, rel, conv = L.solve(s.b)
    st = L.learned_status()
    assert conv_p and conv
    assert it <= 4 * it_plain, (it, it_plain, st, L.learned_fallbacks())
    if st["learned_used"]:
        assert it <= it_plain + 10, (it, it_plain, st)
    else:
        _, it2, _, conv2 = L.solve(s.b)  # later solves run the plain preconditioner from the start
        assert conv2 and it2 <= it_plain + 3, (it2, it_plain)
    for G in (P, L):
        G.close()
