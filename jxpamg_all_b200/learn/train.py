"""Train the learned-settings MLP on the GPU and export its weights.

    python -m jxpamg_all_b200.learn.train --systems 110 --slabs 40 --full 8 --three 40 \
        --holdout 8 --holdout-three 6 --holdout-full 4 --out-dir DIR

1. datagen.generate: every training system is solved with each candidate
   setting (18 candidates + the plain smoothers: 19 solves per system);
2. the per-level features of the candidates within 2 % of each system's
   lowest cost, labelled with their settings (as logits), form the training set;
3. full-batch Adam on the library's own CUDA kernels (jxcpr_mlp_loss_grad,
   jxcpr_mlp_adam) -- no autograd, no framework optimiser;
4. held-out systems are solved with the learned settings (fast_smoother 2,
   with the convergence-factor fallback), the default Chebyshev settings and
   the plain smoothers, and the modelled costs are compared;
5. outputs: learned_weights.inc (the initialiser compiled into the library),
   weights.npz, runs.npz (the training runs) and report.json in DIR.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import time

import numpy as np

from .. import lib
from . import datagen
from .model import N_OUT, N_WEIGHTS, init_weights, write_weights_inc


def train_mlp(X, T, steps=800, lr=3e-3, seed=0, log=print):
    """Full-batch Adam with the jxcpr_mlp_* kernels; returns (weights, loss history)."""
    import torch

    so = lib.load()
    rng = np.random.default_rng(seed)
    mu = X.mean(axis=0)
    sigma = X.std(axis=0) + 1e-3
    w0 = init_weights(rng, mu, sigma)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    w, x, t = dev(w0), dev(X), dev(T)
    B = X.shape[0]
    grad = torch.zeros(N_WEIGHTS, dtype=torch.float32, device="cuda")
    m = torch.zeros_like(grad)
    v = torch.zeros_like(grad)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    work = torch.zeros(B * 134, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    P = lambda tt: ctypes.c_void_p(tt.data_ptr())  # noqa: E731
    hist = []
    for step in range(1, steps + 1):
        lib.check(so.jxcpr_mlp_loss_grad(P(w), P(x), P(t), B, P(grad), P(loss), P(work), st))
        lib.check(so.jxcpr_mlp_adam(P(w), P(grad), P(m), P(v), ctypes.c_float(lr), ctypes.c_float(0.9),
                                    ctypes.c_float(0.999), ctypes.c_float(1e-8), step, st))
        if step == 1 or step % 100 == 0:
            torch.cuda.synchronize()
            hist.append((step, float(loss.item())))
            log(f"step {step} loss {hist[-1][1]:.5f}")
    torch.cuda.synchronize()
    return w.cpu().numpy(), hist


def evaluate(indices, weights, log=print):
    """Learned vs default Chebyshev vs plain smoothers on held-out systems (modelled cost, iterations)."""
    so = lib.load()
    wbuf = np.ascontiguousarray(weights, np.float32)
    lib.check(so.jxcpr_mlp_set_weights(wbuf.ctypes.data_as(ctypes.c_void_p)))
    out = []
    for idx in indices:
        s = datagen.system_variant(idx)
        base = datagen.variant_options(idx)
        dev = datagen.upload(s)
        learned = datagen.solve_case(s, dev, dict(base, fast_smoother=2))
        cheb = datagen.solve_case(s, dev, dict(base, fast_smoother=1, record_features=1))
        plain = datagen.solve_case(s, dev, dict(base, fast_smoother=0, record_features=1))
        rec = dict(index=int(idx), cells=s.num_block_rows, learned=learned, chebyshev_default=cheb, plain=plain)
        out.append(rec)
        log(f"holdout {idx}: cost learned/cheb {learned['cost'] / cheb['cost']:.3f} "
            f"learned/plain {learned['cost'] / plain['cost']:.3f} iters {learned['iters']}/{cheb['iters']}/"
            f"{plain['iters']} learned used {learned['learned']}")
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--systems", type=int, default=110)
    ap.add_argument("--holdout", type=int, default=16)
    ap.add_argument("--steps", type=int, default=800)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--out-dir", required=True)
    ap.add_argument("--runs", help="start from the training runs of an earlier generation (runs.npz)")
    ap.add_argument("--slabs", type=int, default=0, help="60x220 slabs of the config-1 geometry to add")
    ap.add_argument("--full", type=int, default=0, help="full config-1 geometries (other seeds) to add")
    ap.add_argument("--three", type=int, default=0, help="three-phase (3x3, config-4 family) systems to add")
    ap.add_argument("--holdout-three", type=int, default=0, help="held-out three-phase systems")
    ap.add_argument("--holdout-full", type=int, default=0, help="held-out full config-1 geometries")
    args = ap.parse_args(argv)
    import torch

    torch.cuda.set_device(0)
    os.makedirs(args.out_dir, exist_ok=True)
    t0 = time.time()
    runs = None
    if args.runs:
        d = np.load(args.runs, allow_pickle=False)
        runs = {k: d[k] for k in d.files}
    indices = list(range(args.systems)) if not args.runs else []
    indices += [datagen.SLAB_BASE + i for i in range(args.slabs)]
    indices += [datagen.FULL_BASE + i for i in range(args.full)]
    indices += [datagen.THREE_BASE + i for i in range(args.three)]
    if indices:
        new = datagen.compact(datagen.generate(indices))
        runs = new if runs is None else datagen.merge(runs, new)
        np.savez_compressed(os.path.join(args.out_dir, "runs.npz"), **runs)
    X, T = datagen.dataset(runs)
    t_data = time.time() - t0
    w, hist = train_mlp(X, T, steps=args.steps, lr=args.lr)
    t_train = time.time() - t0 - t_data
    # held-out systems (never in the training runs): config-0-like grids, three-phase grids, full
    # config-1 geometries
    hold_idx = [5000 + i for i in range(args.holdout)]
    hold_idx += [datagen.THREE_BASE + 5000 + i for i in range(args.holdout_three)]
    hold_idx += [100000 + i for i in range(args.holdout_full)]
    holdout = evaluate(hold_idx, w)
    np.savez(os.path.join(args.out_dir, "weights.npz"), w=w)
    n_sys = int(runs["cost"].shape[0])
    n_solves = n_sys * (runs["cost"].shape[1] + 1)
    write_weights_inc(os.path.join(args.out_dir, "learned_weights.inc"), w,
                      f"Trained on {n_sys} seeded config-0/1/4-family variants ({n_solves} solves), {X.shape[0]} "
                      f"level samples, {args.steps} full-batch Adam steps; final loss {hist[-1][1]:.5f}.")
    ratio = lambda key: float(np.mean([h[key]["cost"] / h["plain"]["cost"] for h in holdout]))  # noqa: E731
    vs_cheb = [h["learned"]["cost"] / h["chebyshev_default"]["cost"] for h in holdout]
    best = np.min(runs["cost"], axis=1)
    report = dict(systems=n_sys, solves=n_solves,
                  train_mean_best_cost_ratio_vs_plain=float(np.mean(best / runs["plain_cost"])), samples=int(X.shape[0]), outputs=N_OUT,
                  loss_history=hist, data_seconds=t_data, train_seconds=t_train,
                  holdout_mean_cost_ratio_learned_vs_plain=ratio("learned"),
                  holdout_mean_cost_ratio_cheb_default_vs_plain=ratio("chebyshev_default"),
                  holdout_mean_cost_ratio_learned_vs_cheb_default=float(np.mean(vs_cheb)),
                  holdout_learned_used=int(sum(bool(h["learned"]["learned"]["learned_used"]) for h in holdout)),
                  holdout=[dict(index=h["index"], cells=h["cells"],
                                iters=[h["learned"]["iters"], h["chebyshev_default"]["iters"], h["plain"]["iters"]],
                                cost=[h["learned"]["cost"], h["chebyshev_default"]["cost"], h["plain"]["cost"]],
                                learned_status=h["learned"]["learned"])
                           for h in holdout])
    json.dump(report, open(os.path.join(args.out_dir, "report.json"), "w"), indent=1)
    print(json.dumps({k: v for k, v in report.items() if k not in ("holdout", "loss_history")}))


if __name__ == "__main__":
    main()
