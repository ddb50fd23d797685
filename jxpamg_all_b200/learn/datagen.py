"""Training data for the learned settings.

Systems: seeded variants of the config-0/config-1 reservoir Jacobians (2x2
BSR): grids drawn from 16x16x8 .. 60x110x40 (capped in cell count, half of
them with a channelised lower part), 60x220 slabs of the config-1 geometry,
full 60x220x85 config-1 geometries with other seeds than the benchmark's, and
three-phase black-oil variants (3x3 BSR, the config-4 family: True-IMPES
decoupling, GMRES(60), the plain CPR stage-2 weights) on the small grids.  Each
system is solved by the mixed CPR-GMRES path of the measured configuration
(FP32 preconditioner, flexible GMRES, chunk-ordered stage 2, Chebyshev-3 on
the dense levels) once per candidate setting (18) -- strength threshold of level 0,
strength threshold of the coarser levels, Chebyshev interval -- and once with
the plain smoothers.  The label of a system is the candidate with the lowest
cost = iterations x modelled bytes per iteration (bytes moved by the
preconditioner levels, stage 2 and the GMRES operations, from the operator
sizes of that hierarchy): iteration counts alone would always favour the
densest hierarchy.
"""
from __future__ import annotations

import numpy as np

from .. import synth
from ..solver import CprGmres

# (theta level 0, theta levels >= 1, Chebyshev lower, Chebyshev upper); the library snaps
# predictions to these values (csrc/learned.cu), so the two lists must agree
CANDIDATES = [(t0, tc, lo, hi) for t0 in (0.25, 0.5) for tc in (0.25, 0.5, 0.7)
              for (lo, hi) in ((0.1, 1.2), (0.3, 1.1), (0.5, 1.2))]
# the measured path's preconditioner (FP32 storage, the reference mixed driver's stage-2 weights);
# layouts not autotuned and graphs off, so that a training solve sets up quickly
MIXED = dict(decouple=1, k_dim=30, max_iter=300, tol=1e-6, stage2_maxit=3, smoother_order=1, coarse_exact=0,
             precision=1, flexible=1, autotune=0, graphs=0, stage2_relax_weight=1.0, stage2_omega=0.8)
# the three-phase family's method (True-IMPES, GMRES(60), the plain CPR stage-2 weights)
MIXED3 = dict(MIXED, decouple=5, k_dim=60, max_iter=1000, stage2_relax_weight=0.7, stage2_omega=0.9)
MAX_CELLS = 100_000


SLAB_BASE, FULL_BASE, THREE_BASE = 20000, 30000, 40000


def variant_options(idx):
    """The solver options of system idx's family."""
    return MIXED3 if THREE_BASE <= idx < THREE_BASE + 10000 else MIXED


def system_variant(idx, base_seed=20240):
    """Seeded training / evaluation system number idx.

    idx < 20000: config-0-like grids (16..60 x 16..110 x 8..40, <= MAX_CELLS cells);
    20000 <= idx < 30000: config-1 slabs, 60 x 220 x (10..40) with a channelised lower part;
    30000 <= idx < 40000 or idx >= 50000: full config-1 geometry (60 x 220 x 85, 50 channelised layers)
    with other seeds;
    40000 <= idx < 50000: three-phase grids drawn as the config-0-like ones (Sg, gas viscosity of config 4).
    """
    rng = np.random.default_rng(base_seed + idx)
    if THREE_BASE <= idx < THREE_BASE + 10000:
        while True:
            nx, ny, nz = int(rng.integers(16, 61)), int(rng.integers(16, 111)), int(rng.integers(8, 31))
            if nx * ny * nz <= MAX_CELLS:
                break
        ch = int(round(nz * rng.uniform(0.3, 0.7))) if rng.random() < 0.5 else 0
        return synth.reservoir_system(nx, ny, nz, seed=base_seed + 7919 * idx, phases=3, channelised_layers=ch)
    if idx >= FULL_BASE:
        return synth.reservoir_system(60, 220, 85, seed=base_seed + 7919 * idx, phases=2, channelised_layers=50)
    if idx >= SLAB_BASE:
        nz = int(rng.integers(10, 41))
        ch = int(round(nz * 50 / 85))
        return synth.reservoir_system(60, 220, nz, seed=base_seed + 7919 * idx, phases=2, channelised_layers=ch)
    while True:
        nx, ny, nz = int(rng.integers(16, 61)), int(rng.integers(16, 111)), int(rng.integers(8, 41))
        if nx * ny * nz <= MAX_CELLS:
            break
    ch = int(round(nz * rng.uniform(0.3, 0.7))) if rng.random() < 0.5 else 0
    return synth.reservoir_system(nx, ny, nz, seed=base_seed + 7919 * idx, phases=2, channelised_layers=ch)


def iteration_bytes(G, s, precision=2, k_dim=30):
    """Modelled bytes one GMRES iteration moves with the hierarchy of G."""
    xb = 8 if precision == 0 else 4
    tb = 8 if precision == 0 else 4
    passes = {1: 6, 2: 8, 3: 6}  # matrix passes per V-cycle: colour GS, l1-Jacobi, Chebyshev-3 (+ residual)
    total = 0.0
    L = G.num_levels()
    for lev in range(L - 1):
        n, _, nnz = G.level_sizes(lev, 0)
        info = G.level_info(lev)
        vb = {0: 8, 1: 4, 2: 2}[info["storage"]]
        total += passes.get(info["smoother"], 6) * (nnz * (vb + 4) + 3 * n * xb)
        for what in (1, 2):
            nr, nc_, nz_ = G.level_sizes(lev, what)
            total += nz_ * (tb + 4) + (nr + nc_) * xb
    ncoarse = G.level_sizes(L - 1, 0)[0]
    total += ncoarse * ncoarse * 8
    bs, nb, nnzb = s.block_size, s.num_block_rows, s.nnzb
    vb2 = 8 if precision == 0 else 4
    total += 3 * (nnzb * (bs * bs * vb2 + 4) + nb * bs * 8 * 4)   # stage 2
    total += nnzb * (bs * bs * 8 + 4) + 2 * s.n * 8                # GMRES SpMV
    total += (k_dim // 2) * 4 * s.n * 8                             # average orthogonalisation passes
    return total


def solve_case(s, dev, options):
    """Set up and solve one system; returns (iterations, converged, cost, features, thetas, solver stats)."""
    import torch

    G = CprGmres(**options)
    G.set_stream(torch.cuda.current_stream().cuda_stream)
    G.setup(dev["ia"].data_ptr(), dev["ja"].data_ptr(), dev["a"].data_ptr(), s.block_size, nb=s.num_block_rows,
            nnzb=s.nnzb, device=True)
    dev["x"].zero_()
    _, it, rel, conv = G.solve(dev["b"].data_ptr(), dev["x"].data_ptr(), device=True)
    torch.cuda.synchronize()
    L = G.num_levels()
    feats = [G.level_features(lev) for lev in range(L - 1)]
    thetas = [G.level_info(lev)["theta"] for lev in range(L - 1)]
    cost = it * iteration_bytes(G, s, options.get("precision", 0), options.get("k_dim", 30)) if conv else float("inf")
    status = G.learned_status() if options.get("fast_smoother") == 2 else None
    G.close()
    return dict(iters=int(it), converged=bool(conv), rel=float(rel), cost=float(cost),
                features=[None if f is None else f.tolist() for f in feats], thetas=thetas, learned=status)


def upload(s):
    import torch

    d = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).cuda()  # noqa: E731
    return dict(ia=d(s.ia), ja=d(s.ja), a=d(s.a), b=d(s.b), x=torch.zeros(s.n, dtype=torch.float64, device="cuda"))


def candidate_options(c, base=None):
    t0, tc, lo, hi = c
    return dict(MIXED if base is None else base, fast_smoother=1, strong_threshold=float(t0),
                strong_threshold_coarse=float(tc), cheb_lower=float(lo), cheb_upper=float(hi), record_features=1)


def generate(indices, log=print):
    """Solve every candidate on the systems `indices`; returns a list of records."""
    records = []
    for idx in indices:
        s = system_variant(idx)
        base = variant_options(idx)
        dev = upload(s)
        res = []
        for c in CANDIDATES:
            r = solve_case(s, dev, candidate_options(c, base))
            r["candidate"] = list(c)
            res.append(r)
        plain = solve_case(s, dev, dict(base, fast_smoother=0, record_features=1))
        best = int(np.argmin([r["cost"] for r in res]))
        records.append(dict(index=int(idx), shape=[s.nx, s.ny, s.nz], cells=s.num_block_rows, results=res,
                            plain=plain, best=best))
        log(f"system {idx}: {s.nx}x{s.ny}x{s.nz} best {CANDIDATES[best]} iters {res[best]['iters']} "
            f"cost ratio vs plain {res[best]['cost'] / plain['cost']:.3f}")
    return records


def compact(records):
    """Training runs as arrays: cost / iters [S, C], plain cost / iters [S], features [S, C, L, 16]
    (NaN-padded), candidate settings [C, 4], cells [S]."""
    S, C = len(records), len(CANDIDATES)
    L = max(len(r["features"]) for rec in records for r in rec["results"])
    feats = np.full((S, C, L, 16), np.nan, np.float32)
    cost = np.zeros((S, C))
    iters = np.zeros((S, C), np.int32)
    for si, rec in enumerate(records):
        for ci, r in enumerate(rec["results"]):
            cost[si, ci] = r["cost"]
            iters[si, ci] = r["iters"]
            for lev, f in enumerate(r["features"]):
                if f is not None:
                    feats[si, ci, lev] = f
    return dict(cost=cost, iters=iters, feats=feats, candidates=np.asarray(CANDIDATES, np.float64),
                plain_cost=np.array([rec["plain"]["cost"] for rec in records]),
                plain_iters=np.array([rec["plain"]["iters"] for rec in records], np.int32),
                cells=np.array([rec["cells"] for rec in records], np.int64))


def merge(a, b):
    """Concatenate two compact run sets (feature arrays padded to the deeper hierarchy)."""
    L = max(a["feats"].shape[2], b["feats"].shape[2])

    def pad(f):
        out = np.full(f.shape[:2] + (L, 16), np.nan, np.float32)
        out[:, :, :f.shape[2]] = f
        return out

    m = {k: np.concatenate([a[k], b[k]]) for k in ("cost", "iters", "plain_cost", "plain_iters", "cells")}
    m["feats"] = np.concatenate([pad(a["feats"]), pad(b["feats"])])
    m["candidates"] = a["candidates"]
    return m


def dataset(runs, eps=0.02):
    """Per-level samples X [N,16], T [N,3] (target logits): every candidate whose cost is within
    (1 + eps) of the system's best contributes the features of its own hierarchy, labelled with its
    settings, so that near-ties average out instead of picking one arbitrarily."""
    from .model import to_logits

    X, T = [], []
    cand = runs["candidates"]
    for si in range(runs["cost"].shape[0]):
        c = runs["cost"][si]
        best = np.min(c)
        if not np.isfinite(best):
            continue
        for ci in np.nonzero(c <= best * (1.0 + eps))[0]:
            t0, tc, lo, hi = cand[ci]
            for lev in range(runs["feats"].shape[2]):
                f = runs["feats"][si, ci, lev]
                if np.isnan(f).any():
                    break
                X.append(f)
                T.append(to_logits(t0 if lev == 0 else tc, lo, hi))
    return np.asarray(X, np.float32), np.asarray(T, np.float32)
