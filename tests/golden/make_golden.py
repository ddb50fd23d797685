"""Generates tests/golden/*.npz from the reference library compiled from source
(oracle/_ref/libjxf_ref64.so) on the seeded synthetic systems.

    OMP_NUM_THREADS=1 python tests/golden/make_golden.py          # the small systems
    OMP_NUM_THREADS=1 python tests/golden/make_golden.py c1       # the 1,122,000-cell system

For each case: the decoupled system's AMG hierarchy as the reference builds it
(CF markers per level, SHA-256 of every level's A_l / P_l index arrays, value
checksums), one CPR application on a seeded vector, and the full CPR-GMRES(30)
solve to 1e-6 (iterations, residual history, solution).
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from jxpamg_all_b200 import synth  # noqa: E402

CASES = [("small", 1), ("c0", 1), ("c0", 5), ("tiny3", 1)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make(name, decouple):
    s = synth.config_system(name)
    a, b = oracle.ref_bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, decouple)
    R = oracle.RefCPR(s.ia, s.ja, a, s.block_size)
    out = {"num_levels": np.int32(R.num_levels())}
    for lev in range(R.num_levels()):
        ia, ja, av, m = R.level_matrix(lev, 0)
        out[f"A{lev}_n"] = np.int32(len(ia) - 1)
        out[f"A{lev}_nnz"] = np.int32(ia[-1])
        out[f"A{lev}_sha_ia"] = sha(ia)
        out[f"A{lev}_sha_ja"] = sha(ja)
        out[f"A{lev}_sum_abs"] = np.float64(np.abs(av).sum())
        cf = R.level_cf(lev, len(ia) - 1)
        if cf is not None:
            out[f"CF{lev}"] = cf.astype(np.int8)
        P = R.level_matrix(lev, 1)
        if P is not None:
            out[f"P{lev}_sha_ia"] = sha(P[0])
            out[f"P{lev}_sha_ja"] = sha(P[1])
            out[f"P{lev}_sum_abs"] = np.float64(np.abs(P[2]).sum())
    r = np.random.default_rng(123).standard_normal(s.n)
    out["cpr_r"] = r
    out["cpr_z"] = R.apply(r)
    sol = oracle.ref_gmres(s.ia, s.ja, s.a, s.block_size, s.b, decouple=decouple, tol=1e-6, max_iter=300)
    out["gmres_iters"] = np.int32(sol["iters"])
    out["gmres_rel"] = np.float64(sol["rel"])
    out["gmres_norms"] = sol["norms"]
    out["gmres_x"] = sol["x"]
    out["decoupled_rhs_sha"] = sha(b)
    out["decoupled_a_sha"] = sha(a)
    path = os.path.join(HERE, f"{name}_dec{decouple}.npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in out.items()})
    print(path, "levels", R.num_levels(), "iters", sol["iters"])


# The 1,122,000-cell channelised system (60x220x85, 2x2 blocks, seed 1) is too large to store whole:
# its fixture keeps the hierarchy as level sizes and SHA-256 digests (CF markers, A_l / P_l index
# arrays), the solve as iterations, residual history, norms of x and x at X_SAMPLE seeded indices.
X_SAMPLE = 1 << 16
X_SAMPLE_SEED = 2024


def x_sample_index(n):
    return np.sort(np.random.default_rng(X_SAMPLE_SEED).choice(n, size=min(X_SAMPLE, n), replace=False))


def make_large(name, decouple):
    s = synth.config_system(name)
    a, b = oracle.ref_bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, decouple)
    R = oracle.RefCPR(s.ia, s.ja, a, s.block_size)
    out = {"num_levels": np.int32(R.num_levels())}
    for lev in range(R.num_levels()):
        ia, ja, av, m = R.level_matrix(lev, 0)
        n = len(ia) - 1
        out[f"A{lev}_n"] = np.int32(n)
        out[f"A{lev}_nnz"] = np.int32(ia[-1])
        out[f"A{lev}_sha_ia"] = sha(ia)
        out[f"A{lev}_sha_ja"] = sha(ja)
        out[f"A{lev}_sum_abs"] = np.float64(np.abs(av).sum())
        cf = R.level_cf(lev, n)
        if cf is not None:
            out[f"CF{lev}_sha"] = sha(cf.astype(np.int8))
            out[f"CF{lev}_ncoarse"] = np.int32((cf > 0).sum())
        P = R.level_matrix(lev, 1)
        if P is not None:
            out[f"P{lev}_sha_ia"] = sha(P[0])
            out[f"P{lev}_sha_ja"] = sha(P[1])
            out[f"P{lev}_sum_abs"] = np.float64(np.abs(P[2]).sum())
    del R
    sol = oracle.ref_gmres(s.ia, s.ja, s.a, s.block_size, s.b, decouple=decouple, tol=1e-6, max_iter=300)
    x = sol["x"]
    idx = x_sample_index(len(x))
    out["gmres_iters"] = np.int32(sol["iters"])
    out["gmres_rel"] = np.float64(sol["rel"])
    out["gmres_norms"] = sol["norms"]
    out["x_norm2"] = np.float64(np.linalg.norm(x))
    out["x_sum"] = np.float64(x.sum())
    out["x_sample_idx"] = idx.astype(np.int32)
    out["x_sample"] = x[idx]
    out["decoupled_rhs_sha"] = sha(b)
    out["decoupled_a_sha"] = sha(a)
    path = os.path.join(HERE, f"{name}_dec{decouple}.npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in out.items()})
    print(path, "levels", out["num_levels"], "iters", sol["iters"])


if __name__ == "__main__":
    if os.environ.get("OMP_NUM_THREADS") != "1":
        sys.exit("run with OMP_NUM_THREADS=1 (the reference's results depend on the thread count)")
    which = sys.argv[1:] or ["small"]
    if "small" in which:
        for nm, dec in CASES:
            make(nm, dec)
    if "c1" in which:
        make_large("c1", 1)
