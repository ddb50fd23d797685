"""A C program written against the reference's interface (tests/dropin/driver.c,
the call sequence of the reference's CPR-GMRES driver) linked with
libjxcpr_b200.so: it reaches the same solution as the library's own API, bit
for bit, through the BSR text and binary readers, and JXFPAMG_Solver_Interface
(solver 220) solves the same system handed over as 1-based scalar CSR."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from jxpamg_all_b200.solver import CprGmres
from tests.dropin_util import build_driver, bsr_to_scalar_csr, write_bsr_binary, write_bsr_text

pytestmark = pytest.mark.gpu


def _run(exe, *args, env=None):
    p = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stderr + p.stdout
    it = int(p.stdout.split()[1])
    return it


@pytest.mark.parametrize("name", ["small", "c0", "tiny3"])
@pytest.mark.parametrize("fmt", ["bsr", "bin"])
def test_reference_driver_sequence_matches_api(tmp_path, systems, name, fmt):
    s = systems(name)
    exe = build_driver(tmp_path)
    A = tmp_path / ("A.txt" if fmt == "bsr" else "A.bin")
    (write_bsr_text if fmt == "bsr" else write_bsr_binary)(str(A), s)
    s.b.tofile(tmp_path / "b.bin")
    it = _run(exe, fmt, A, tmp_path / "b.bin", tmp_path / "x.bin", 1)
    x = np.fromfile(tmp_path / "x.bin")
    G = CprGmres(decouple=1, k_dim=30, max_iter=300, tol=1e-6).setup(s.ia, s.ja, s.a, s.block_size)
    xg, itg, _, conv = G.solve(s.b)
    assert conv and it == itg and np.array_equal(x, xg)
    # and the reference library itself needs the same number of iterations (exact-order path)
    if oracle.ref_available():
        r = oracle.ref_gmres(s.ia, s.ja, s.a, s.block_size, s.b, decouple=1, tol=1e-6, max_iter=300)
        assert r["iters"] == it


def test_driver_honours_environment_options(tmp_path, systems):
    s = systems("c0")
    exe = build_driver(tmp_path)
    write_bsr_text(str(tmp_path / "A.txt"), s)
    s.b.tofile(tmp_path / "b.bin")
    env = dict(os.environ, JXCPR_OPTIONS="smoother_order=1,coarse_exact=0,precision=1,flexible=1")
    it = _run(exe, "bsr", tmp_path / "A.txt", tmp_path / "b.bin", tmp_path / "x.bin", 1, env=env)
    x = np.fromfile(tmp_path / "x.bin")
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    res = b - oracle.bsr_matvec(s.ia, s.ja, a, s.block_size, x)
    assert it > 0 and np.linalg.norm(res) <= 1.05e-6 * np.linalg.norm(b)


@pytest.mark.parametrize("name", ["small", "c0"])
def test_solver_interface_csr_220(tmp_path, systems, name):
    s = systems(name)
    exe = build_driver(tmp_path)
    ia, ja, a = bsr_to_scalar_csr(s, one_based=True, diag_last=True)
    ia.tofile(tmp_path / "ia.bin")
    ja.tofile(tmp_path / "ja.bin")
    a.tofile(tmp_path / "a.bin")
    s.b.tofile(tmp_path / "b.bin")
    it = _run(exe, "csr", tmp_path / "ia.bin", tmp_path / "ja.bin", tmp_path / "a.bin", tmp_path / "b.bin",
              tmp_path / "x.bin", s.n, s.block_size)
    x = np.fromfile(tmp_path / "x.bin")
    # the same system through the library's API with case 220's settings (no decoupling, one stage-2 sweep)
    G = CprGmres(decouple=0, k_dim=30, max_iter=1000, tol=1e-6, stage2_maxit=1).setup(s.ia, s.ja, s.a,
                                                                                     s.block_size)
    xg, itg, _, conv = G.solve(s.b)
    assert conv and it == itg and np.array_equal(x, xg)
