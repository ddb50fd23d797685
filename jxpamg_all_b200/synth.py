"""Seeded synthetic fully-implicit reservoir Jacobians in block-sparse (BSR) form.

The reference ships no test data (its SPE10 inputs are absent), so every
parity test and benchmark runs on systems made here.  The generator builds a
7-point two-point-flux (TPFA) Jacobian of a black-oil model on an nx*ny*nz
grid:

* unknowns per cell: pressure p, water saturation Sw (and gas saturation Sg
  for the three-phase case); equations per cell: one mass balance per phase;
* permeability: ln k ~ N(0, 2^2) per layer, correlated along x (AR(1) with
  correlation length 5 cells); kz = 0.1 kx.  The "channelised" variant puts a
  binary facies map in the lower layers (channel fraction 0.3, channel
  ln k ~ N(3, 0.5^2), background ln k ~ N(-2, 1.5^2));
* porosity 0.2*exp(0.1 N(0,1)); harmonic-mean transmissibilities;
* Corey relative permeabilities (exponent 2), viscosities water 1 cP,
  oil 5 cP, gas 0.02 cP; Sw ~ U(0.2, 0.8), Sg ~ U(0, 0.3);
* accumulation phi*ct*V/dt with dt = 1 day and ct = 1e-5; off-diagonal
  blocks are the upwinded flux derivatives;
* right-hand side b = A x_true with x_true ~ N(0, 1).

Layout follows the reference BSR container (``jxf_BSRMatrix`` in
jxfpamg-0220/include/jxf_bsr_mv.h:38-50): 0-based block CSR, cell-major
ordering (i fastest), unknowns interleaved per cell, blocks stored
row-major, and the diagonal block FIRST in every block row followed by the
other columns in ascending order (the convention the reference's ABF
decoupling, HGS smoother and strength routine assume).
"""
from __future__ import annotations

import dataclasses

import numpy as np

__all__ = ["BSRSystem", "reservoir_system", "config_system", "CONFIGS", "batch_grids", "batch_systems"]


@dataclasses.dataclass
class BSRSystem:
    """A BSR matrix with its right-hand side and the vector it was made from."""

    nx: int
    ny: int
    nz: int
    block_size: int
    ia: np.ndarray  # int32 [nb+1]
    ja: np.ndarray  # int32 [nnzb]
    a: np.ndarray  # float64 [nnzb*b*b], row-major blocks
    b: np.ndarray  # float64 [nb*b]
    x_true: np.ndarray  # float64 [nb*b]

    @property
    def num_block_rows(self) -> int:
        return int(self.ia.shape[0] - 1)

    @property
    def nnzb(self) -> int:
        return int(self.ja.shape[0])

    @property
    def n(self) -> int:
        return self.num_block_rows * self.block_size


def _ar1_along_x(rng, shape, sigma, corr_len):
    """Stationary AR(1) Gaussian field along the last axis (x)."""
    rho = float(np.exp(-1.0 / corr_len))
    eps = rng.standard_normal(shape)
    out = np.empty(shape)
    out[..., 0] = sigma * eps[..., 0]
    s = sigma * np.sqrt(1.0 - rho * rho)
    for i in range(1, shape[-1]):
        out[..., i] = rho * out[..., i - 1] + s * eps[..., i]
    return out


def _facies(rng, nzf, ny, nx, frac):
    """Binary channel map: smoothed anisotropic noise thresholded to `frac`."""
    g = rng.standard_normal((nzf, ny, nx))
    # long correlation along x, short along y: repeated box smoothing
    for _ in range(3):
        g = (np.roll(g, 1, axis=2) + g + np.roll(g, -1, axis=2)) / 3.0
        g = (np.roll(g, 2, axis=2) + g + np.roll(g, -2, axis=2)) / 3.0
    g = (np.roll(g, 1, axis=1) + 2 * g + np.roll(g, -1, axis=1)) / 4.0
    thr = np.quantile(g, 1.0 - frac, axis=(1, 2), keepdims=True)
    return g > thr


def _harmonic(k1, k2):
    return 2.0 * k1 * k2 / (k1 + k2)


def reservoir_system(nx, ny, nz, seed, phases=2, channelised_layers=0, dtype=np.float64):
    """Build the Jacobian system described in the module docstring.

    ``phases`` is 2 (p, Sw) or 3 (p, Sw, Sg); ``channelised_layers`` is the
    number of bottom layers that carry the binary facies map.
    """
    if phases not in (2, 3):
        raise ValueError("phases must be 2 or 3")
    rng = np.random.default_rng(seed)
    nb = nx * ny * nz
    bs = phases

    # ---- rock properties, array shape (nz, ny, nx) -------------------------
    lnk = _ar1_along_x(rng, (nz, ny, nx), 2.0, 5.0)
    if channelised_layers > 0:
        nzf = min(channelised_layers, nz)
        chan = _facies(rng, nzf, ny, nx, 0.3)
        ch = rng.normal(3.0, 0.5, size=chan.shape)
        bg = rng.normal(-2.0, 1.5, size=chan.shape)
        lnk[nz - nzf:] = np.where(chan, ch, bg)
    kx = np.exp(lnk)
    kz = 0.1 * kx
    phi = 0.2 * np.exp(0.1 * rng.standard_normal((nz, ny, nx)))

    sw = rng.uniform(0.2, 0.8, size=(nz, ny, nx))
    sg = rng.uniform(0.0, 0.3, size=(nz, ny, nx)) if phases == 3 else np.zeros((nz, ny, nx))
    so = np.clip(1.0 - sw - sg, 0.0, 1.0)
    # pressure state: a drive gradient along x plus noise (fixes the upwind directions)
    xs = np.arange(nx, dtype=np.float64)[None, None, :]
    pres = 300.0 - 0.5 * xs + 0.05 * rng.standard_normal((nz, ny, nx))

    mu = np.array([1.0, 5.0, 0.02])
    # Corey exponent 2: kr = s^2, dkr/ds = 2 s
    lam_w, dlam_w = sw ** 2 / mu[0], 2.0 * sw / mu[0]
    lam_o, dlam_o = so ** 2 / mu[1], 2.0 * so / mu[1]  # derivative w.r.t. So
    lam_g, dlam_g = sg ** 2 / mu[2], 2.0 * sg / mu[2]

    V, dt, ct = 1.0, 1.0, 1e-5
    acc = phi * V / dt

    # ---- block diagonal: accumulation ------------------------------------
    # rows = phase equations (w, o[, g]); cols = unknowns (p, Sw[, Sg])
    D = np.zeros((nz, ny, nx, bs, bs))
    D[..., 0, 0] = acc * ct * sw
    D[..., 0, 1] = acc
    D[..., 1, 0] = acc * ct * so
    D[..., 1, 1] = -acc
    if bs == 3:
        D[..., 1, 2] = -acc
        D[..., 2, 0] = acc * ct * sg
        D[..., 2, 2] = acc

    flat = lambda arr: arr.reshape(-1)  # noqa: E731
    cell = np.arange(nb).reshape(nz, ny, nx)
    lam = [flat(lam_w), flat(lam_o), flat(lam_g)]
    dlam = [flat(dlam_w), flat(dlam_o), flat(dlam_g)]
    pf = flat(pres)
    Dflat = D.reshape(nb, bs, bs)

    rows, cols, blks = [], [], []

    def add_links(c1, c2, T):
        """Two-point flux between cell arrays c1 and c2 with transmissibility T."""
        c1, c2, T = flat(c1), flat(c2), flat(T)
        dp = pf[c1] - pf[c2]
        up = np.where(dp >= 0.0, c1, c2)  # upstream cell
        # derivative of the flux F_a = T lam_a(up) (p1 - p2) leaving c1
        for (ci, cj, sgn) in ((c1, c2, 1.0), (c2, c1, -1.0)):
            # equation rows of cell ci, unknowns of cell cj (off-diagonal block)
            B = np.zeros((ci.shape[0], bs, bs))
            Ddiag = np.zeros((ci.shape[0], bs, bs))
            for ph in range(bs):
                lam_up = lam[ph][up]
                # pressure derivatives: dF/dp_ci = T lam, dF/dp_cj = -T lam (sign per side)
                Ddiag[:, ph, 0] += T * lam_up
                B[:, ph, 0] -= T * lam_up
                # saturation derivatives at the upstream cell
                dlu = dlam[ph][up] * sgn * dp * T
                if ph == 0:
                    sat_cols = [(1, 1.0)]
                elif ph == 1:
                    sat_cols = [(1, -1.0)] + ([(2, -1.0)] if bs == 3 else [])
                else:
                    sat_cols = [(2, 1.0)]
                for col, ds in sat_cols:
                    contrib = dlu * ds
                    own = up == ci
                    Ddiag[own, ph, col] += contrib[own]
                    B[~own, ph, col] += contrib[~own]
            np.add.at(Dflat, ci, Ddiag)
            rows.append(ci)
            cols.append(cj)
            blks.append(B)

    add_links(cell[:, :, :-1], cell[:, :, 1:], _harmonic(kx[:, :, :-1], kx[:, :, 1:]))
    add_links(cell[:, :-1, :], cell[:, 1:, :], _harmonic(kx[:, :-1, :], kx[:, 1:, :]))
    add_links(cell[:-1, :, :], cell[1:, :, :], _harmonic(kz[:-1], kz[1:]))

    rows.append(np.arange(nb))
    cols.append(np.arange(nb))
    blks.append(Dflat)
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    B = np.concatenate(blks, axis=0)
    # order: by row, diagonal first, then ascending column
    key_off = (c != r).astype(np.int64)
    order = np.lexsort((c, key_off, r))
    r, c, B = r[order], c[order], B[order]

    ia = np.zeros(nb + 1, dtype=np.int32)
    np.cumsum(np.bincount(r, minlength=nb), out=ia[1:])
    ja = c.astype(np.int32)
    a = np.ascontiguousarray(B.reshape(-1)).astype(dtype)

    x_true = rng.standard_normal(nb * bs)
    b = bsr_matvec_np(ia, ja, a.astype(np.float64), bs, x_true)
    return BSRSystem(nx, ny, nz, bs, ia, ja, a, b, x_true)


def bsr_matvec_np(ia, ja, a, bs, x):
    """y = A x for a BSR matrix (vectorised numpy, used only to form b)."""
    nb = ia.shape[0] - 1
    A = a.reshape(-1, bs, bs)
    xb = x.reshape(-1, bs)
    prod = np.einsum("kij,kj->ki", A, xb[ja])
    rows = np.repeat(np.arange(nb), np.diff(ia))
    y = np.zeros((nb, bs))
    np.add.at(y, rows, prod)
    return y.reshape(-1)


# Workloads: (nx, ny, nz, phases, channelised bottom layers, seed)
CONFIGS = {
    "c0": (20, 40, 10, 2, 0, 0),  # 8,000 cells, 2x2
    "c1": (60, 220, 85, 2, 50, 1),  # 1,122,000 cells, 2x2, channelised lower 50 layers
    "c4": (60, 220, 85, 3, 50, 2),  # 3x3 black-oil variant
    "tiny": (6, 5, 4, 2, 0, 7),  # 120 cells, unit tests
    "small": (12, 10, 6, 2, 2, 3),  # 720 cells, unit tests with facies
    "tiny3": (5, 4, 3, 3, 0, 11),  # 60 cells, 3x3 unit tests
    "slab45": (60, 220, 45, 2, 15, 5),  # 594,000 cells: profiling case, level-0 sweep larger than L2
}


def config_system(name: str) -> BSRSystem:
    nx, ny, nz, ph, ch, seed = CONFIGS[name]
    return reservoir_system(nx, ny, nz, seed, phases=ph, channelised_layers=ch)


# Batched-solve workload: independent two-phase systems built as the 8,000-cell
# log-normal case, system k with seed k, grid sizes drawn uniformly per axis
# between these corners (about 2K to 264K cells).
BATCH_GRID_MIN = (16, 16, 8)
BATCH_GRID_MAX = (60, 110, 40)
BATCH_SIZE_SEED = 2024


def batch_grids(count=64, size_seed=BATCH_SIZE_SEED, grid_min=BATCH_GRID_MIN, grid_max=BATCH_GRID_MAX):
    """The (nx, ny, nz) of each system of the batch, drawn from their own seeded generator."""
    rng = np.random.default_rng(size_seed)
    lo, hi = np.array(grid_min), np.array(grid_max)
    return [tuple(int(v) for v in rng.integers(lo, hi + 1)) for _ in range(count)]


def batch_systems(count=64, first_seed=0, size_seed=BATCH_SIZE_SEED, grid_min=BATCH_GRID_MIN,
                  grid_max=BATCH_GRID_MAX):
    """`count` independent 2x2 systems of uneven size (system k: seed first_seed + k)."""
    return [reservoir_system(nx, ny, nz, first_seed + k)
            for k, (nx, ny, nz) in enumerate(batch_grids(count, size_seed, grid_min, grid_max))]
