"""Seeded synthetic media and sources for the benchmark configurations.

The reference reads no dataset for this path; its media are analytic
(Source/functions.cpp:1362-1456).  The configurations are stood in for by
seeded synthetic fields with the stated shapes and value ranges:

  * background c = 1500 + 1500 * depth / L_depth (linear gradient to
    3000 m/s), with depth along y: the reference's own linear model puts its
    gradient in x,y and keeps the medium invariant in z, the axis its FFT
    preconditioner diagonalises;
  * three Gaussian anomalies, amplitude uniform in +-20 %, radius uniform in
    8h..15h, centres uniform in the interior;
  * Gaussian point sources (sigma = 1.5 h) normalised to integral -1 (the
    reference's point source -1/(hx hy hz) integrates to -1,
    Source/functions.cpp:4576).

Random numbers come from one splitmix64 stream (Steele, Lea & Flood 2014):
state += 0x9E3779B97F4A7C15, then two xor-shift-multiply rounds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MASK = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.state = seed & MASK

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / 9007199254740992.0))

    def randint(self, lo: int, hi: int) -> int:
        """Uniform integer in [lo, hi]."""
        return lo + int(self.uniform() * (hi - lo + 1)) if hi > lo else lo


@dataclass
class Problem:
    """One Mode N solve: grid sizes, PML, step, frequency, s^2 and sources."""

    nx: int
    ny: int
    nz: int
    h: float
    pml: int
    omega: float
    s2: np.ndarray                 # (nz, ny, nx) float64 squared slowness
    sources: list                  # list of (i, j, k) float grid positions
    beta_phys: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    def rhs(self, src_index: int = 0, sigma_h: float = 1.5) -> np.ndarray:
        return gaussian_source(self.shape, self.h, self.sources[src_index], sigma_h)


def gaussian_source(shape, h: float, pos, sigma_h: float = 1.5) -> np.ndarray:
    """exp(-r^2 / (2 sigma^2)) at grid position ``pos`` = (i, j, k), scaled
    to sum(f) * h^3 = -1; truncated at 5 sigma."""
    nz, ny, nx = shape
    i0, j0, k0 = pos
    sig = sigma_h
    ax = [np.arange(n, dtype=np.float64) for n in (nx, ny, nz)]
    gx = np.exp(-((ax[0] - i0) ** 2) / (2 * sig * sig))
    gy = np.exp(-((ax[1] - j0) ** 2) / (2 * sig * sig))
    gz = np.exp(-((ax[2] - k0) ** 2) / (2 * sig * sig))
    for g_, c in ((gx, i0), (gy, j0), (gz, k0)):
        g_[np.abs(np.arange(g_.size) - c) > 5 * sig] = 0.0
    f = gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    f *= -1.0 / (f.sum() * h ** 3)
    return f.astype(np.complex128)


def anomalies(rng: SplitMix64, shape, pml: int, h: float, count: int = 3, amp: float = 0.2,
              rmin: float = 8.0, rmax: float = 15.0):
    """Multiplicative Gaussian anomaly field 1 + sum_a A_a exp(-r^2/(2 R_a^2))."""
    nz, ny, nx = shape
    field_ = np.ones(shape, dtype=np.float64)
    k = np.arange(nz, dtype=np.float64)[:, None, None]
    j = np.arange(ny, dtype=np.float64)[None, :, None]
    i = np.arange(nx, dtype=np.float64)[None, None, :]
    params = []
    for _ in range(count):
        a = rng.uniform(-amp, amp)
        r = rng.uniform(rmin, rmax)
        ci = rng.uniform(pml, nx - 1 - pml)
        cj = rng.uniform(pml, ny - 1 - pml)
        ck = rng.uniform(pml, nz - 1 - pml)
        field_ += a * np.exp(-((i - ci) ** 2 + (j - cj) ** 2 + (k - ck) ** 2) / (2 * r * r))
        params.append((a, r, ci, cj, ck))
    return field_, params


def layered_medium(nx, ny, nz, h, pml, seed, n_anom=3, amp=0.2, ppw=8.0, n_sources=1,
                   c_top=1500.0, c_bottom=3000.0, src_random=True) -> Problem:
    """The heterogeneous recipe: linear depth (y) gradient plus anomalies."""
    rng = SplitMix64(seed)
    shape = (nz, ny, nx)
    y = np.arange(ny, dtype=np.float64)
    depth = np.clip((y - pml) / max(1, ny - 1 - 2 * pml), 0.0, 1.0)
    c_bg = c_top + (c_bottom - c_top) * depth
    mult, params = anomalies(rng, shape, pml, h, count=n_anom, amp=amp)
    c = c_bg[None, :, None] * mult
    c_min = float(c.min())
    omega = 2.0 * math.pi * c_min / (ppw * h)
    s2 = 1.0 / (c * c)
    sources = []
    for s in range(n_sources):
        if src_random:
            sources.append((rng.uniform(pml + 4, nx - 5 - pml), rng.uniform(pml + 4, ny - 5 - pml),
                            rng.uniform(pml + 4, nz - 5 - pml)))
        else:
            sources.append(((nx - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0))
    return Problem(nx, ny, nz, h, pml, omega, s2, sources,
                   meta={"seed": seed, "anomalies": params, "c_min": c_min, "ppw": ppw})


def config_c1() -> Problem:
    """64^3 homogeneous c = 1500 m/s, h = 10 m, PML 8, 10 ppw, centred source."""
    n, h, pml = 64, 10.0, 8
    c = 1500.0
    omega = 2.0 * math.pi * c / (10.0 * h)
    s2 = np.full((n, n, n), 1.0 / (c * c))
    return Problem(n, n, n, h, pml, omega, s2, [((n - 1) / 2.0,) * 3], meta={"config": "C1"})


def config_c2(n: int = 128, pml: int = 12, seed: int = 2024) -> Problem:
    p = layered_medium(n, n, n, 10.0, pml, seed, ppw=8.0)
    p.meta["config"] = "C2"
    return p


def config_c3(n: int = 160, pml: int = 12, seed: int = 2024) -> Problem:
    p = layered_medium(n, n, n, 10.0, pml, seed, ppw=8.0)
    p.meta["config"] = "C3"
    return p


def config_small(n: int = 32, pml: int = 6, seed: int = 7, ppw: float = 8.0, n_sources: int = 1) -> Problem:
    """Small heterogeneous case for parity tests."""
    p = layered_medium(n, n, n, 10.0, pml, seed, ppw=ppw, n_sources=n_sources,
                       amp=0.2)
    p.meta["config"] = f"small{n}"
    return p


def config_c4(seed: int = 4044):
    """The batched configuration: 16 seeded sources on a 96^3 medium plus 8
    uneven grids (48^3, 64x80x72, 112x96x64 and 5 more with sides drawn
    from the multiples of 8 in 48..112), each with its own seeded
    heterogeneous medium (depth gradient, three +-20 % anomalies), an
    8-point PML and one seeded source.  Returns the list of Problems, the
    96^3 one first; sizes are (nx, ny, nz)."""
    rng = SplitMix64(seed)
    sizes = [(48, 48, 48), (64, 80, 72), (112, 96, 64)]
    while len(sizes) < 8:
        sizes.append(tuple(8 * rng.randint(6, 14) for _ in range(3)))
    probs = [layered_medium(96, 96, 96, 10.0, 8, seed + 1, ppw=8.0, n_sources=16)]
    for q, (nx, ny, nz) in enumerate(sizes):
        probs.append(layered_medium(nx, ny, nz, 10.0, 8, seed + 2 + q, ppw=8.0, n_sources=1))
    for q, p in enumerate(probs):
        p.meta["config"] = "C4" if q == 0 else f"C4-uneven{q}"
    return probs


def config_c5(n: int = 200, pml: int = 16, seed: int = 5055, n_sources: int = 8, n_recv: int = 50):
    """The gradient configuration: a true model (depth gradient plus three
    +-10 % Gaussian anomalies) that synthesises the data, the starting model
    (the same depth gradient without anomalies, at the same frequency), 8
    seeded sources and n_recv x n_recv receivers on the plane j = pml + 2
    (the top of the interior; depth runs along y), spread evenly over the
    interior in x and z.  Returns (start, true, recv) with recv the linear
    grid indices (k*ny + j)*nx + i as int64."""
    true = layered_medium(n, n, n, 10.0, pml, seed, amp=0.1, ppw=8.0, n_sources=n_sources)
    start = layered_medium(n, n, n, 10.0, pml, seed, n_anom=0, ppw=8.0, n_sources=0)
    start.omega = true.omega
    start.sources = list(true.sources)
    xs = np.linspace(pml + 1, n - 2 - pml, n_recv).round().astype(np.int64)
    j = pml + 2
    kk, ii = np.meshgrid(xs, xs, indexing="ij")
    recv = ((kk * n + j) * n + ii).ravel().astype(np.int64)
    true.meta["config"] = "C5-true"
    start.meta["config"] = "C5-start"
    return start, true, recv
