"""Grid descriptor and PML stretching shared by both operators (oracle).

Follows the reference's ``size_m`` (``Source/definitions.h:55-68``), the PML
damping ``d(x)`` (``Source/functions.cpp:893-906``) and ``alpha(size_m,
double)`` (``Source/functions.cpp:1839-1878``), including its left/right
asymmetry at half indices.  Vector layout is ``l = i + nx*j + nx*ny*k``
(x fastest), as ``take_coord3D`` (``Source/functions.cpp:225-230``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

PI = 3.141592653589793238462643  # Source/definitions.h:155


@dataclass
class Axis:
    """One axis of the grid: mirrors ``size_m`` (Source/definitions.h:55-68)."""

    n: int                 # total points on the axis (PML/sponge included)
    h: float               # grid step
    pml_pts: int = 0       # PML points on each end (alpha != 1 there)
    spg_pts: int = 0       # sponge points on each end (Mode R z axis only)
    l: float = 0.0         # axis length as the reference defines it
    n_nopml: int = 0       # physical points

    def __post_init__(self):
        if self.l == 0.0:
            self.l = self.n * self.h
        if self.n_nopml == 0:
            self.n_nopml = self.n - 2 * max(self.pml_pts, self.spg_pts)


def d_pml(x: float) -> float:
    """PML damping profile d(x) = 1000 x^2 (Source/functions.cpp:893-906)."""
    return 1000.0 * x * x


def alpha(ax: Axis, i: float, omega: float) -> complex:
    """PML stretch alpha at (possibly half-) index ``i``.

    Source/functions.cpp:1839-1878: with h = 1/pml, the left layer uses
    x = 1 - i*h for i < pml, the right layer x = 1 + (i - n + 1)*h for
    i >= n - pml, and alpha = -i*omega / (d(x) - i*omega).  The test
    ``i < pml`` puts i = pml - 0.5 inside the left layer while i = n - pml -
    0.5 is outside the right layer (the reference's asymmetry, kept).
    """
    if ax.pml_pts == 0:
        return 1.0 + 0.0j
    h = 1.0 / ax.pml_pts
    if i < ax.pml_pts or i >= (ax.n - ax.pml_pts):
        if i < ax.pml_pts:
            x = 1.0 - i * h
        else:
            x = 1.0 + (i - ax.n + 1) * h
        return complex(0.0, -omega) / complex(d_pml(x), -omega)
    return 1.0 + 0.0j


def pml_coeffs(ax: Axis, omega: float):
    """Per-index second-difference coefficients along one axis.

    Returns complex arrays (cm, cp) of length n with
      cm[i] = alpha(i) alpha(i - 1/2) / h^2   (coefficient of u[i-1])
      cp[i] = alpha(i) alpha(i + 1/2) / h^2   (coefficient of u[i+1])
    and the diagonal contribution -(cm + cp); this is ``beta2D_pml``
    (Source/functions.cpp:2347-2402) cases -1/+1 (x) and -2/+2 (y).
    """
    n = ax.n
    cm = np.empty(n, dtype=np.complex128)
    cp = np.empty(n, dtype=np.complex128)
    h2 = ax.h * ax.h
    for i in range(n):
        a = alpha(ax, float(i), omega)
        cm[i] = a * alpha(ax, i - 0.5, omega) / h2
        cp[i] = a * alpha(ax, i + 0.5, omega) / h2
    return cm, cp


@dataclass
class Grid3D:
    x: Axis
    y: Axis
    z: Axis
    omega: float
    meta: dict = field(default_factory=dict)

    @property
    def shape_zyx(self):
        return (self.z.n, self.y.n, self.x.n)

    @property
    def size(self) -> int:
        return self.x.n * self.y.n * self.z.n

    @property
    def size2d(self) -> int:
        return self.x.n * self.y.n


def reference_grid(n_nopml: int, pml_pts: int, spg_pts: int, length: float = 3200.0,
                   nu: float = 4.0, source_shift: bool = False) -> Grid3D:
    """Mode R grid as ``main`` builds it (Source/main.cpp:95-193).

    x, y: ``n_nopml + 2*pml`` points with PML; z: ``n_nopml + 2*spg`` points,
    no PML, sponge layers.  Without SOURCE_SHIFT: l = L + 2*p*L/n_nopml,
    h = l/n; with it: l = L + 2*p*L/(n_nopml+1), h = l/(n+1).
    """
    n1 = n_nopml + 2 * pml_pts
    n3 = n_nopml + 2 * spg_pts
    if source_shift:
        lx = length + (2.0 * pml_pts * length) / (n_nopml + 1)
        lz = length + (2.0 * spg_pts * length) / (n_nopml + 1)
        hx = lx / (n1 + 1)
        hz = lz / (n3 + 1)
    else:
        lx = length + (2.0 * pml_pts * length) / n_nopml
        lz = length + (2.0 * spg_pts * length) / n_nopml
        hx = lx / n1
        hz = lz / n3
    x = Axis(n=n1, h=hx, pml_pts=pml_pts, l=lx, n_nopml=n_nopml)
    y = Axis(n=n1, h=hx, pml_pts=pml_pts, l=lx, n_nopml=n_nopml)
    z = Axis(n=n3, h=hz, pml_pts=0, spg_pts=spg_pts, l=lz, n_nopml=n_nopml)
    omega = 2.0 * PI * nu
    return Grid3D(x, y, z, omega, meta={"source_shift": source_shift, "nu": nu, "length": length})


def reference_source_index(g: Grid3D):
    """Grid index of the point source placed by main (Source/main.cpp:184-211).

    The source sits at (xc/2, yc/2, zc/2) with xc = l (+h when n is odd, or
    exactly l with SOURCE_SHIFT); ``F3D_ex_complex`` matches the node with
    coordinate (i+1)*h (Source/functions.cpp:4564-4589,4655-4668).
    """
    idx = []
    for ax in (g.x, g.y, g.z):
        xc = ax.l
        if not g.meta.get("source_shift") and ax.n % 2 != 0:
            xc += ax.h
        i = int(round((xc / 2.0) / ax.h)) - 1
        idx.append(i)
    return tuple(idx)


def physical_mask(g: Grid3D) -> np.ndarray:
    """Boolean (nz, ny, nx) mask of the physical domain (``reducePML3D``,
    Source/functions.cpp:238-263): i,j outside the PML and k outside the
    sponge."""
    m = np.zeros(g.shape_zyx, dtype=bool)
    zlo = max(g.z.spg_pts, g.z.pml_pts)
    m[zlo:g.z.n - zlo, g.y.pml_pts:g.y.n - g.y.pml_pts, g.x.pml_pts:g.x.n - g.x.pml_pts] = True
    return m


def ppw_frequency(c_min: float, h: float, ppw: float) -> float:
    """Angular frequency giving ``ppw`` points per minimum wavelength."""
    return 2.0 * math.pi * c_min / (ppw * h)
