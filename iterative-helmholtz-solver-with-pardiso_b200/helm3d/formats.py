"""Result files of the reference's driver and its convergence-order tools.

Host-side tooling around the solver (no device code): it writes and reads
the files the reference's driver writes, in its text formats, so that logs
and solutions of this library can be compared with the reference's own
(HETERO/*.dat), and restates the two convergence-order computations the
reference runs on saved solutions.

- Convergence logs: file name Source/FGMRES.cpp:50, one line per outer
  iteration ``"%d %e %e %lf"`` = (iteration, residual, relative residual,
  relative change of the solution), Source/FGMRES.cpp:631 and :647.
- Full 3D solutions on the physical grid: ``sol3D_N<n>.dat``, one
  ``"%18.16lf %18.16lf"`` line (re, im) per point, x fastest, then y, then
  z, Source/main.cpp:827-834; the physical grid is reducePML3D's
  (Source/functions.cpp:238-264): x and y without their PML, z without its
  absorbing layer.
- Runge ratio of three resolutions n1 < n2 < n3 (n + 1 doubling):
  Source/functions.cpp:932-1146 (the dim = 3 branch that is compiled):
  the finest solution injected onto each coarser grid (point
  ``step (i + 1) - 1`` with ``step = (n3 + 1) / (n + 1)``), minus that grid's
  solution, measured by IntegralNorm3D (sum of moduli times h,
  Source/functions.cpp:1348-1360); the ratio f1 / f2.
- beta_3D_norm2 files: Source/functions.cpp:1147-1240 (Beta3D) with
  :1290-1304 (compute_and_print_circle_norm_nopml) and :629-670
  (check_norm_circle_3D_nopml): the finer solution injected onto the
  coarser grid, and for every outer radius i h (i = 2 .. n1 - 1) the relative
  Frobenius error of the coarser solution over the shell 2h <= r <= i h
  around the source, one ``"%lf %lf"`` line (i h, error).
"""
from __future__ import annotations

import math
from typing import Iterable, List, Sequence, Tuple

import numpy as np


# ------------------------------------------------------------ convergence logs
def convergence_filename(n_nopml: int, pml_pts: int, length_x: float, freq: float, spg_width: float,
                         beta: float) -> str:
    """The reference's log name: N = physical points per side, PML points,
    domain length and frequency (printed as integers), the z sponge width
    2 h_z spg_pts (width 6, no decimals) and the preconditioner shift beta."""
    return "convergence_N%d_PML%d_Lx%d_FREQ%d_SPG%6.0f_BETA%5.3f_FGMRES.dat" % (
        n_nopml, pml_pts, int(length_x), int(freq), spg_width, beta)


def convergence_line(it: int, res: float, relres: float, change: float) -> str:
    """One log line, C's ``"%d %e %e %lf\\n"``."""
    return "%d %s %s %s\n" % (it, _c_e(res), _c_e(relres), _c_f(change))


def write_convergence(path: str, rows: Iterable[Sequence[float]]) -> None:
    with open(path, "w") as f:
        for it, res, relres, change in rows:
            f.write(convergence_line(int(it), res, relres, change))


def read_convergence(path: str) -> List[Tuple[int, float, float, float]]:
    out = []
    with open(path) as f:
        for line in f:
            p = line.split()
            if len(p) == 4:
                out.append((int(p[0]), float(p[1]), float(p[2]), float(p[3])))
    return out


def convergence_rows(history: Sequence[float], f_norm: float, start: int = 0,
                     changes: Sequence[float] | None = None) -> List[Tuple[int, float, float, float]]:
    """Log rows from a solve's per-iteration relative residuals (``Solver.solve(...,
    history=k)`` → ``last_history``) and the right-hand side's norm; the
    relative change of the solution per iteration is NaN unless given
    (this library forms the iterate at the end of a restart cycle only)."""
    rows = []
    for q, rr in enumerate(history):
        ch = float("nan") if changes is None or q >= len(changes) else float(changes[q])
        rows.append((start + q, float(rr) * float(f_norm), float(rr), ch))
    return rows


# ---------------------------------------------------------------- solutions
def physical(u: np.ndarray, nx: int, ny: int, nz: int, pml_x: int, pml_y: int, z_margin: int) -> np.ndarray:
    """The physical part of a grid vector (reducePML3D): x in [pml_x, nx -
    pml_x), y in [pml_y, ny - pml_y), z in [z_margin, nz - z_margin), x fastest
    (z_margin = the z PML of mode N, or the z sponge of mode R)."""
    v = np.asarray(u).reshape(nz, ny, nx)
    return np.ascontiguousarray(v[z_margin:nz - z_margin, pml_y:ny - pml_y, pml_x:nx - pml_x]).reshape(-1)


def physical_of(u: np.ndarray, grid) -> np.ndarray:
    """`physical` with the margins of a helm3d.Grid."""
    zm = max(int(grid.pml_z), int(grid.spg_z))
    return physical(u, grid.nx, grid.ny, grid.nz, grid.pml_x, grid.pml_y, zm)


def sol3d_filename(n_nopml: int) -> str:
    return "sol3D_N%d.dat" % n_nopml


def write_sol3d(path: str, u_phys: np.ndarray) -> None:
    """One ``"%18.16lf %18.16lf"`` line (re, im) per physical point."""
    u = np.asarray(u_phys, dtype=np.complex128).reshape(-1)
    with open(path, "w") as f:
        for z in u:
            f.write("%18.16f %18.16f\n" % (z.real, z.imag))


def read_sol3d(path: str, count: int | None = None) -> np.ndarray:
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    u = a[:, 0] + 1j * a[:, 1]
    return u if count is None else u[:count]


# ----------------------------------------------------- convergence-order tools
def inject(fine: np.ndarray, n_fine: int, n_coarse: int) -> np.ndarray:
    """The fine cube solution (n_fine per side, x fastest) at the coarse
    grid's points: coarse (i, j, k) = fine (s (i + 1) - 1, ...), s = (n_fine + 1)
    / (n_coarse + 1) (integer division, as the reference)."""
    s = (n_fine + 1) // (n_coarse + 1)
    v = np.asarray(fine).reshape(n_fine, n_fine, n_fine)
    idx = s * (np.arange(n_coarse) + 1) - 1
    return np.ascontiguousarray(v[np.ix_(idx, idx, idx)]).reshape(-1)


def integral_norm3d(v: np.ndarray, h: float) -> float:
    """IntegralNorm3D: the sum of the moduli times h (one factor of h)."""
    return float(np.abs(np.asarray(v)).sum() * h)


def runge_ratio(u_2h: np.ndarray, u_h: np.ndarray, u_h2: np.ndarray, n1: int, n2: int, n3: int, h1: float,
                h2: float) -> Tuple[float, float, float]:
    """(f1, f2, f1 / f2) with f1 = ||I u_h2 - u_2h|| on grid 1 and f2 = ||I u_h2 -
    u_h|| on grid 2 (IntegralNorm3D), I the injection of the finest."""
    f1 = integral_norm3d(inject(u_h2, n3, n1) - np.asarray(u_2h).reshape(-1), h1)
    f2 = integral_norm3d(inject(u_h2, n3, n2) - np.asarray(u_h).reshape(-1), h2)
    return f1, f2, (f1 / f2 if f2 != 0 else float("inf"))


def beta_filename(nx_nopml: int, ny_nopml: int, spg_pts: int) -> str:
    return "beta_3D_norm2_Nx%dNy%d_SPG%d.dat" % (nx_nopml, ny_nopml, spg_pts)


def shell_errors(u_coarse: np.ndarray, u_fine: np.ndarray, n1: int, h: float,
                 source: Tuple[float, float, float]) -> List[Tuple[float, float]]:
    """Beta3D's rows (i h, error) for i = 2 .. n1 - 1: the relative Frobenius
    error of the coarse solution against the finer one injected onto the
    coarse grid (n2 = 2 (n1 + 1) - 1 points per side), over the points with
    2h <= r <= i h, r measured from the source to ((i + 1) h, (j + 1) h,
    (k + 1) h)."""
    n2 = 2 * (n1 + 1) - 1
    ref = inject(u_fine, n2, n1).reshape(n1, n1, n1)
    sol = np.asarray(u_coarse).reshape(n1, n1, n1)
    c = (np.arange(n1) + 1) * h
    z, y, x = np.meshgrid(c - source[2], c - source[1], c - source[0], indexing="ij")
    r = np.sqrt(x * x + y * y + z * z)
    rows = []
    for i in range(2, n1):
        m = (r >= 2 * h) & (r <= i * h)
        den = np.linalg.norm(ref[m])
        num = np.linalg.norm(sol[m] - ref[m])
        rows.append((i * h, num / den if den != 0 else (float("nan") if num == 0 else float("inf"))))
    return rows


def beta_line(radius: float, err: float) -> str:
    """One beta_3D_norm2 line, C's ``"%lf %lf\\n"``."""
    return "%s %s\n" % (_c_f(radius), _c_f(err))


def write_beta(path: str, rows: Iterable[Tuple[float, float]]) -> None:
    with open(path, "w") as f:
        for rad, err in rows:
            f.write(beta_line(rad, err))


def read_pairs(path: str) -> List[Tuple[float, float]]:
    out = []
    with open(path) as f:
        for line in f:
            p = line.split()
            if len(p) == 2:
                out.append((float(p[0]), float(p[1])))
    return out


# ---------------------------------------------------- C printf conventions
def _c_f(x: float) -> str:
    """C's %f / %lf (glibc spells the non-finite values inf, -inf, nan, -nan)."""
    x = float(x)
    if math.isnan(x):
        return "-nan" if math.copysign(1.0, x) < 0 else "nan"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return "%f" % x


def _c_e(x: float) -> str:
    """C's %e (two-digit exponents at least, as Python's)."""
    x = float(x)
    if math.isnan(x) or math.isinf(x):
        return _c_f(x)
    return "%e" % x
