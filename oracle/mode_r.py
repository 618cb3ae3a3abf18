"""Mode R: the reference operator and solvers, restated in NumPy/SciPy (oracle).

Mode R is the reference's own formulation (Source/FGMRES.cpp:6-725):
    K w = (I - dL * L0^{-1}) w = f,     u = L0^{-1} w,
where L0 is the z-invariant operator diagonalised by an FFT along z
(Source/functions.cpp:5837-6061) and dL is the pointwise squared-slowness
difference with a Gaussian sponge taper (Source/functions.cpp:1740-1824).
PARDISO (per-kz 2D factor/solve) is replaced by ``scipy.sparse.linalg.splu``
and MKL DFTI by ``numpy.fft`` (forward unscaled, backward scaled 1/nz, as
the DFTI descriptor at Source/functions.cpp:5858-5869).

Quirks of the reference kept here (all switchable where it matters):
  q1 ``SetSoundSpeed2D`` never resets its accumulator between columns
     (Source/functions.cpp:1716-1727);
  q2 kz index table (Source/FGMRES.cpp:182-190);
  q3 HOMO media: L0 uses kk = omega/c_z, dL uses the q1 mean c0;
  q4 PML half-index asymmetry (oracle.grid.alpha);
  q5 Arnoldi coefficient conj(V_i^H w) (Source/FGMRES.cpp:511), only with
     ``arnoldi="reference"``; the default is correct MGS.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .grid import PI, Grid3D, pml_coeffs, physical_mask, reference_source_index

C_Z = 1280.0  # Source/definitions.h:255 (c_z, HOMO sound speed)


# --------------------------------------------------------------------------
# media (Source/functions.cpp:1362-1456, 2636-2716, 1686-1824)
# --------------------------------------------------------------------------
def sound_speed_3d(g: Grid3D, media: str = "homo") -> np.ndarray:
    """``SetSoundSpeed3D`` + ``HeteroSoundSpeed3DExtensionToPML``.

    ``homo``: c = c_z (MakeSound3D under HOMO).  ``linear``: model 1 of
    Source/functions.cpp:1370-1378, c = c1*X + c2*Y + c3 with c3 = 600,
    c2 = (1500 - c3)/y.l, c1 = (1800 - c3 - c2*y.l)/x.l, evaluated at
    X = (i + 1 - pml)*hx, Y = (j + 1 - pml)*hy on the physical x,y range
    for every k, then extended into the x,y PML by copying edge values.
    """
    x, y, z = g.x, g.y, g.z
    c = np.zeros(g.shape_zyx, dtype=np.float64)
    px, py = x.pml_pts, y.pml_pts
    if media == "homo":
        c[:, py:y.n - py, px:x.n - px] = C_Z
    elif media == "linear":
        c3 = 600.0
        c2 = (1500.0 - c3) / y.l
        c1 = (1800.0 - c3 - c2 * y.l) / x.l
        ii = np.arange(px, x.n - px, dtype=np.float64)
        jj = np.arange(py, y.n - py, dtype=np.float64)
        X = (ii + 1 - px) * x.h
        Y = (jj + 1 - py) * y.h
        c[:, py:y.n - py, px:x.n - px] = (c1 * X[None, None, :] + c2 * Y[None, :, None] + c3)
    else:
        raise ValueError(media)
    extend_to_pml(c, px, py)
    return c


def extend_to_pml(a: np.ndarray, px: int, py: int) -> None:
    """Copy edge values into the x,y PML, x first then y, in place
    (Source/functions.cpp:2636-2716)."""
    nx = a.shape[-1]
    ny = a.shape[-2]
    if px:
        a[..., :, :px] = a[..., :, px:px + 1]
        a[..., :, nx - px:] = a[..., :, nx - px - 1:nx - px]
    if py:
        a[..., :py, :] = a[..., py:py + 1, :]
        a[..., ny - py:, :] = a[..., ny - py - 1:ny - py, :]


def sound_speed_2d(g: Grid3D, c3d: np.ndarray, quirk_q1: bool = True) -> np.ndarray:
    """``SetSoundSpeed2D`` (Source/functions.cpp:1686-1738) + PML extension.

    Harmonic mean over the non-sponge z range of 1/c^2 per (i,j) column,
    columns visited j outer, i inner.  With q1 the running sum carries over
    from one column to the next: s <- (s + sum_k 1/c^2) / nz_phys.
    """
    x, y, z = g.x, g.y, g.z
    nzp = z.n - 2 * z.spg_pts
    inv2 = 1.0 / (c3d[z.spg_pts:z.n - z.spg_pts] ** 2)
    col = inv2.sum(axis=0)  # (ny, nx)
    c2d = np.zeros((y.n, x.n), dtype=np.float64)
    s = 0.0
    for j in range(y.pml_pts, y.n - y.pml_pts):
        for i in range(x.pml_pts, x.n - x.pml_pts):
            if quirk_q1:
                s = (s + col[j, i]) / nzp
            else:
                s = col[j, i] / nzp
            c2d[j, i] = math.sqrt(1.0 / s)
    extend_to_pml(c2d, x.pml_pts, y.pml_pts)
    return c2d


def delta_l(g: Grid3D, c3d: np.ndarray, c2d: np.ndarray, beta: float) -> np.ndarray:
    """``GenerateDeltaL`` (Source/functions.cpp:1740-1824).

    dL = omega^2 ((1 + i beta)/c0^2 - 1/c^2) for spg <= k <= nz - spg
    (inclusive upper end), and a Gaussian taper (sigma = 0.3) of the edge
    plane into both sponges.
    """
    z = g.z
    w2 = g.omega * g.omega
    nz, spg = z.n, z.spg_pts
    dl = np.zeros(g.shape_zyx, dtype=np.complex128)
    ks = np.arange(spg, nz - spg + 1)
    ks = ks[ks < nz]
    dl[ks] = w2 * (complex(1.0, beta) / (c2d[None] ** 2) - 1.0 / (c3d[ks] ** 2))
    sigma = 0.3
    z0 = spg * z.h
    zN = (nz - spg) * z.h
    L0 = z0
    Ln = z.l - zN
    for k in range(0, spg):
        zp = k * z.h
        dl[k] = dl[spg] * math.exp(-(zp - z0) * (zp - z0) / (L0 * L0) / (sigma * sigma))
    for k in range(nz - spg + 1, nz):
        zp = k * z.h
        dl[k] = dl[nz - spg] * math.exp(-(zp - zN) * (zp - zN) / (Ln * Ln) / (sigma * sigma))
    return dl


def kz2_reference(nz: int, lz: float) -> np.ndarray:
    """kz^2 table with the reference's index map q2 (Source/FGMRES.cpp:182-190):
    index k < nz/2 - 1 -> k, otherwise -> nz - k (integer nz/2)."""
    k = np.arange(nz)
    kk = np.where(k < nz // 2 - 1, k, nz - k).astype(np.float64)
    return 4.0 * PI * PI * kk * kk / (lz * lz)


# --------------------------------------------------------------------------
# per-kz 2D operator (Source/functions.cpp:3270-3370, 2347-2402)
# --------------------------------------------------------------------------
def assemble_2d(g: Grid3D, shift: np.ndarray) -> sp.csc_matrix:
    """5-point PML matrix of ``GenSparseMatrixOnline2DwithPMLFast`` with
    ``shift`` (ny, nx) added on the diagonal (``freqs`` update).

    Row (i,j): u[i-1,j] * alpha_x(i)alpha_x(i-1/2)/hx^2, u[i+1,j] *
    alpha_x(i)alpha_x(i+1/2)/hx^2, the same with y, and the diagonal
    -(sum of the four) + shift; Dirichlet outside the grid.
    """
    nx, ny = g.x.n, g.y.n
    cmx, cpx = pml_coeffs(g.x, g.omega)
    cmy, cpy = pml_coeffs(g.y, g.omega)
    diag = -(cmx + cpx)[None, :] - (cmy + cpy)[:, None] + shift
    n = nx * ny
    lo_x = np.broadcast_to(cmx[None, :], (ny, nx)).copy()
    hi_x = np.broadcast_to(cpx[None, :], (ny, nx)).copy()
    lo_y = np.broadcast_to(cmy[:, None], (ny, nx)).copy()
    hi_y = np.broadcast_to(cpy[:, None], (ny, nx)).copy()
    # scipy diags: offset -1 entry m -> A[m+1, m] is row m+1's coefficient of u[m]
    d_m1 = lo_x.ravel()[1:].copy()
    d_m1[(np.arange(1, n) % nx) == 0] = 0.0
    d_p1 = hi_x.ravel()[:-1].copy()
    d_p1[(np.arange(0, n - 1) % nx) == nx - 1] = 0.0
    d_mx = lo_y.ravel()[nx:]
    d_px = hi_y.ravel()[:-nx]
    A = sp.diags([d_mx, d_m1, diag.ravel(), d_p1, d_px], [-nx, -1, 0, 1, nx],
                 shape=(n, n), format="csc", dtype=np.complex128)
    return A


@dataclass
class ModeR:
    """Set-up state of the reference solve: the oracle's ``FGMRES`` setup
    block (Source/FGMRES.cpp:72-298)."""

    g: Grid3D
    beta: float
    dl: np.ndarray          # (nz, ny, nx) complex
    c3d: np.ndarray
    c2d: np.ndarray
    shifts: np.ndarray      # (nz, ny, nx) complex diagonal shift per kz
    mats: list
    lus: list
    skip: np.ndarray | None = None   # SAVE_MEM: modes neither factored nor solved

    @property
    def shape(self):
        return self.g.shape_zyx

    # -- L0^{-1} and L0 (Source/functions.cpp:5837-6061, 6247-6318) -------
    def l0_solve(self, f: np.ndarray) -> np.ndarray:
        fh = np.fft.fft(f.reshape(self.shape), axis=0)
        out = np.empty_like(fh)
        for k in range(self.g.z.n):
            if self.skip is not None and self.skip[k]:
                out[k] = 0.0      # D2csr[k]->solve == 0: x_sol_prd = 0 (functions.cpp:6020-6024)
            else:
                out[k] = self.lus[k].solve(fh[k].ravel()).reshape(fh[k].shape)
        return np.fft.ifft(out, axis=0)

    def l0_apply(self, u: np.ndarray) -> np.ndarray:
        uh = np.fft.fft(u.reshape(self.shape), axis=0)
        out = np.empty_like(uh)
        for k in range(self.g.z.n):
            out[k] = (self.mats[k] @ uh[k].ravel()).reshape(uh[k].shape)
        return np.fft.ifft(out, axis=0)

    def apply_k(self, w: np.ndarray) -> np.ndarray:
        """``ApplyCoeffMatrixA_CSR``: g = w - dL * L0^{-1} w
        (Source/functions.cpp:5554-5575)."""
        w = w.reshape(self.shape)
        return w - self.dl * self.l0_solve(w)

    def apply_a(self, u: np.ndarray) -> np.ndarray:
        """u-space operator A_R u = L0 u - dL u (so K = A_R L0^{-1})."""
        u = u.reshape(self.shape)
        return self.l0_apply(u) - self.dl * u


def kz_skip_reference(kz2: np.ndarray, omega: float, ratio: float) -> np.ndarray:
    """The reference's SAVE_MEM rule (Source/FGMRES.cpp:197-206): mode k is
    neither factored nor solved when kww >= ratio * k2, kww its kz table
    value and k2 = kk^2, kk = omega / c_z (definitions.h)."""
    return kz2 >= ratio * (omega / C_Z) ** 2


def setup(g: Grid3D, beta: float = 0.5, media: str = "homo", quirk_q1: bool = True,
          kz2: np.ndarray | None = None, factor: bool = True, kz_skip_ratio: float = 0.0) -> ModeR:
    """Media, dL, per-kz 2D matrices and their factorizations (kz_skip_ratio
    > 0: the reference's SAVE_MEM build with that ratio, 5 at nu = 4 Hz)."""
    c3d = sound_speed_3d(g, media)
    c2d = sound_speed_2d(g, c3d, quirk_q1=quirk_q1)
    dl = delta_l(g, c3d, c2d, beta)
    if kz2 is None:
        kz2 = kz2_reference(g.z.n, g.z.l)
    w = g.omega
    if media == "homo":
        base = np.full((g.y.n, g.x.n), (w / C_Z) ** 2 * complex(1.0, beta))   # q3
    else:
        base = (w / c2d) ** 2 * complex(1.0, beta)
    shifts = base[None, :, :] - kz2[:, None, None]
    skip = kz_skip_reference(kz2, w, kz_skip_ratio) if kz_skip_ratio > 0 else None
    mats, lus = [], []
    for k in range(g.z.n):
        A = assemble_2d(g, shifts[k])
        mats.append(A)
        lus.append(spla.splu(A) if factor and (skip is None or not skip[k]) else None)
    return ModeR(g, beta, dl, c3d, c2d, shifts, mats, lus, skip)


def point_source_rhs(g: Grid3D) -> np.ndarray:
    """``SetRHS3D``: -1/(hx hy hz) at the source node (Source/functions.cpp:4564-4668)."""
    f = np.zeros(g.shape_zyx, dtype=np.complex128)
    i, j, k = reference_source_index(g)
    f[k, j, i] = -1.0 / (g.x.h * g.y.h * g.z.h)
    return f


# --------------------------------------------------------------------------
# FGMRES in the reference's structure (Source/FGMRES.cpp:464-684)
# --------------------------------------------------------------------------
@dataclass
class FgmresLog:
    rows: list          # (iteration, Res_phys, RelRes_phys, diff_sol)
    x: np.ndarray       # final Krylov iterate w
    u: np.ndarray       # final solution u = L0^{-1} w


def fgmres_reference(st: ModeR, f: np.ndarray, m: int = 10, rest: int = 5, thresh: float = 1e-4,
                     rel_res_exit: float = 1e-4, arnoldi: str = "mgs") -> FgmresLog:
    """Restarted GMRES on K w = f exactly as the reference drives it.

    Every inner step solves the small LS problem from scratch (zgels,
    :552-570), forms x = x_init + V y (:575), recomputes the true residual
    K x - f and its physical-domain norm (:579-592), applies L0^{-1} to get
    u (:601) and logs (restart*m + j, Res, RelRes, |u_k - u_{k-1}|/|u_{k-1}|)
    (:647).  Exit when RelRes < rel_res_exit (:650).
    """
    shape = st.shape
    N = st.g.size
    mask = physical_mask(st.g)
    fv = f.reshape(-1)
    norm_f = np.linalg.norm(fv)
    x_init = np.zeros(N, dtype=np.complex128)
    u_prev = np.zeros(int(mask.sum()), dtype=np.complex128)
    rows = []
    x0 = x_init.copy()
    u = np.zeros(shape, dtype=np.complex128)
    finish = False
    for restart in range(rest):
        if finish:
            break
        x0 = x_init.copy()
        w = st.apply_k(x0).reshape(-1)
        r0 = fv - w
        beta = np.linalg.norm(r0)
        V = np.zeros((m + 1, N), dtype=np.complex128)
        H = np.zeros((m + 1, m), dtype=np.complex128)
        V[0] = r0 / beta
        for j in range(m):
            w = st.apply_k(V[j]).reshape(-1)
            for i in range(j + 1):
                if arnoldi == "reference":
                    hij = np.vdot(w, V[i])          # zdotc(w, V_i) = conj(V_i^H w)  (q5)
                else:
                    hij = np.vdot(V[i], w)          # V_i^H w
                H[i, j] = hij
                w = w - hij * V[i]
            H[j + 1, j] = np.linalg.norm(w)
            if abs(H[j + 1, j]) < thresh:
                break
            V[j + 1] = w / H[j + 1, j].real
            e = np.zeros(j + 2, dtype=np.complex128)
            e[0] = beta
            y = np.linalg.lstsq(H[:j + 2, :j + 1], e, rcond=None)[0]
            x0 = x_init + V[:j + 1].T @ y
            r = st.apply_k(x0).reshape(-1) - fv
            res = np.linalg.norm(r.reshape(shape)[mask])
            relres = res / norm_f
            u = st.l0_solve(x0)
            u_phys = u[mask]
            nprev = np.linalg.norm(u_prev)
            diff = np.linalg.norm(u_phys - u_prev) / nprev if nprev > 0 else math.inf
            u_prev = u_phys.copy()
            rows.append((restart * m + j, res, relres, diff))
            if relres < rel_res_exit:
                finish = True
                break
        x_init = x0.copy()
    return FgmresLog(rows, x0.reshape(shape), u)


def nullify_source_cross(g: Grid3D, u: np.ndarray) -> np.ndarray:
    """``NullifySource2D(x, y, u + plane nz/2, size2D/2, 1)``
    (Source/functions.cpp:6628-6644): zero the points 0 and 1 to the left,
    right, below and above flat index size2D/2 of the middle z plane, with the
    reference's flat indexing (for even nx the "left" neighbour of the row's
    first point is the last point of the row below)."""
    out = np.array(u, dtype=np.complex128, copy=True).reshape(g.shape_zyx)
    plane = out[g.z.n // 2].reshape(-1)
    nx = g.x.n
    src = g.size2d // 2
    jsrc, isrc = divmod(src, nx)
    for l in (0, 1):
        for q in (isrc - l + nx * jsrc, isrc + l + nx * jsrc, isrc + nx * (jsrc - l), isrc + nx * (jsrc + l)):
            plane[q] = 0.0
    return out


def bicgstab_reference(st: ModeR, f: np.ndarray, m: int = 10, res_exit: float = 1e-8):
    """BiCGStab as ``BCGSTAB`` drives it (Source/BcGSTAB.cpp:397-560).

    Right-preconditioned BiCGStab on K with the iterate kept in u-space
    (x += alpha L0^{-1} p + omega L0^{-1} s); shadow residual r* = 2 r0;
    residual A_R x - f checked via L0 x then K (:495-496); exit when the
    absolute physical residual < res_exit (:564).  The reference assembles
    its 2D matrices with the 9-point routine (:143), whose entries at the
    diagonal neighbours are exactly zero with the coefficients it uses
    (Source/functions.cpp:2497-2512, 3557-3559), so L0 is the same 5-point
    operator as FGMRES's (pinned by tests/test_oracle_pins.py).
    """
    shape = st.shape
    mask = physical_mask(st.g)
    fv = f.reshape(-1)
    norm_f = np.linalg.norm(fv)
    x = np.zeros_like(fv)
    r = fv - st.apply_k(x).reshape(-1)
    p = r.copy()
    rst = 2.0 * r
    rows = []
    for j in range(m):
        Ay = st.apply_k(p).reshape(-1)
        yv = st.l0_solve(p).reshape(-1)
        alpha = np.vdot(rst, r) / np.vdot(rst, Ay)
        s = r - alpha * Ay
        Az = st.apply_k(s).reshape(-1)
        zv = st.l0_solve(s).reshape(-1)
        om = np.vdot(Az, s) / np.vdot(Az, Az)
        rn = s - om * Az
        x = x + alpha * yv + om * zv
        beta = (alpha / om) * np.vdot(rst, rn) / np.vdot(rst, r)
        p = rn + beta * (p - om * Ay)
        r = rn
        res_vec = st.apply_a(x).reshape(-1) - fv
        res = np.linalg.norm(res_vec.reshape(shape)[mask])
        rows.append((j, res, res / norm_f))
        if res < res_exit:
            break
    return x.reshape(shape), rows
