"""Mode N: the complex 7-point PML-stretched operator, preconditioned by the
reference's FFT-z / per-kz 2D solve (oracle, FP64).

Operator (PML on all six faces, the reference's ``alpha`` on every axis,
oracle.grid.alpha = Source/functions.cpp:1839-1878):

  (A u)_ijk = sum_a [ cp_a (u_{+a} - u) + cm_a (u_{-a} - u) ]
              + omega^2 s2_ijk (1 + i beta_phys) u_ijk,       u = 0 outside,

with cp_a(i) = alpha(i) alpha(i+1/2)/h^2, cm_a(i) = alpha(i) alpha(i-1/2)/h^2:
the reference's 5-point 2D form (``beta2D_pml``, Source/functions.cpp:
2347-2402) extended to z.

Preconditioner M (the reference's L0, Source/functions.cpp:5837-6061): the
z part is replaced by a periodic spectral symbol kz^2 and s2 by its z-mean
s0^2(x,y) over the non-PML z range, with a complex shift beta_prec:

  M_kz = L_xy + omega^2 s0^2 (1 + i beta_prec) - kz^2,

applied as forward FFT along z (unscaled), one 2D solve per kz, inverse FFT
(scaled 1/nz).  kz^2 is either the symbol of the 7-point z difference,
(4/hz^2) sin^2(pi k / nz) ("discrete", the default), the continuous
(2 pi min(k, nz-k) / Lz)^2 ("continuous"), or the reference's table q2.

With z_transform="eigen" the FFT is replaced by the eigenvectors of the 1D
z operator including its PML, D_z = W diag(lam) W^{-1}: the 2D system of
mode k gets the shift lam_k instead of -kz^2, and M^{-1} = W diag(M_k^{-1})
W^{-1} (exact when the medium is z-invariant and beta_prec = 0).

FGMRES here is flexible (Z_j = M^{-1} V_j kept), right preconditioned, with
Givens rotations and classical Gram-Schmidt applied twice (CGS2).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.sparse.linalg as spla

from .grid import Axis, Grid3D, pml_coeffs
from .media import Problem
from .mode_r import assemble_2d, kz2_reference


def kz2_table(nz: int, hz: float, symbol: str = "discrete") -> np.ndarray:
    k = np.arange(nz, dtype=np.float64)
    if symbol == "discrete":
        return (4.0 / (hz * hz)) * np.sin(math.pi * k / nz) ** 2
    lz = nz * hz
    if symbol == "continuous":
        kk = np.minimum(k, nz - k)
        return (2.0 * math.pi * kk / lz) ** 2
    if symbol == "reference":
        return kz2_reference(nz, lz)
    raise ValueError(symbol)


def s0_squared(s2: np.ndarray, pml_z: int) -> np.ndarray:
    """z-mean of s2 over the non-PML z range, per (j, i)."""
    nz = s2.shape[0]
    lo, hi = pml_z, nz - pml_z
    if hi <= lo:
        lo, hi = 0, nz
    return s2[lo:hi].mean(axis=0)


@dataclass
class ModeN:
    prob: Problem
    g: Grid3D
    beta_prec: float
    coef: dict
    kz2: np.ndarray
    shifts: np.ndarray
    lus: list
    zW: np.ndarray | None = None
    zWi: np.ndarray | None = None
    skip: np.ndarray | None = None     # modes solved by the diagonal of their 2D operator
    diag: np.ndarray | None = None     # (nz, ny, nx) that diagonal

    @property
    def shape(self):
        return self.prob.shape

    # ---------------------------------------------------------------- A_N
    def apply_a(self, u: np.ndarray) -> np.ndarray:
        u = u.reshape(self.shape)
        p = self.prob
        out = (p.omega ** 2) * p.s2 * complex(1.0, p.beta_phys) * u
        for axis, name in ((2, "x"), (1, "y"), (0, "z")):
            cm, cp = self.coef[name]
            shp = [1, 1, 1]
            shp[axis] = -1
            cm_b = cm.reshape(shp)
            cp_b = cp.reshape(shp)
            up = np.zeros_like(u)
            um = np.zeros_like(u)
            sl = [slice(None)] * 3
            sl2 = [slice(None)] * 3
            sl[axis] = slice(0, -1)
            sl2[axis] = slice(1, None)
            up[tuple(sl)] = u[tuple(sl2)]     # u_{+a}
            um[tuple(sl2)] = u[tuple(sl)]     # u_{-a}
            out = out + cp_b * (up - u) + cm_b * (um - u)
        return out

    def apply_a_adjoint(self, u: np.ndarray) -> np.ndarray:
        """A^H u (conjugate transpose of the stencil)."""
        u = u.reshape(self.shape)
        p = self.prob
        out = np.conj((p.omega ** 2) * p.s2 * complex(1.0, p.beta_phys)) * u
        for axis, name in ((2, "x"), (1, "y"), (0, "z")):
            cm, cp = self.coef[name]
            n = cm.size
            shp = [1, 1, 1]
            shp[axis] = -1
            diag = -(cm + cp)
            out = out + np.conj(diag).reshape(shp) * u
            # A[i, i+1] = cp[i] -> A^H[i+1, i] = conj(cp[i]); A[i, i-1] = cm[i] -> A^H[i-1, i] = conj(cm[i])
            t_from_cp = np.zeros_like(u)
            t_from_cm = np.zeros_like(u)
            sl = [slice(None)] * 3
            sl2 = [slice(None)] * 3
            sl[axis] = slice(1, None)
            sl2[axis] = slice(0, -1)
            cpc = np.conj(cp[:-1]).reshape(shp)
            cmc = np.conj(cm[1:]).reshape(shp)
            t_from_cp[tuple(sl)] = cpc * u[tuple(sl2)]
            t_from_cm[tuple(sl2)] = cmc * u[tuple(sl)]
            out = out + t_from_cp + t_from_cm
        return out

    # ------------------------------------------------------------------ M
    def apply_prec(self, v: np.ndarray) -> np.ndarray:
        if self.zW is not None:
            vh = np.tensordot(self.zWi, v.reshape(self.shape), axes=(1, 0))
        else:
            vh = np.fft.fft(v.reshape(self.shape), axis=0)
        out = np.empty_like(vh)
        for k in range(self.shape[0]):
            if self.skip is not None and self.skip[k]:
                out[k] = vh[k] / self.diag[k]
            else:
                out[k] = self.lus[k].solve(vh[k].ravel()).reshape(vh[k].shape)
        if self.zW is not None:
            return np.tensordot(self.zW, out, axes=(1, 0))
        return np.fft.ifft(out, axis=0)

    def apply_prec_adjoint(self, v: np.ndarray) -> np.ndarray:
        """(M^{-1})^H v.  FFT: M^{-1} = F^{-1} D^{-1} F and F^H = nz F^{-1}, so
        (M^{-1})^H = F^{-1} D^{-H} F; eigenbasis: (W D^{-1} Wi)^H = Wi^H D^{-H} W^H."""
        if self.zW is not None:
            vh = np.tensordot(self.zW.conj().T, v.reshape(self.shape), axes=(1, 0))
        else:
            vh = np.fft.fft(v.reshape(self.shape), axis=0)
        out = np.empty_like(vh)
        for k in range(self.shape[0]):
            if self.skip is not None and self.skip[k]:
                out[k] = vh[k] / np.conj(self.diag[k])
            else:
                out[k] = self.lus[k].solve(vh[k].ravel(), trans="H").reshape(vh[k].shape)
        if self.zW is not None:
            return np.tensordot(self.zWi.conj().T, out, axes=(1, 0))
        return np.fft.ifft(out, axis=0)

    # ------------------------------------------------- sparse A and gradient
    def assemble_a(self, s2: np.ndarray | None = None):
        """A as a sparse matrix (Kronecker sum of the 1D PML operators plus
        the mass term), unknowns ordered (z, y, x) with x fastest."""
        import scipy.sparse as sp
        p = self.prob
        s2 = p.s2 if s2 is None else s2

        def t1(name):
            cm, cp = self.coef[name]
            return sp.diags([cm[1:], -(cm + cp), cp[:-1]], [-1, 0, 1], format="csr")

        ix, iy, iz = (sp.identity(n, format="csr") for n in (p.nx, p.ny, p.nz))
        a = sp.kron(iz, sp.kron(iy, t1("x"))) + sp.kron(iz, sp.kron(t1("y"), ix)) + sp.kron(t1("z"), sp.kron(iy, ix))
        a = a + sp.diags((p.omega ** 2) * complex(1.0, p.beta_phys) * s2.ravel())
        return a.tocsc()


def zpml_eigen(cm: np.ndarray, cp: np.ndarray):
    """Eigen-decomposition of the tridiagonal z operator with its PML."""
    D = np.diag(-(cm + cp)) + np.diag(cp[:-1], 1) + np.diag(cm[1:], -1)
    lam, W = np.linalg.eig(D)
    return lam, W, np.linalg.inv(W)


def setup(prob: Problem, beta_prec: float = 0.5, kz_symbol: str = "discrete", factor: bool = True,
          z_transform: str = "fft", kz_skip_ratio: float = 0.0) -> ModeN:
    """kz_skip_ratio > 0: the reference's SAVE_MEM idea (Source/FGMRES.cpp:
    197-206) for the 7-point operator: a mode whose kz^2 (FFT) or -Re lambda_k
    (eigenbasis) is at least ratio * k2, k2 = omega^2 max_(x,y) s0^2, is not
    factored; its 2D system is solved by its diagonal instead of being set to
    zero (zeroing stalls FGMRES on this operator)."""
    ax = Axis(n=prob.nx, h=prob.h, pml_pts=prob.pml)
    ay = Axis(n=prob.ny, h=prob.h, pml_pts=prob.pml)
    az = Axis(n=prob.nz, h=prob.h, pml_pts=prob.pml)
    g = Grid3D(ax, ay, az, prob.omega)
    coef = {"x": pml_coeffs(ax, prob.omega), "y": pml_coeffs(ay, prob.omega), "z": pml_coeffs(az, prob.omega)}
    kz2 = kz2_table(prob.nz, prob.h, kz_symbol)
    s0 = s0_squared(prob.s2, prob.pml)
    base = (prob.omega ** 2) * s0 * complex(1.0, beta_prec)
    zW = zWi = None
    if z_transform == "eigen":
        lam, zW, zWi = zpml_eigen(*coef["z"])
        shifts = base[None, :, :] + lam[:, None, None]
    else:
        shifts = base[None, :, :] - kz2[:, None, None]
    skip = diag = None
    if kz_skip_ratio > 0:
        kww = -lam.real if z_transform == "eigen" else kz2
        skip = kww >= kz_skip_ratio * (prob.omega ** 2) * s0.max()
        cmx, cpx = coef["x"]
        cmy, cpy = coef["y"]
        diag = -(cmx + cpx)[None, None, :] - (cmy + cpy)[None, :, None] + shifts
    lus = []
    if factor:
        for k in range(prob.nz):
            lus.append(None if skip is not None and skip[k] else spla.splu(assemble_2d(g, shifts[k])))
    return ModeN(prob, g, beta_prec, coef, kz2, shifts, lus, zW, zWi, skip, diag)


@dataclass
class SolveResult:
    x: np.ndarray
    iters: int
    history: list        # relative residual estimates per iteration
    true_relres: float


def fgmres(apply_a, apply_m, f: np.ndarray, tol: float = 1e-8, m: int = 20, max_iter: int = 500,
           x0: np.ndarray | None = None, orth: str = "cgs2") -> SolveResult:
    """Flexible GMRES(m), right preconditioned, Givens least squares.

    Stops when the Givens residual estimate |g_{j+1}| <= tol ||f||, then
    confirms with the true residual at the end of the cycle (and restarts
    if the true residual is still above tol).
    """
    shape = f.shape
    fv = f.reshape(-1)
    nf = np.linalg.norm(fv)
    x = np.zeros_like(fv) if x0 is None else x0.reshape(-1).copy()
    hist = []
    it = 0
    while True:
        r = fv - apply_a(x.reshape(shape)).reshape(-1)
        beta = np.linalg.norm(r)
        if beta <= tol * nf or it >= max_iter:
            return SolveResult(x.reshape(shape), it, hist, beta / nf)
        V = [r / beta]
        Z = []
        H = np.zeros((m + 1, m), dtype=np.complex128)
        cs = np.zeros(m, dtype=np.complex128)
        sn = np.zeros(m, dtype=np.complex128)
        gv = np.zeros(m + 1, dtype=np.complex128)
        gv[0] = beta
        jlast = 0
        for j in range(m):
            z = apply_m(V[j].reshape(shape)).reshape(-1)
            Z.append(z)
            w = apply_a(z.reshape(shape)).reshape(-1)
            passes = 2 if orth == "cgs2" else 1
            if orth == "mgs":
                for i in range(j + 1):
                    hij = np.vdot(V[i], w)
                    H[i, j] += hij
                    w = w - hij * V[i]
            else:
                Vm = np.array(V)
                for _ in range(passes):
                    hcol = Vm.conj() @ w
                    H[:j + 1, j] += hcol
                    w = w - Vm.T @ hcol
            hn = np.linalg.norm(w)
            H[j + 1, j] = hn
            # apply previous rotations to the new column
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -np.conj(sn[i]) * H[i, j] + np.conj(cs[i]) * H[i + 1, j]
                H[i, j] = t
            a, b = H[j, j], H[j + 1, j]
            den = math.hypot(abs(a), abs(b))
            if den == 0.0:
                cs[j], sn[j] = 1.0, 0.0
            elif abs(a) == 0.0:
                cs[j], sn[j] = 0.0, 1.0
            else:
                cs[j] = abs(a) / den
                sn[j] = (a / abs(a)) * np.conj(b) / den
            H[j, j] = cs[j] * a + sn[j] * b
            H[j + 1, j] = 0.0
            gv[j + 1] = -np.conj(sn[j]) * gv[j]
            gv[j] = cs[j] * gv[j]
            it += 1
            jlast = j
            hist.append(abs(gv[j + 1]) / nf)
            if hn == 0.0:
                break
            V.append(w / hn)
            if abs(gv[j + 1]) <= tol * nf or it >= max_iter:
                break
        k = jlast + 1
        y = np.linalg.solve(np.triu(H[:k, :k]), gv[:k])
        x = x + np.array(Z[:k]).T @ y


# ------------------------------------------------------------ misfit gradient
def misfit(on: ModeN, F: np.ndarray, recv: np.ndarray, data: np.ndarray, s2: np.ndarray | None = None) -> float:
    """J = 1/2 sum_s ||P u_s - d_s||^2 with u_s from a sparse direct solve."""
    import scipy.sparse.linalg as spla
    lu = spla.splu(on.assemble_a(s2))
    j = 0.0
    for s in range(len(F)):
        r = lu.solve(F[s].ravel())[recv] - data[s]
        j += 0.5 * float(np.vdot(r, r).real)
    return j


def misfit_grad(on: ModeN, F: np.ndarray, recv: np.ndarray, data: np.ndarray, solver: str = "direct",
                tol: float = 1e-12):
    """Gradient of J with respect to s2 from two solves per source: A u = f and
    A^H lam = P^T (d - P u); dJ/ds2 = sum_s Re(conj(lam_s) omega^2 (1 + i beta) u_s).
    solver "direct": sparse LU; "fgmres": the preconditioned FGMRES pair."""
    import scipy.sparse.linalg as spla
    p = on.prob
    dA = (p.omega ** 2) * complex(1.0, p.beta_phys)
    g = np.zeros(on.shape)
    j = 0.0
    lu = spla.splu(on.assemble_a()) if solver == "direct" else None
    for s in range(len(F)):
        if lu is not None:
            u = lu.solve(F[s].ravel())
        else:
            u = fgmres(on.apply_a, on.apply_prec, F[s], tol=tol, m=40, max_iter=5000).x.ravel()
        r = u[recv] - data[s]
        j += 0.5 * float(np.vdot(r, r).real)
        adj = np.zeros(u.size, dtype=np.complex128)
        np.add.at(adj, recv, -r)
        if lu is not None:
            lam = lu.solve(adj, trans="H")
        else:
            lam = fgmres(on.apply_a_adjoint, on.apply_prec_adjoint, adj.reshape(on.shape), tol=tol, m=40,
                         max_iter=5000).x.ravel()
        g += (np.conj(lam) * dA * u).real.reshape(on.shape)
    return j, g


def receiver_plane(prob: Problem, stride: int = 1, depth: int = 1) -> np.ndarray:
    """Linear indices of a receiver plane at the top of the interior: the
    y-row pml + depth, interior x and z (every `stride`-th point)."""
    j = prob.pml + depth
    ks = np.arange(prob.pml, prob.nz - prob.pml, stride)
    is_ = np.arange(prob.pml, prob.nx - prob.pml, stride)
    kk, ii = np.meshgrid(ks, is_, indexing="ij")
    return ((kk * prob.ny + j) * prob.nx + ii).ravel().astype(np.int64)
