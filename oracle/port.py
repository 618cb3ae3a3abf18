"""Parallel CPU port of the reference's preconditioned FGMRES solve (test
infrastructure and the CPU baseline of bench.py only; the product library
never imports it).

The method is the reference's (dklyuchinskiy/Iterative-Helmholtz-solver-with-
PARDISO): flexible GMRES right-preconditioned by an FFT along z, one shifted
2D sparse solve per kz, and the inverse FFT (``Solve3DSparseUsingFT_CSR``,
Source/functions.cpp:5837-6061; the FGMRES control flow of
Source/FGMRES.cpp:464-684 with one preconditioner apply per iteration).  It
is the same arithmetic as ``oracle.mode_n`` (operator, kz symbol, shifts,
Givens least squares, CGS2), restructured to use every host core:

  * the nz 2D systems are factored and solved by worker processes (``spawn``
    start method, so a pool started after a CUDA context is safe), each
    owning a fixed set of kz and its SuperLU factors, which stand in for the
    reference's PARDISO phases 11/22/33 (Source/FGMRES.cpp:274-284,
    Source/functions.cpp:5959);
  * the spectral planes live in shared memory, so an apply moves no vectors
    between processes;
  * the z-FFT runs on ``scipy.fft`` with one worker per core (MKL DFTI in
    the reference, Source/functions.cpp:5864-5881);
  * the 7-point operator runs on z-slabs in threads (NumPy releases the
    interpreter lock inside its array loops);
  * the Krylov basis is preallocated, so classical Gram-Schmidt is two
    BLAS matrix-vector products per pass.

``python -m oracle.port --n 200`` runs the full solve of the 200^3
heterogeneous workload with the reference's method in complex128 and
writes its convergence record (iterations, residual history, timings, a
strided sample of the solution) to tests/golden/port_fftz_n200.npz;
``--z-transform eigen --tol 1e-12`` solves the same source with the
PML-eigenbasis preconditioner to 1e-12 (tests/golden/port_eigen_n200.npz),
the FP64 reference solution that GPU solutions are measured against.
"""
from __future__ import annotations

import argparse
import math
import multiprocessing as mp
import os
import time
from concurrent.futures import ThreadPoolExecutor
from multiprocessing import shared_memory

import numpy as np

from .grid import Axis, Grid3D, pml_coeffs

# ----------------------------------------------------------------- workers
_W: dict = {}


def _worker_main(conn, shm_name, shape, grid: Grid3D, ks):
    """Owns the SuperLU factors of the kz planes ``ks``."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    import scipy.sparse.linalg as spla

    from .mode_r import assemble_2d
    shm = shared_memory.SharedMemory(name=shm_name)
    planes = np.ndarray(shape, dtype=np.complex128, buffer=shm.buf)
    lus = {}
    try:
        while True:
            msg = conn.recv()
            cmd = msg[0]
            if cmd == "factor":
                shifts = msg[1]                      # (len(ks), ny, nx)
                t0 = time.perf_counter()
                for q, k in enumerate(ks):
                    lus[k] = spla.splu(assemble_2d(grid, shifts[q]))
                conn.send(("ok", time.perf_counter() - t0))
            elif cmd == "solve":
                trans = msg[1]
                for k in ks:
                    planes[k] = lus[k].solve(planes[k].ravel(), trans=trans).reshape(shape[1:])
                conn.send(("ok", 0.0))
            elif cmd == "quit":
                break
    finally:
        del planes
        shm.close()
        conn.close()


class PortPreconditioner:
    """M^{-1} = F^{-1} diag(M_kz^{-1}) F over a process pool (or the PML
    eigenbasis W diag(M_k^{-1}) W^{-1} when z_transform == "eigen")."""

    def __init__(self, prob, beta_prec: float = 0.25, kz_symbol: str = "discrete", z_transform: str = "fft",
                 workers: int | None = None):
        from . import mode_n
        self.prob = prob
        self.shape = prob.shape
        self.workers = max(1, min(workers or (os.cpu_count() or 1), prob.nz))
        on = mode_n.setup(prob, beta_prec=beta_prec, kz_symbol=kz_symbol, factor=False, z_transform=z_transform)
        self.on = on
        self.zW, self.zWi = on.zW, on.zWi
        nbytes = int(np.prod(self.shape)) * 16
        self.shm = shared_memory.SharedMemory(create=True, size=nbytes)
        self.planes = np.ndarray(self.shape, dtype=np.complex128, buffer=self.shm.buf)
        ctx = mp.get_context("spawn")
        nz = prob.nz
        self.parts = [list(range(w, nz, self.workers)) for w in range(self.workers)]
        self.conns, self.procs = [], []
        for ks in self.parts:
            a, b = ctx.Pipe()
            pr = ctx.Process(target=_worker_main, args=(b, self.shm.name, self.shape, on.g, ks), daemon=True)
            pr.start()
            self.conns.append(a)
            self.procs.append(pr)
        self.factor_s = None

    def factor(self) -> float:
        """Factor every kz system (wall seconds)."""
        t0 = time.perf_counter()
        for c, ks in zip(self.conns, self.parts):
            c.send(("factor", np.ascontiguousarray(self.on.shifts[ks])))
        for c in self.conns:
            st, _ = c.recv()
            assert st == "ok"
        self.factor_s = time.perf_counter() - t0
        return self.factor_s

    def _solve_planes(self, trans: str = "N"):
        for c in self.conns:
            c.send(("solve", trans))
        for c in self.conns:
            st, _ = c.recv()
            assert st == "ok"

    def apply(self, v: np.ndarray) -> np.ndarray:
        import scipy.fft as sfft
        v = v.reshape(self.shape)
        if self.zW is not None:
            self.planes[...] = np.tensordot(self.zWi, v, axes=(1, 0))
        else:
            self.planes[...] = sfft.fft(v, axis=0, workers=self.workers)
        self._solve_planes("N")
        if self.zW is not None:
            return np.tensordot(self.zW, self.planes, axes=(1, 0))
        return sfft.ifft(self.planes, axis=0, workers=self.workers)

    def close(self):
        for c in self.conns:
            try:
                c.send(("quit",))
            except Exception:
                pass
        for p in self.procs:
            p.join(timeout=10)
            if p.is_alive():
                p.terminate()
        self.conns, self.procs = [], []
        try:
            del self.planes
            self.shm.close()
            self.shm.unlink()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class PortOperator:
    """The 7-point PML operator (oracle.mode_n.ModeN.apply_a) evaluated on
    z-slabs in threads: the diagonal d = omega^2 s2 (1 + i beta) - sum of
    the six coefficients, plus the six neighbour terms, zero outside."""

    def __init__(self, prob, threads: int | None = None):
        ax = Axis(n=prob.nx, h=prob.h, pml_pts=prob.pml)
        ay = Axis(n=prob.ny, h=prob.h, pml_pts=prob.pml)
        az = Axis(n=prob.nz, h=prob.h, pml_pts=prob.pml)
        self.cx = pml_coeffs(ax, prob.omega)
        self.cy = pml_coeffs(ay, prob.omega)
        self.cz = pml_coeffs(az, prob.omega)
        self.shape = prob.shape
        self.mass = (prob.omega ** 2) * complex(1.0, prob.beta_phys) * prob.s2
        self.dxy = -(self.cx[0] + self.cx[1])[None, :] - (self.cy[0] + self.cy[1])[:, None]
        self.threads = max(1, threads or (os.cpu_count() or 1))

    def _slab(self, u, out, k0, k1):
        cmx, cpx = self.cx
        cmy, cpy = self.cy
        cmz, cpz = self.cz
        o = out[k0:k1]
        us = u[k0:k1]
        dz = -(cmz[k0:k1] + cpz[k0:k1])[:, None, None]
        np.multiply(self.mass[k0:k1] + self.dxy[None] + dz, us, out=o)
        o[:, :, :-1] += cpx[None, None, :-1] * us[:, :, 1:]
        o[:, :, 1:] += cmx[None, None, 1:] * us[:, :, :-1]
        o[:, :-1, :] += cpy[None, :-1, None] * us[:, 1:, :]
        o[:, 1:, :] += cmy[None, 1:, None] * us[:, :-1, :]
        hi = min(k1, self.shape[0] - 1)
        if hi > k0:
            o[:hi - k0] += cpz[k0:hi, None, None] * u[k0 + 1:hi + 1]
        lo = max(k0, 1)
        if k1 > lo:
            o[lo - k0:] += cmz[lo:k1, None, None] * u[lo - 1:k1 - 1]

    def __call__(self, u: np.ndarray) -> np.ndarray:
        u = u.reshape(self.shape)
        out = np.empty(self.shape, dtype=np.complex128)
        nz = self.shape[0]
        nt = min(self.threads, nz)
        bounds = [(nz * t // nt, nz * (t + 1) // nt) for t in range(nt)]
        with ThreadPoolExecutor(nt) as ex:
            list(ex.map(lambda b: self._slab(u, out, b[0], b[1]), bounds))
        return out


def fgmres(apply_a, apply_m, f: np.ndarray, tol: float = 1e-8, m: int = 20, max_iter: int = 1000,
           max_cycles_iters: int | None = None, log=None):
    """Flexible GMRES(m) with a preallocated basis; the arithmetic of
    oracle.mode_n.fgmres (CGS2, Givens rotations, stop on the rotated
    residual estimate, confirmed by the true residual at the cycle's end).
    Returns (x, iterations, history, true relres, per-iteration seconds)."""
    shape = f.shape
    fv = f.reshape(-1)
    n = fv.size
    nf = np.linalg.norm(fv)
    x = np.zeros(n, dtype=np.complex128)
    V = np.empty((m + 1, n), dtype=np.complex128)
    Z = np.empty((m, n), dtype=np.complex128)
    hist, times = [], []
    it = 0
    while True:
        r = fv - apply_a(x.reshape(shape)).reshape(-1)
        beta = np.linalg.norm(r)
        if beta <= tol * nf or it >= max_iter:
            return x.reshape(shape), it, hist, beta / nf, times
        np.divide(r, beta, out=V[0])
        del r
        H = np.zeros((m + 1, m), dtype=np.complex128)
        cs = np.zeros(m, dtype=np.complex128)
        sn = np.zeros(m, dtype=np.complex128)
        gv = np.zeros(m + 1, dtype=np.complex128)
        gv[0] = beta
        jlast = 0
        for j in range(m):
            t0 = time.perf_counter()
            Z[j] = apply_m(V[j].reshape(shape)).reshape(-1)
            w = apply_a(Z[j].reshape(shape)).reshape(-1)
            for _ in range(2):
                hcol = V[:j + 1].conj() @ w
                H[:j + 1, j] += hcol
                w -= V[:j + 1].T @ hcol
            hn = np.linalg.norm(w)
            H[j + 1, j] = hn
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
            times.append(time.perf_counter() - t0)
            if log is not None:
                log(it, hist[-1], times[-1])
            if hn == 0.0:
                break
            np.divide(w, hn, out=V[j + 1])
            if abs(gv[j + 1]) <= tol * nf or it >= max_iter:
                break
            if max_cycles_iters is not None and it >= max_cycles_iters:
                break
        k = jlast + 1
        y = np.linalg.solve(np.triu(H[:k, :k]), gv[:k])
        x += Z[:k].T @ y
        if max_cycles_iters is not None and it >= max_cycles_iters:
            r = fv - apply_a(x.reshape(shape)).reshape(-1)
            return x.reshape(shape), it, hist, np.linalg.norm(r) / nf, times


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, default=200)
    ap.add_argument("--pml", type=int, default=16)
    ap.add_argument("--source", type=int, default=0)
    ap.add_argument("--restart", type=int, default=20)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--beta-prec", type=float, default=0.25)
    ap.add_argument("--z-transform", default="fft", choices=["fft", "eigen"])
    ap.add_argument("--stride", type=int, default=8)
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(repo, "iterative-helmholtz-solver-with-pardiso_b200"))
    from helm3d import media
    p = media.layered_medium(args.n, args.n, args.n, 10.0, args.pml, 2024, ppw=8.0, n_sources=16)
    f = p.rhs(args.source)
    t0 = time.perf_counter()
    with PortPreconditioner(p, beta_prec=args.beta_prec, workers=args.workers, z_transform=args.z_transform) as pre:
        tf = pre.factor()
        print(f"factor {tf:.1f} s ({args.workers} workers)", flush=True)
        op = PortOperator(p, threads=args.workers)
        x, its, hist, rr, times = fgmres(op, pre.apply, f, tol=args.tol, m=args.restart, max_iter=5000,
                                         log=lambda i, r, t: print(f"it {i} {r:.3e} {t:.2f}s", flush=True))
    total = time.perf_counter() - t0
    print(f"iterations {its} relres {rr:.3e} total {total:.0f} s", flush=True)
    out = args.out or os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                                   f"port_{'fftz' if args.z_transform == 'fft' else 'eigen'}_n{args.n}.npz")
    s = args.stride
    np.savez_compressed(out, n=args.n, pml=args.pml, source=args.source, restart=args.restart, tol=args.tol,
                        beta_prec=args.beta_prec, z_transform=args.z_transform, iterations=its, relres=rr, history=np.array(hist),
                        factor_s=tf, iteration_s=np.array(times), workers=args.workers, stride=s,
                        sample=x[::s, ::s, ::s].copy(), norm=np.linalg.norm(x))
    print("wrote", out)


if __name__ == "__main__":
    main()
