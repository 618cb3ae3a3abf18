"""Python binding of the helm3d C ABI (include/helm3d.h) over ctypes.

The solver itself is libhelm3d.so (CUDA kernels for sm_100a + C++ host);
this module only marshals arguments.  Vectors are complex128 arrays laid out
(nz, ny, nx); NumPy arrays are passed as host pointers (the library copies
them), torch CUDA tensors as device pointers.  There is no fallback: the
shared library is loaded on first use (``lib``, ``load()``), and if it is
missing that first use raises ImportError.  Importing the package alone
loads nothing, so its pure-Python modules (``helm3d.media``,
``helm3d.formats``) can be used by CPU-only code without the CUDA library.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# HELM3D_LIB selects another build of the same library (e.g. one compiled
# with -DHELM3D_CHECKS, whose kernels check their indices)
LIB_PATH = os.environ.get("HELM3D_LIB") or os.path.join(_HERE, "libhelm3d.so")

_cdll = None

MODE_R, MODE_N = 0, 1
PREC_C128, PREC_C64 = 0, 1
KZ_DISCRETE, KZ_CONTINUOUS, KZ_REFERENCE = 0, 1, 2
ZT_FFT, ZT_PML_EIGEN = 0, 1

OK = 0
ERR_ARG, ERR_OOM, ERR_CUDA, ERR_SINGULAR, ERR_NOT_CONVERGED, ERR_BREAKDOWN, ERR_NONFINITE, ERR_NO_DEVICE = range(1, 9)


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("hx", ctypes.c_double), ("hy", ctypes.c_double), ("hz", ctypes.c_double),
                ("pml_x", ctypes.c_int), ("pml_y", ctypes.c_int), ("pml_z", ctypes.c_int),
                ("spg_z", ctypes.c_int), ("lz", ctypes.c_double), ("omega", ctypes.c_double)]


class Opts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("precision", ctypes.c_int), ("kz_symbol", ctypes.c_int),
                ("beta_prec", ctypes.c_double), ("beta_phys", ctypes.c_double), ("s2_l0", ctypes.c_double),
                ("quirk_q1", ctypes.c_int), ("restart", ctypes.c_int), ("max_iter", ctypes.c_int),
                ("tol", ctypes.c_double), ("stop_phys", ctypes.c_int), ("device", ctypes.c_int),
                ("verbose", ctypes.c_int), ("z_transform", ctypes.c_int), ("kz_skip_ratio", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_int), ("restarts", ctypes.c_int),
                ("relres", ctypes.c_double), ("relres_phys", ctypes.c_double), ("ms_factor", ctypes.c_double),
                ("ms_solve", ctypes.c_double), ("history", ctypes.POINTER(ctypes.c_double)),
                ("history_cap", ctypes.c_int), ("history_len", ctypes.c_int)]


_vp = ctypes.c_void_p
_sig = {
    "helm3d_default_opts": (ctypes.c_int, [ctypes.POINTER(Opts)]),
    "helm3d_create": (ctypes.c_int, [ctypes.POINTER(Grid), _vp, ctypes.POINTER(Opts), ctypes.POINTER(_vp)]),
    "helm3d_set_medium": (ctypes.c_int, [_vp, _vp]),
    "helm3d_solve": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.POINTER(Stats)]),
    "helm3d_solve_medium": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.POINTER(Stats)]),
    "helm3d_solve_group": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp),
                                          ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(Stats)]),
    "helm3d_solve_bicgstab": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(Stats)]),
    "helm3d_solve_adjoint": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(Stats)]),
    "helm3d_apply_op": (ctypes.c_int, [_vp, _vp, _vp]),
    "helm3d_apply_prec_batch": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int]),
    "helm3d_apply_op_adjoint": (ctypes.c_int, [_vp, _vp, _vp]),
    "helm3d_apply_prec": (ctypes.c_int, [_vp, _vp, _vp]),
    "helm3d_apply_prec_adjoint": (ctypes.c_int, [_vp, _vp, _vp]),
    "helm3d_apply_prec_noalloc": (ctypes.c_int, [_vp, _vp, _vp]),
    "helm3d_misfit_grad": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp,
                                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(Stats)]),
    "helm3d_set_stream": (ctypes.c_int, [_vp, _vp]),
    "helm3d_profile": (ctypes.c_int, [_vp, ctypes.c_int]),
    "helm3d_profile_read": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                           ctypes.c_int]),
    "helm3d_device_bytes": (ctypes.c_size_t, [_vp]),
    "helm3d_kernel_launches": (ctypes.c_longlong, [_vp]),
    "helm3d_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "helm3d_last_error": (ctypes.c_char_p, [_vp]),
    "helm3d_destroy": (ctypes.c_int, [_vp]),
}


def load() -> ctypes.CDLL:
    """Load libhelm3d.so (once) and declare the C signatures; raises
    ImportError if the library is not built."""
    global _cdll
    if _cdll is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"helm3d: {LIB_PATH} is not built (run `make` in {os.path.dirname(_HERE)})")
        d = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _sig.items():
            f = getattr(d, name)
            f.restype = res
            f.argtypes = args
        _cdll = d
    return _cdll


class _Lib:
    """``helm3d.lib``: the CDLL, loaded on first attribute access."""

    def __getattr__(self, name):
        return getattr(load(), name)


lib = _Lib()

EXPORTS = tuple(_sig)

KERNEL_KINDS = ("factor", "fft_fwd", "sweep", "fft_inv", "stencil", "krylov")


class Helm3dError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"helm3d status {code} ({lib.helm3d_status_string(code).decode()}): {msg}")
        self.code = code


def default_opts(**kw) -> Opts:
    o = Opts()
    lib.helm3d_default_opts(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(k)
        setattr(o, k, v)
    return o


def _ptr(a):
    """Data pointer of a NumPy array (host) or a torch tensor (device/host)."""
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)


def _c128(a):
    if hasattr(a, "data_ptr"):
        return a
    return np.ascontiguousarray(a, dtype=np.complex128)


class Solver:
    """One set-up solve (grid + medium + options) on one GPU."""

    def __init__(self, grid: Grid, s2, opts: Opts | None = None):
        self.grid = grid
        self.opts = opts if opts is not None else default_opts()
        self.shape = (grid.nz, grid.ny, grid.nx)
        s2 = s2 if hasattr(s2, "data_ptr") else np.ascontiguousarray(s2, dtype=np.float64)
        self._s2 = s2
        h = ctypes.c_void_p()
        rc = lib.helm3d_create(ctypes.byref(grid), _ptr(s2), ctypes.byref(self.opts), ctypes.byref(h))
        if rc != OK:
            raise Helm3dError(rc, "helm3d_create failed: " + (lib.helm3d_last_error(None) or b"").decode())
        self.h = h
        self.last_stats = None

    def close(self):
        if getattr(self, "h", None):
            lib.helm3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, rc, what):
        raise Helm3dError(rc, f"{what}: {lib.helm3d_last_error(self.h).decode()}")

    def _out_like(self, f, nrhs=1):
        if hasattr(f, "data_ptr"):
            import torch
            return torch.empty_like(f)
        return np.empty(((nrhs,) if nrhs > 1 else ()) + self.shape, dtype=np.complex128)

    def solve(self, f, nrhs: int = 1, u=None, history: int = 0, allow_not_converged=False):
        f = _c128(f)
        u = self._out_like(f, nrhs) if u is None else u
        st = Stats()
        hist = None
        if history:
            hist = (ctypes.c_double * history)()
            st.history = hist
            st.history_cap = history
        rc = lib.helm3d_solve(self.h, _ptr(f), _ptr(u), nrhs, ctypes.byref(st))
        if rc != OK and not (allow_not_converged and rc == ERR_NOT_CONVERGED):
            self._err(rc, "solve")
        self.last_stats = st
        self.last_history = list(hist[:st.history_len]) if hist is not None else []
        return u

    def solve_medium(self, s2, f, nrhs: int = 1, u=None, allow_not_converged=False):
        """A new medium, its factor and the solve in one call
        (helm3d_solve_medium): host right-hand sides are copied in while
        the medium is factored."""
        s2 = s2 if hasattr(s2, "data_ptr") else np.ascontiguousarray(s2, dtype=np.float64)
        self._s2 = s2
        f = _c128(f)
        u = self._out_like(f, nrhs) if u is None else u
        st = Stats()
        rc = lib.helm3d_solve_medium(self.h, _ptr(s2), _ptr(f), _ptr(u), nrhs, ctypes.byref(st))
        if rc != OK and not (allow_not_converged and rc == ERR_NOT_CONVERGED):
            self._err(rc, "solve_medium")
        self.last_stats = st
        self.last_history = []
        return u

    def solve_bicgstab(self, f, history: int = 0, allow_not_converged=False):
        f = _c128(f)
        u = self._out_like(f)
        st = Stats()
        hist = None
        if history:
            hist = (ctypes.c_double * history)()
            st.history = hist
            st.history_cap = history
        rc = lib.helm3d_solve_bicgstab(self.h, _ptr(f), _ptr(u), ctypes.byref(st))
        if rc != OK and not (allow_not_converged and rc == ERR_NOT_CONVERGED):
            self._err(rc, "solve_bicgstab")
        self.last_stats = st
        self.last_history = list(hist[:st.history_len]) if hist is not None else []
        return u

    def solve_adjoint(self, g, allow_not_converged=False):
        g = _c128(g)
        lam = self._out_like(g)
        st = Stats()
        rc = lib.helm3d_solve_adjoint(self.h, _ptr(g), _ptr(lam), ctypes.byref(st))
        if rc != OK and not (allow_not_converged and rc == ERR_NOT_CONVERGED):
            self._err(rc, "solve_adjoint")
        self.last_stats = st
        return lam

    def _apply(self, fn, x, what):
        x = _c128(x)
        y = self._out_like(x)
        rc = fn(self.h, _ptr(x), _ptr(y))
        if rc != OK:
            self._err(rc, what)
        return y

    def apply_op(self, x):
        return self._apply(lib.helm3d_apply_op, x, "apply_op")

    def apply_op_adjoint(self, x):
        return self._apply(lib.helm3d_apply_op_adjoint, x, "apply_op_adjoint")

    def apply_prec(self, x):
        return self._apply(lib.helm3d_apply_prec, x, "apply_prec")

    def apply_prec_adjoint(self, x):
        return self._apply(lib.helm3d_apply_prec_adjoint, x, "apply_prec_adjoint")

    def apply_prec_batch(self, X, adjoint=False):
        """M^{-1} (or M^{-H}) of each of the nrhs <= 16 vectors X[r] (shape
        (nrhs, nz, ny, nx)) in one batched apply."""
        X = _c128(X)
        Y = X.new_empty(X.shape) if hasattr(X, "data_ptr") else np.empty(X.shape, dtype=np.complex128)
        rc = lib.helm3d_apply_prec_batch(self.h, _ptr(X), _ptr(Y), int(X.shape[0]), 1 if adjoint else 0)
        if rc != OK:
            self._err(rc, "apply_prec_batch")
        return Y

    def misfit_grad(self, f, recv, data, nsrc: int | None = None, grad=None, allow_not_converged=False):
        """(J, dJ/ds2) for J = 1/2 sum_s ||u_s[recv] - data_s||^2, A u_s = f_s.

        f: (nsrc, nz, ny, nx) complex128, recv: int64 linear indices, data:
        (nsrc, nrecv) complex128; NumPy arrays (host) or torch tensors
        (device).  The gradient comes back like f (a float64 tensor on f's
        device, or a NumPy array)."""
        f = _c128(f)
        nsrc = int(f.shape[0]) if nsrc is None else nsrc
        if hasattr(recv, "data_ptr"):
            recv_c = recv.contiguous()
        else:
            recv_c = np.ascontiguousarray(recv, dtype=np.int64)
        data_c = _c128(data)
        if grad is None:
            if hasattr(f, "data_ptr"):
                import torch
                grad = torch.empty(self.shape, dtype=torch.float64, device=f.device)
            else:
                grad = np.empty(self.shape, dtype=np.float64)
        J = ctypes.c_double()
        st = Stats()
        rc = lib.helm3d_misfit_grad(self.h, _ptr(f), nsrc, _ptr(recv_c), int(recv_c.shape[0]), _ptr(data_c),
                                    _ptr(grad), ctypes.byref(J), ctypes.byref(st))
        if rc != OK and not (allow_not_converged and rc == ERR_NOT_CONVERGED):
            self._err(rc, "misfit_grad")
        self.last_stats = st
        return J.value, grad

    def set_medium(self, s2):
        s2 = s2 if hasattr(s2, "data_ptr") else np.ascontiguousarray(s2, dtype=np.float64)
        self._s2 = s2
        rc = lib.helm3d_set_medium(self.h, _ptr(s2))
        if rc != OK:
            self._err(rc, "set_medium")

    def set_stream(self, stream):
        """Order the solver's work on a CUDA stream (a torch.cuda.Stream, a raw
        handle, or None for the solver's own stream)."""
        handle = None if stream is None else getattr(stream, "cuda_stream", stream)
        rc = lib.helm3d_set_stream(self.h, ctypes.c_void_p(handle) if handle else None)
        if rc != OK:
            self._err(rc, "set_stream")

    def profile(self, enable: bool = True):
        lib.helm3d_profile(self.h, 1 if enable else 0)

    def profile_read(self) -> dict:
        """Summed device ms and launch count per kernel family since the last read."""
        n = len(KERNEL_KINDS)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        rc = lib.helm3d_profile_read(self.h, ms, cnt, n)
        if rc != OK:
            self._err(rc, "profile_read")
        return {k: (ms[i], cnt[i]) for i, k in enumerate(KERNEL_KINDS)}

    @property
    def device_bytes(self) -> int:
        return int(lib.helm3d_device_bytes(self.h))

    @property
    def kernel_launches(self) -> int:
        return int(lib.helm3d_kernel_launches(self.h))


def solve_group(solvers, fs, nrhs=None, us=None, allow_not_converged=False):
    """Solve several Solvers (grids of different sizes) at once: one lockstep
    FGMRES whose restart cycles run as one CUDA graph over all the grids.
    fs[i]: right-hand sides of solvers[i] (NumPy arrays or torch CUDA
    tensors, (nrhs_i, nz, ny, nx) or (nz, ny, nx)).  Returns the solutions,
    each shaped like its right-hand sides, and sets each solver's last_stats."""
    n = len(solvers)
    fs = [_c128(f) for f in fs]
    if nrhs is None:
        nrhs = [int(f.shape[0]) if len(f.shape) == 4 else 1 for f in fs]
    if us is None:
        us = [f.new_empty(f.shape) if hasattr(f, "data_ptr") else np.empty(f.shape, dtype=np.complex128)
              for f in fs]
    hs = (_vp * n)(*[s.h for s in solvers])
    fp = (_vp * n)(*[_ptr(f) for f in fs])
    up = (_vp * n)(*[_ptr(u) for u in us])
    ks = (ctypes.c_int * n)(*nrhs)
    st = (Stats * n)()
    rc = lib.helm3d_solve_group(hs, n, fp, up, ks, st)
    if rc != OK and not (allow_not_converged and rc == ERR_NOT_CONVERGED):
        msgs = "; ".join((lib.helm3d_last_error(s.h) or b"").decode() for s in solvers)
        raise Helm3dError(rc, f"solve_group: {msgs}")
    for s, x in zip(solvers, st):
        s.last_stats = x
    return us


def grid_mode_n(nx, ny, nz, h, pml, omega) -> Grid:
    return Grid(nx=nx, ny=ny, nz=nz, hx=h, hy=h, hz=h, pml_x=pml, pml_y=pml, pml_z=pml, spg_z=0, lz=0.0,
                omega=omega)


def grid_mode_r(nx, ny, nz, hx, hz, pml, spg, lz, omega) -> Grid:
    return Grid(nx=nx, ny=ny, nz=nz, hx=hx, hy=hx, hz=hz, pml_x=pml, pml_y=pml, pml_z=0, spg_z=spg, lz=lz,
                omega=omega)
