"""helm3d_apply_prec_noalloc against helm3d_apply_prec, through the C ABI.

The no-alloc entry point serves callers that cannot allocate device memory
where they apply the preconditioner (allocator/pool callbacks, memory held by
a caching allocator, paths that must avoid cudaMalloc's synchronization); its
planes live in a fixed static device array instead.  This file is collected
last so that a failing run that stops at the first failure has run every
other test already; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from helpers import mode_n_solver, mode_r_case, mode_r_solver, small_problem

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    import helm3d
    fn = helm3d.lib.helm3d_apply_prec_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def _check_two_calls(s, shape, tol, seed=5):
    """Two calls in a row (they share, and reuse, the static planes), each
    against helm3d_apply_prec of the same vector."""
    import torch

    import helm3d
    fn = _noalloc_fn()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(seed)
    for call in range(2):
        x = torch.from_numpy(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).to(dev)
        y_ref = s.apply_prec(x)
        y = torch.full_like(x, float("nan"))
        rc = fn(s.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()))
        assert rc == helm3d.OK, helm3d.lib.helm3d_last_error(s.h)
        err = float(torch.linalg.vector_norm(y - y_ref) / torch.linalg.vector_norm(y_ref))
        assert err <= tol, (call, err)


# every branch the entry point dispatches: the z-FFT (complex64 and
# complex128 planes), the FP64 PML-eigenbasis z-transform (complex128) and
# the tensor-core eigenbasis z-transform (complex64)
@pytest.mark.parametrize("prec,zt", [(1, 0), (0, 0), (0, 1), (1, 1)])
def test_apply_prec_noalloc_matches_apply_prec(prec, zt):
    p = small_problem(24, 20, 18, pml=4, seed=21)
    s = mode_n_solver(p, precision=prec, z_transform=zt)
    _check_two_calls(s, p.shape, 1e-10 if prec == 0 else 2e-5)


def test_apply_prec_noalloc_mode_r():
    """The reference's own operator (mode R): L0^{-1} by the z-FFT, complex128."""
    g, st = mode_r_case(10, 4, 3)
    s = mode_r_solver(g, st)
    _check_two_calls(s, g.shape_zyx, 1e-10, seed=9)


def test_apply_prec_noalloc_rejects_oversize_and_host_pointers():
    import torch

    import helm3d

    fn = _noalloc_fn()
    # 112 x 112 x 96 complex128 planes = 19 MB > 8 MiB
    p = small_problem(112, 112, 96, pml=4, seed=3)
    s = mode_n_solver(p, precision=0)
    dev = torch.device("cuda", 0)
    x = torch.zeros(p.shape, dtype=torch.complex128, device=dev)
    y = torch.zeros_like(x)
    assert fn(s.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr())) == helm3d.ERR_ARG
    assert b"8 MiB" in helm3d.lib.helm3d_last_error(s.h)
    q = small_problem(16, 16, 16, pml=3, seed=4)
    t = mode_n_solver(q, precision=1)
    xh = np.zeros(q.shape, dtype=np.complex128)
    yh = np.zeros_like(xh)
    assert fn(t.h, ctypes.c_void_p(xh.ctypes.data), ctypes.c_void_p(yh.ctypes.data)) == helm3d.ERR_ARG
    # x and y on another GPU than the context's
    if torch.cuda.device_count() > 1:
        x1 = torch.zeros(q.shape, dtype=torch.complex128, device=torch.device("cuda", 1))
        y1 = torch.zeros_like(x1)
        assert fn(t.h, ctypes.c_void_p(x1.data_ptr()), ctypes.c_void_p(y1.data_ptr())) == helm3d.ERR_ARG
        assert b"context's device" in helm3d.lib.helm3d_last_error(t.h)
