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

from helpers import mode_n_solver, small_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [1, 0])
def test_apply_prec_noalloc_matches_apply_prec(prec):
    import torch

    import helm3d

    fn = helm3d.lib.helm3d_apply_prec_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    p = small_problem(24, 20, 18, pml=4, seed=21)
    s = mode_n_solver(p, precision=prec)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    tol = 1e-10 if prec == 0 else 2e-5
    for call in range(2):   # two calls in a row share (and reuse) the static planes
        x = torch.from_numpy(rng.standard_normal(p.shape) + 1j * rng.standard_normal(p.shape)).to(dev)
        y_ref = s.apply_prec(x)
        y = torch.full_like(x, float("nan"))
        rc = fn(s.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()))
        assert rc == helm3d.OK, helm3d.lib.helm3d_last_error(s.h)
        err = float(torch.linalg.vector_norm(y - y_ref) / torch.linalg.vector_norm(y_ref))
        assert err <= tol, (call, err)


def test_apply_prec_noalloc_rejects_oversize_and_host_pointers():
    import torch

    import helm3d

    fn = helm3d.lib.helm3d_apply_prec_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
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
