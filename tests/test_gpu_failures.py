"""Failure paths of the C ABI on the GPU, each made on the host or by a
short wait limit, none of them faulting the GPU: every call returns its
status code, and the device and the context stay usable afterwards.

The reference only prints solver errors and carries on
(Source/FGMRES.cpp:276,284; Source/functions.cpp:5961); here every entry
point returns a helm3d_status.
"""
import ctypes

import numpy as np
import pytest

from helpers import mode_n_solver, rand_c, rel, small_problem
from oracle import mode_n

pytestmark = pytest.mark.gpu


def _solve_rc(s, f):
    import helm3d
    f = np.ascontiguousarray(f, dtype=np.complex128)
    u = np.empty_like(f)
    st = helm3d.Stats()
    rc = helm3d.lib.helm3d_solve(s.h, f.ctypes.data, u.ctypes.data, 1, ctypes.byref(st))
    return rc, st, u


def test_nonfinite_right_hand_side():
    """A NaN in f is reported as HELM3D_ERR_NONFINITE; the next solve of the
    same context converges."""
    import helm3d
    p = small_problem(20, 18, 16, pml=3, seed=5)
    s = mode_n_solver(p, precision=1)
    f = p.rhs(0).copy()
    f[3, 4, 5] = np.nan
    rc, _, _ = _solve_rc(s, f)
    assert rc == helm3d.ERR_NONFINITE, rc
    rc, st, _ = _solve_rc(s, p.rhs(0))
    assert rc == helm3d.OK and st.relres <= 1e-10
    s.close()


def test_iteration_cap_is_not_converged():
    """max_iter = 1: HELM3D_ERR_NOT_CONVERGED after one iteration, with the
    residual reached so far in the stats and the iterate in u."""
    import helm3d
    p = small_problem(20, 18, 16, pml=3, seed=6)
    s = mode_n_solver(p, precision=1, max_iter=1)
    rc, st, u = _solve_rc(s, p.rhs(0))
    assert rc == helm3d.ERR_NOT_CONVERGED, rc
    assert st.status == helm3d.ERR_NOT_CONVERGED and st.iterations == 1
    assert 0 < st.relres < 1 and np.all(np.isfinite(u))
    s.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_exactly_singular_block(prec):
    """An exactly singular 2D system: 3 x 3 x 4 grid without PML, h = 1,
    omega = 2, s2 = 1, no shift, FFT along z.  The block of kz = 0 on the
    first line is tridiag(1, 4 - 2 - 2, 1) = tridiag(1, 0, 1), singular for
    n = 3, and every value of its elimination is an exact small integer, so
    a pivot is exactly zero: helm3d_create reports HELM3D_ERR_SINGULAR."""
    import helm3d
    g = helm3d.Grid(nx=3, ny=3, nz=4, hx=1.0, hy=1.0, hz=1.0, pml_x=0, pml_y=0, pml_z=0, spg_z=0, lz=0.0,
                    omega=2.0)
    o = helm3d.default_opts(precision=prec, beta_prec=0.0, z_transform=helm3d.ZT_FFT)
    s2 = np.ones(3 * 3 * 4)
    h = ctypes.c_void_p()
    rc = helm3d.lib.helm3d_create(ctypes.byref(g), s2.ctypes.data, ctypes.byref(o), ctypes.byref(h))
    assert rc == helm3d.ERR_SINGULAR, rc
    assert b"zero pivot" in helm3d.lib.helm3d_last_error(None)
    # a regular medium on the same grid factors
    s2[:] = 0.3
    rc = helm3d.lib.helm3d_create(ctypes.byref(g), s2.ctypes.data, ctypes.byref(o), ctypes.byref(h))
    assert rc == helm3d.OK, rc
    helm3d.lib.helm3d_destroy(h)


def test_device_memory_exhausted_then_recovers():
    """A grid whose block factor (nz ny nx^2 complex64 = 215 GB) exceeds the
    device's memory (192 GB on a B200): helm3d_create returns HELM3D_ERR_OOM
    and frees what it took; a small context on the same device works right
    after."""
    import helm3d
    nx, ny, nz = 256, 256, 1600
    g = helm3d.grid_mode_n(nx, ny, nz, 10.0, 8, 2 * np.pi * 1500 / 80.0)
    o = helm3d.default_opts(precision=helm3d.PREC_C64, z_transform=helm3d.ZT_FFT)
    s2 = np.full(nx * ny * nz, 1.0 / 1500.0 ** 2)
    h = ctypes.c_void_p()
    rc = helm3d.lib.helm3d_create(ctypes.byref(g), s2.ctypes.data, ctypes.byref(o), ctypes.byref(h))
    del s2
    assert rc == helm3d.ERR_OOM, rc
    p = small_problem(16, 16, 16, pml=3, seed=7)
    s = mode_n_solver(p, precision=1)
    rc, st, _ = _solve_rc(s, p.rhs(0))
    assert rc == helm3d.OK and st.relres <= 1e-10
    s.close()


def test_expired_wait_is_reported_and_the_context_recovers(monkeypatch):
    """A bounded wait that runs out: with HELM3D_TEST_EXPIRE_WAIT (read at
    launch) the block sweep's consumers first wait on a barrier that nothing
    arrives on, limited to 64 polls (HELM3D_WAIT_LIMIT); the wait expires,
    the kernel sets its status bit and finishes without waiting (its copies
    drained), and the apply returns HELM3D_ERR_CUDA.  Without the switch,
    the next apply of the same context is right."""
    import helm3d
    p = small_problem(24, 20, 18, pml=4, seed=8)
    on = mode_n.setup(p, beta_prec=0.25)
    v = rand_c(p.shape, seed=4)
    s = mode_n_solver(p, precision=1)
    monkeypatch.setenv("HELM3D_FORCE_SWEEP", "0")
    monkeypatch.setenv("HELM3D_WAIT_LIMIT", "64")
    monkeypatch.setenv("HELM3D_TEST_EXPIRE_WAIT", "1")
    y = np.empty_like(v)
    rc = helm3d.lib.helm3d_apply_prec(s.h, np.ascontiguousarray(v).ctypes.data, y.ctypes.data)
    assert rc == helm3d.ERR_CUDA, rc
    assert b"bounded wait" in helm3d.lib.helm3d_last_error(s.h)
    monkeypatch.delenv("HELM3D_TEST_EXPIRE_WAIT")
    monkeypatch.delenv("HELM3D_WAIT_LIMIT")
    assert rel(s.apply_prec(v), on.apply_prec(v)) < 5e-5
    s.close()


def test_failed_set_medium_refuses_solves():
    """After set_medium fails (a NaN in the medium: HELM3D_ERR_NONFINITE),
    solves of that context return the same error instead of using a
    broken factor; a good medium makes it usable again."""
    import helm3d
    p = small_problem(20, 18, 16, pml=3, seed=9)
    s = mode_n_solver(p, precision=1)
    bad = p.s2.copy()
    bad[2, 2, 2] = np.nan
    rc = helm3d.lib.helm3d_set_medium(s.h, np.ascontiguousarray(bad).ctypes.data)
    assert rc == helm3d.ERR_NONFINITE, rc
    rc, _, _ = _solve_rc(s, p.rhs(0))
    assert rc == helm3d.ERR_NONFINITE, rc
    s.set_medium(p.s2)
    rc, st, _ = _solve_rc(s, p.rhs(0))
    assert rc == helm3d.OK and st.relres <= 1e-10
    s.close()
