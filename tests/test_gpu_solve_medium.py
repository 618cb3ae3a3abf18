"""helm3d_solve_medium (a new medium, its factor and the solve in one call,
as the reference's FGMRES sets up, factors and solves in one call:
Source/FGMRES.cpp:72-298, :300-725) on the GPU: the same solutions as
helm3d_set_medium followed by helm3d_solve, bit for bit (the same kernels in
the same order; only the host right-hand sides' copy moves under the
factor), with host and device buffers, a batch larger than one lockstep
batch, and a failed factor reported by the call and refused by later
solves (needs a B200)."""
import ctypes
import dataclasses

import numpy as np
import pytest

from helpers import mode_n_solver, rand_c, small_problem
from oracle import mode_n

pytestmark = pytest.mark.gpu


def _rhs(p, n, seed):
    return np.stack([rand_c(p.shape, seed=seed + r) for r in range(n)])


@pytest.mark.parametrize("zt,nrhs", [(0, 3), (1, 3), (1, 17)])
def test_solve_medium_equals_set_medium_then_solve_host(zt, nrhs):
    """Host (pinned and pageable) buffers; 17 sources exceed one lockstep
    batch of 16, so the call stages them batch by batch itself."""
    import torch
    p = small_problem(20, 18, 16, pml=3, seed=31)
    # a second medium on the same grid and frequency: +-5 % on s2
    rng = np.random.default_rng(32)
    q = dataclasses.replace(p, s2=np.ascontiguousarray(p.s2 * (1.0 + 0.05 * rng.uniform(-1, 1, p.s2.shape))))
    F = _rhs(p, nrhs, 40)
    s = mode_n_solver(p, precision=1, z_transform=zt, tol=1e-9)
    s.set_medium(q.s2)
    U0 = s.solve(F, nrhs=nrhs)
    its0 = s.last_stats.iterations
    U1 = s.solve_medium(q.s2, F, nrhs=nrhs)
    assert s.last_stats.iterations == its0
    assert np.array_equal(U0, U1)
    Fp = torch.from_numpy(F).pin_memory()
    Up = torch.empty_like(Fp).pin_memory()
    s.solve_medium(q.s2, Fp, nrhs=nrhs, u=Up)
    assert np.array_equal(Up.numpy(), U0)
    on = mode_n.setup(q, factor=False)
    for r in range(nrhs):
        assert np.linalg.norm(on.apply_a(U1[r]) - F[r]) / np.linalg.norm(F[r]) < 2e-9
    s.close()


def test_solve_medium_device_buffers():
    import torch
    p = small_problem(24, 20, 18, pml=3, seed=33)
    F = _rhs(p, 4, 50)
    s = mode_n_solver(p, precision=1, z_transform=1, tol=1e-9)
    U0 = s.solve(F, nrhs=4)
    s2d = torch.from_numpy(np.ascontiguousarray(p.s2)).to("cuda:0")
    Fd = torch.from_numpy(F).to("cuda:0")
    Ud = s.solve_medium(s2d, Fd, nrhs=4)
    assert np.array_equal(Ud.cpu().numpy(), U0)
    s.close()


def test_solve_medium_failed_factor_is_reported_and_refused():
    """A NaN in the medium: the call returns HELM3D_ERR_NONFINITE (the host
    right-hand sides were already being copied in), later solves of the
    context return it too, and a good medium through the same call makes
    the context usable again."""
    import helm3d
    p = small_problem(20, 18, 16, pml=3, seed=34)
    s = mode_n_solver(p, precision=1, z_transform=1, tol=1e-9)
    F = np.ascontiguousarray(_rhs(p, 2, 60))
    U = np.empty_like(F)
    bad = p.s2.copy()
    bad[3, 2, 1] = np.nan
    bad = np.ascontiguousarray(bad)
    st = helm3d.Stats()
    rc = helm3d.lib.helm3d_solve_medium(s.h, bad.ctypes.data, F.ctypes.data, U.ctypes.data, 2, ctypes.byref(st))
    assert rc == helm3d.ERR_NONFINITE, rc
    rc = helm3d.lib.helm3d_solve(s.h, F.ctypes.data, U.ctypes.data, 2, ctypes.byref(st))
    assert rc == helm3d.ERR_NONFINITE, rc
    U1 = s.solve_medium(p.s2, F, nrhs=2)
    on = mode_n.setup(p, factor=False)
    for r in range(2):
        assert np.linalg.norm(on.apply_a(U1[r]) - F[r]) / np.linalg.norm(F[r]) < 2e-9
    s.close()
