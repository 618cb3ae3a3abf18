"""Adjoint preconditioner, adjoint solve and the misfit gradient on the GPU
against the oracle (needs a B200).

Tolerances: the complex128 adjoint preconditioner agrees with the oracle's
(M^{-1})^H to 1e-9 (complex64: 2e-5 FFT, 1e-3 eigenbasis); the gradient from
complex128 solves to 1e-8 relative residual agrees with the oracle's
direct-solve gradient to 1e-6 and with central finite differences of direct
solves to 1e-4 on 20 seeded cells.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from helpers import mode_n_solver, rand_c, rel, small_problem
from oracle import media, mode_n

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("zt", ["fft", "eigen"])
@pytest.mark.parametrize("prec", [0, 1])
def test_prec_adjoint_matches_oracle(zt, prec):
    import helm3d
    p = small_problem(20, 18, 16, pml=4, seed=5)
    on = mode_n.setup(p, beta_prec=0.25, z_transform=zt)
    s = mode_n_solver(p, precision=prec, beta_prec=0.25,
                      z_transform=helm3d.ZT_PML_EIGEN if zt == "eigen" else helm3d.ZT_FFT)
    v = rand_c(p.shape, seed=3)
    tol = 1e-9 if prec == 0 else (2e-5 if zt == "fft" else 1e-3)
    assert rel(s.apply_prec_adjoint(v), on.apply_prec_adjoint(v)) < tol
    if prec == 0:
        x = rand_c(p.shape, seed=4)
        lhs = np.vdot(v, s.apply_prec(x))
        rhs = np.vdot(s.apply_prec_adjoint(v), x)
        assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


@pytest.mark.parametrize("prec", [0, 1])
def test_adjoint_solve(prec):
    p = media.config_small(24, 4, seed=6)
    on = mode_n.setup(p, factor=False)
    s = mode_n_solver(p, precision=prec, tol=1e-10)
    g = rand_c(p.shape, seed=9)
    lam = s.solve_adjoint(g)
    adj_its = s.last_stats.iterations
    assert np.linalg.norm(on.apply_a_adjoint(lam) - g) / np.linalg.norm(g) < 2e-10
    s.solve(g)
    assert adj_its <= 1.5 * s.last_stats.iterations + 5


def _gradient_case(n=16, pml=3, nsrc=3):
    p = media.layered_medium(n, n, n, 10.0, pml, 21, ppw=8.0, n_sources=nsrc)
    F = np.stack([p.rhs(i) for i in range(nsrc)])
    recv = mode_n.receiver_plane(p)
    true = media.layered_medium(n, n, n, 10.0, pml, 77, ppw=8.0)
    s2_true = p.s2 * (1.0 + 0.1 * (true.s2 / true.s2.max()))
    on = mode_n.setup(p, factor=False)
    lu = spla.splu(on.assemble_a(s2_true))
    data = np.stack([lu.solve(F[s].ravel())[recv] for s in range(nsrc)])
    return p, on, F, recv, data


@pytest.mark.parametrize("prec", [0, 1])
def test_misfit_gradient_matches_oracle_and_finite_differences(prec):
    p, on, F, recv, data = _gradient_case()
    s = mode_n_solver(p, precision=prec, tol=1e-12, max_iter=5000)
    J, g = s.misfit_grad(F, recv, data)
    J0, g0 = mode_n.misfit_grad(on, F, recv, data)   # two direct solves per source
    assert abs(J - J0) <= 1e-9 * J0
    assert np.linalg.norm(g - g0) <= 1e-6 * np.linalg.norm(g0)
    rng = np.random.default_rng(1234)
    cells = rng.choice(p.s2.size, 20, replace=False)
    gmax = np.abs(g).max()
    for l in cells:
        eps = 1e-4 * p.s2.ravel()[l]
        s2p = p.s2.copy().ravel()
        s2m = p.s2.copy().ravel()
        s2p[l] += eps
        s2m[l] -= eps
        fd = (mode_n.misfit(on, F, recv, data, s2p.reshape(p.shape)) -
              mode_n.misfit(on, F, recv, data, s2m.reshape(p.shape))) / (2 * eps)
        gl = g.ravel()[l]
        assert abs(fd - gl) <= 1e-4 * max(abs(gl), 1e-3 * gmax), (l, fd, gl)


def test_misfit_gradient_batches_and_device_buffers():
    """18 sources (two lockstep batches) with device buffers equal the sum of
    single-source gradients."""
    import torch
    p, on, F, recv, data = _gradient_case(n=12, pml=2, nsrc=18)
    s = mode_n_solver(p, precision=1, tol=1e-11, max_iter=5000)
    dev = torch.device("cuda", 0)
    J, g = s.misfit_grad(torch.from_numpy(F).to(dev), torch.from_numpy(recv).to(dev),
                         torch.from_numpy(data).to(dev))
    g = g.cpu().numpy()
    Js, gs = 0.0, np.zeros(p.shape)
    for i in range(18):
        Ji, gi = s.misfit_grad(F[i:i + 1], recv, data[i:i + 1])
        Js += Ji
        gs += gi
    assert abs(J - Js) <= 1e-9 * Js
    assert np.linalg.norm(g - gs) <= 1e-7 * np.linalg.norm(gs)


def test_autograd_binding():
    import torch

    from helm3d import autograd as hag
    p, on, F, recv, data = _gradient_case(n=12, pml=2, nsrc=2)
    s = mode_n_solver(p, precision=0, tol=1e-12, max_iter=5000)
    dev = torch.device("cuda", 0)
    s2 = torch.from_numpy(p.s2.copy()).to(dev).requires_grad_(True)
    J = hag.misfit(s2, s, torch.from_numpy(F).to(dev), torch.from_numpy(recv).to(dev),
                   torch.from_numpy(data).to(dev))
    (2.0 * J).backward()
    J0, g0 = mode_n.misfit_grad(on, F, recv, data)
    assert abs(J.item() - J0) <= 1e-9 * J0
    assert np.linalg.norm(s2.grad.cpu().numpy() - 2.0 * g0) <= 1e-6 * np.linalg.norm(2.0 * g0)
