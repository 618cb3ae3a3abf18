"""The adjoint machinery of the oracle, pinned on small grids (CPU only):
the symmetrizing scale behind the adjoint sweep, the adjoint preconditioner,
and the misfit gradient against central finite differences of direct solves."""
import numpy as np
import scipy.sparse as sp

from helpers import rand_c
from oracle import grid as ogrid
from oracle import media, mode_n


def _problem(n=10, pml=2, seed=3, nsrc=2):
    return media.layered_medium(n, n + 1, n - 1, 10.0, pml, seed, ppw=8.0, n_sources=nsrc)


def test_alpha_scaled_2d_system_is_complex_symmetric():
    """Dxy^{-1} S_k is complex symmetric, Dxy = diag(alpha_x(i) alpha_y(j)):
    every coupling is alpha(node) alpha(half node) / h^2, so S_k^{-H} =
    conj(Dxy)^{-1} conj(S_k^{-1}) conj(Dxy) (the adjoint sweep)."""
    p = _problem()
    on = mode_n.setup(p, beta_prec=0.25, factor=False)
    cmx, cpx = on.coef["x"]
    cmy, cpy = on.coef["y"]
    tx = sp.diags([cmx[1:], -(cmx + cpx), cpx[:-1]], [-1, 0, 1]).toarray()
    ty = sp.diags([cmy[1:], -(cmy + cpy), cpy[:-1]], [-1, 0, 1]).toarray()
    shift = on.shifts[3].ravel()
    S = np.kron(np.eye(p.ny), tx) + np.kron(ty, np.eye(p.nx)) + np.diag(shift)
    ax = ogrid.Axis(n=p.nx, h=p.h, pml_pts=p.pml)
    ay = ogrid.Axis(n=p.ny, h=p.h, pml_pts=p.pml)
    d = np.array([ogrid.alpha(ay, j, p.omega) * ogrid.alpha(ax, i, p.omega)
                  for j in range(p.ny) for i in range(p.nx)])
    St = S / d[:, None]
    assert np.abs(St - St.T).max() <= 1e-12 * np.abs(St).max()
    Si = np.linalg.inv(S)
    lhs = Si.conj().T
    rhs = (np.conj(Si) * np.conj(d)[None, :]) / np.conj(d)[:, None]
    assert np.abs(lhs - rhs).max() <= 1e-10 * np.abs(lhs).max()


def test_prec_adjoint_identity_fft_and_eigen():
    p = _problem()
    for zt in ("fft", "eigen"):
        on = mode_n.setup(p, beta_prec=0.25, z_transform=zt)
        x = rand_c(p.shape, seed=1)
        y = rand_c(p.shape, seed=2)
        lhs = np.vdot(y, on.apply_prec(x))
        rhs = np.vdot(on.apply_prec_adjoint(y), x)
        assert abs(lhs - rhs) <= 1e-11 * abs(lhs), zt


def test_assembled_operator_matches_stencil():
    p = _problem()
    on = mode_n.setup(p, factor=False)
    x = rand_c(p.shape, seed=4)
    assert np.linalg.norm(on.assemble_a() @ x.ravel() - on.apply_a(x).ravel()) <= 1e-13 * np.linalg.norm(
        on.apply_a(x))


def _gradient_case(n=10, pml=2):
    p = _problem(n=n, pml=pml)
    F = np.stack([p.rhs(i) for i in range(len(p.sources))])
    recv = mode_n.receiver_plane(p)
    # data from a model with a +10 % slowness-squared anomaly
    true = media.layered_medium(p.nx, p.ny, p.nz, p.h, p.pml, 99, ppw=8.0)
    s2_true = p.s2 * (1.0 + 0.1 * (true.s2 / true.s2.max()))
    on_true = mode_n.setup(p, factor=False)
    import scipy.sparse.linalg as spla
    lu = spla.splu(on_true.assemble_a(s2_true))
    data = np.stack([lu.solve(F[s].ravel())[recv] for s in range(len(F))])
    return p, F, recv, data


def test_gradient_matches_finite_differences():
    p, F, recv, data = _gradient_case()
    on = mode_n.setup(p, factor=False)
    j0, g = mode_n.misfit_grad(on, F, recv, data)
    assert abs(j0 - mode_n.misfit(on, F, recv, data)) <= 1e-12 * j0
    rng = np.random.default_rng(0)
    cells = rng.choice(p.s2.size, 12, replace=False)
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


def test_gradient_fgmres_pair_matches_direct():
    p, F, recv, data = _gradient_case()
    on = mode_n.setup(p, beta_prec=0.25)
    j1, g1 = mode_n.misfit_grad(on, F, recv, data, solver="direct")
    j2, g2 = mode_n.misfit_grad(on, F, recv, data, solver="fgmres", tol=1e-13)
    assert abs(j1 - j2) <= 1e-9 * j1
    assert np.linalg.norm(g1 - g2) <= 1e-8 * np.linalg.norm(g1)
