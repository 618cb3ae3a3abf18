"""Skipped kz modes (opts.kz_skip_ratio, the reference's SAVE_MEM switch,
Source/FGMRES.cpp:197-206) on the GPU against the oracle (needs a B200).

Mode R: the modes with kww >= 5 k2 of the 58^3 reference grid (26..32, the
ones the reference itself skipped, tests/golden/ref_fgmres_savemem_*) are
neither factored nor solved; L0^{-1} matches the oracle's SAVE_MEM
restatement to 1e-10 and the solve the oracle's solution to 1e-6.
Mode N: skipped modes are solved by the diagonal of their 2D operator;
M^{-1} and M^{-H} match the oracle's (1e-9 complex128, 5e-5 complex64) for
every factor and sweep kind (CUDA-core, tensor-core, packed), and FGMRES
reaches the requested residual, measured with the oracle's FP64 operator.
Tolerances as in test_gpu_parity."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import mode_n_solver, mode_r_solver, rand_c, rel, small_problem
from oracle import grid as ogrid
from oracle import mode_n, mode_r

pytestmark = pytest.mark.gpu


def test_mode_r_savemem_l0_inverse_and_solve():
    z = np.load(os.path.join(GOLDEN, "ref_fgmres_savemem_n50p4s4.npz"))
    n, pml, spg, beta, niter, rest = z["params"]
    g = ogrid.reference_grid(int(n), int(pml), int(spg))
    st = mode_r.setup(g, beta=float(beta), media="homo", kz_skip_ratio=5.0)
    assert np.flatnonzero(st.skip).tolist() == z["skipped"].tolist()
    s = mode_r_solver(g, st, beta=float(beta), tol=1e-11, max_iter=3000, kz_skip_ratio=5.0)
    v = rand_c(g.shape_zyx, seed=4)
    assert rel(s.apply_prec(v), st.l0_solve(v)) < 1e-10
    assert rel(s.apply_op(v), st.apply_k(v)) < 1e-10
    f = mode_r.point_source_rhs(g)
    u = s.solve(f)
    assert s.last_stats.relres < 1e-10
    w = mode_n.fgmres(st.apply_k, lambda x: x, f, tol=1e-12, m=30, max_iter=3000).x
    assert rel(u, st.l0_solve(w)) < 1e-6
    # the same settings without skipping give another L0^{-1}
    s0 = mode_r_solver(g, st, beta=float(beta), tol=1e-11, max_iter=3000)
    assert rel(s0.apply_prec(v), st.l0_solve(v)) > 1e-6
    s.close()
    s0.close()


@pytest.mark.parametrize("prec,zt,nx,sweep", [(0, "fft", 24, None), (1, "fft", 24, None), (1, "eigen", 24, None),
                                              (1, "eigen", 128, 9), (1, "eigen", 128, 8), (1, "eigen", 200, 9),
                                              (1, "eigen", 24, 0)])
def test_mode_n_skip_preconditioner(prec, zt, nx, sweep, monkeypatch):
    """M^{-1} and M^{-H} with skipped modes, batched (3 vectors); block sizes
    24 (register factor), 128 (tensor-core factor, one CTA per kz) and 200
    (the CTA-pair factor); sweep variants forced where given."""
    import helm3d
    if sweep is not None:
        monkeypatch.setenv("HELM3D_FORCE_SWEEP", str(sweep))
    p = small_problem(nx, 10, 40, pml=4, seed=nx + 7)
    on = mode_n.setup(p, beta_prec=0.25, z_transform=zt, kz_skip_ratio=2.0)
    assert 0 < on.skip.sum() < p.nz
    X = np.stack([rand_c(p.shape, seed=110 + r) for r in range(3)])
    s = mode_n_solver(p, precision=prec, z_transform=helm3d.ZT_PML_EIGEN if zt == "eigen" else helm3d.ZT_FFT,
                      kz_skip_ratio=2.0)
    Y = s.apply_prec_batch(X)
    Yh = s.apply_prec_batch(X, adjoint=True)
    tol = 1e-9 if prec == 0 else 5e-5
    for r in range(3):
        assert rel(Y[r], on.apply_prec(X[r])) < tol, r
        assert rel(Yh[r], on.apply_prec_adjoint(X[r])) < tol, r
    # one vector through the single apply (and the no-alloc entry point's sweep)
    assert rel(s.apply_prec(X[0]), on.apply_prec(X[0])) < tol
    s.close()


@pytest.mark.parametrize("zt", ["fft", "eigen"])
def test_mode_n_skip_fgmres(zt):
    """FGMRES with skipped modes (ratio 2) reaches the requested residual,
    measured with the oracle's FP64 operator, for 3 batched sources."""
    import helm3d
    p = small_problem(24, 20, 40, pml=4, seed=95)
    on = mode_n.setup(p, factor=False)
    F = np.stack([rand_c(p.shape, seed=120 + r) for r in range(3)])
    s = mode_n_solver(p, precision=1, tol=1e-10, z_transform=helm3d.ZT_PML_EIGEN if zt == "eigen" else helm3d.ZT_FFT,
                      kz_skip_ratio=2.0)
    U = s.solve(F, nrhs=3)
    for r in range(3):
        assert np.linalg.norm(on.apply_a(U[r]) - F[r]) / np.linalg.norm(F[r]) < 2e-10
    s.close()
