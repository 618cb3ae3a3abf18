"""Every launch shape the autotuner may pick computes what the default shape
computes: each factor shape of a block size, each sweep stage/ring size,
each stencil z chunk and each reduction grid, forced one at a time
(HELM3D_FORCE_<FAMILY>=v) and checked against the FP64 oracle or the default
(needs a B200).  Tolerances as in test_gpu_parity: 1e-9 (complex128
preconditioner), 5e-5 (complex64), solutions 1e-8 relative to the default."""
import numpy as np
import pytest

from helpers import mode_n_solver, rand_c, rel, small_problem
from oracle import mode_n

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,nx,nv", [(1, 128, 3), (1, 100, 3), (1, 40, 2), (1, 17, 2), (1, 200, 3), (1, 201, 3),
                                         (1, 224, 3), (1, 129, 2), (1, 250, 2), (0, 200, 1), (0, 128, 1)])
def test_factor_shapes(prec, nx, nv, monkeypatch):
    """Block sizes 128 (one CTA or a pair per kz), 200 (padded to 224: 4- or
    8-CTA clusters) and 250 (padded to 256) against the oracle, every shape;
    complex64 blocks of n <= 128 (128, 100, 40, 17: full and partial panels)
    also with the tensor-core factor, and of 128 < n <= 224 (129, 200, 201,
    224: even and odd splits over the CTA pair, full and partial last
    panels) with the CTA-pair tensor-core factor (the last variant)."""
    p = small_problem(nx, 10, 8, pml=3, seed=nx + prec)
    on = mode_n.setup(p, beta_prec=0.25)
    v = rand_c(p.shape, seed=3)
    ref = on.apply_prec(v)
    tol = 1e-9 if prec == 0 else 5e-5
    for var in range(nv):
        monkeypatch.setenv("HELM3D_FORCE_FACTOR", str(var))
        s = mode_n_solver(p, precision=prec, beta_prec=0.25)
        assert rel(s.apply_prec(v), ref) < tol, (nx, var)
        s.close()


@pytest.mark.parametrize("family,count", [("SWEEP", 10), ("STENCIL", 12), ("REDUCE", 3), ("UPDATE", 2)])
@pytest.mark.parametrize("nrhs", [1, 3])
def test_solve_shapes_agree(family, count, nrhs, monkeypatch):
    """A batched solve with every variant of one family forced: the same
    solutions (one right-hand side: the plain sweep; three: the register-
    tiled sweep), each at the requested residual."""
    p = small_problem(24, 20, 18, pml=4, seed=71)
    F = np.stack([rand_c(p.shape, seed=80 + r) for r in range(nrhs)])
    on = mode_n.setup(p, factor=False)
    base = None
    for var in range(count):
        monkeypatch.setenv(f"HELM3D_FORCE_{family}", str(var))
        s = mode_n_solver(p, precision=1, tol=1e-10)
        U = s.solve(F, nrhs=nrhs)
        assert s.last_stats.relres < 1e-10
        for r in range(nrhs):
            f = F[r]
            u = U[r] if nrhs > 1 else U
            assert np.linalg.norm(on.apply_a(u) - f) / np.linalg.norm(f) < 2e-10
        if base is None:
            base = U
        else:
            assert rel(U, base) < 1e-8, (family, var)
        s.close()


@pytest.mark.parametrize("nx,nrhs", [(128, 16), (96, 8), (100, 3), (24, 16), (20, 5), (200, 16), (160, 5), (129, 3),
                                     (250, 1), (9, 2)])
def test_tensor_core_sweep_batches(nx, nrhs, monkeypatch):
    """The tensor-core sweep (variants 6 and 7: G^T chunks of 32 and 16 rows,
    3xTF32 products; variant 8: FP16 hi/lo products with power-of-two block
    and right-hand-side scales; variant 9: the same products on the factor
    packed once into FP16 hi/lo tiles) in a batched complex64 preconditioner
    apply, forward and adjoint, against the oracle's M^{-1} x_r and M^{-H} x_r
    of every vector, beside the CUDA-core sweep (variant 0); block sizes one
    full row block (128), padded (96, 100, 24, 20, 9), two row blocks (200,
    160, 129, 250), batches padded to 8 or 16."""
    p = small_problem(nx, 10, 8, pml=3, seed=nx + nrhs)
    on = mode_n.setup(p, beta_prec=0.25)
    X = np.stack([rand_c(p.shape, seed=100 + r) for r in range(nrhs)])
    ref = [on.apply_prec(X[r]) for r in range(nrhs)]
    refh = [on.apply_prec_adjoint(X[r]) for r in range(nrhs)]
    s = mode_n_solver(p, precision=1, beta_prec=0.25)
    for var in (0, 6, 7, 8, 9):
        monkeypatch.setenv("HELM3D_FORCE_SWEEP", str(var))
        Y = s.apply_prec_batch(X)
        Yh = s.apply_prec_batch(X, adjoint=True)
        for r in range(nrhs):
            assert rel(Y[r], ref[r]) < 5e-5, (var, r)
            assert rel(Yh[r], refh[r]) < 5e-5, (var, r)
    s.close()


def test_tune_cache_file(tmp_path, monkeypatch):
    """With HELM3D_TUNE_CACHE the choices are written to the file, one
    `family|shape variant` line each (a shape not tuned before in this
    process: 26 x 22 x 14)."""
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("HELM3D_TUNE_CACHE", str(path))
    p = small_problem(26, 22, 14, pml=4, seed=72)
    s = mode_n_solver(p, precision=1, tol=1e-9)
    s.solve(rand_c(p.shape, seed=9))
    s.close()
    if not path.exists():
        # the process read another cache file first (the path is read once
        # per process); nothing to check then
        pytest.skip("tuning cache path fixed earlier in this process")
    lines = [ln.split() for ln in path.read_text().splitlines() if ln.strip()]
    fams = {ln[0].split("|")[0] for ln in lines}
    assert {"SWEEP", "STENCIL", "REDUCE"} <= fams
    assert all(int(ln[1]) >= 0 for ln in lines)
