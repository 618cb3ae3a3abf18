"""Groups of grids of uneven sizes solved as one (helm3d_solve_group): each
restart cycle of every grid in one CUDA graph.  Every context of the group
returns the solutions that its own solve returns (needs a B200)."""
import numpy as np
import pytest

from helpers import mode_n_solver, mode_r_case, mode_r_solver, rand_c, rel, small_problem
from oracle import mode_n

pytestmark = pytest.mark.gpu


def _group_case():
    import helm3d
    probs = [small_problem(16, 14, 12, pml=3, seed=31), small_problem(20, 20, 20, pml=4, seed=32),
             small_problem(24, 18, 16, pml=4, seed=33)]
    opts = [dict(precision=1), dict(precision=0), dict(precision=1, z_transform=helm3d.ZT_PML_EIGEN)]
    nrhs = [1, 3, 2]
    F = [np.stack([rand_c(p.shape, seed=40 + 7 * i + r) for r in range(k)]) for i, (p, k) in
         enumerate(zip(probs, nrhs))]
    return probs, opts, nrhs, F


@pytest.mark.parametrize("graph", ["1", "0"])
def test_group_matches_single_solves(graph, monkeypatch):
    import helm3d
    monkeypatch.setenv("HELM3D_GRAPH", graph)
    probs, opts, nrhs, F = _group_case()
    solvers = [mode_n_solver(p, tol=1e-10, **o) for p, o in zip(probs, opts)]
    U = helm3d.solve_group(solvers, F)
    its = [s.last_stats.iterations for s in solvers]
    for i, (p, s) in enumerate(zip(probs, solvers)):
        assert s.last_stats.relres < 1e-10
        on = mode_n.setup(p, factor=False)
        single = s.solve(F[i], nrhs=nrhs[i]).reshape(nrhs[i], -1)
        assert U[i].shape == F[i].shape
        ui = U[i].reshape(nrhs[i], -1)
        assert abs(s.last_stats.iterations - its[i]) <= nrhs[i]
        for r in range(nrhs[i]):
            assert np.linalg.norm(on.apply_a(ui[r]) - F[i][r]) / np.linalg.norm(F[i][r]) < 2e-10
            assert rel(ui[r], single[r]) < 1e-8
        s.close()


def test_group_device_buffers_and_mode_r():
    """torch device tensors in and out, a mode R context beside mode N ones."""
    import torch

    import helm3d
    probs, opts, nrhs, F = _group_case()
    solvers = [mode_n_solver(p, tol=1e-10, **o) for p, o in zip(probs[:2], opts[:2])]
    g, st = mode_r_case(10, 4, 3)
    sr = mode_r_solver(g, st, tol=1e-11, max_iter=3000)
    Fr = np.stack([rand_c(g.shape_zyx, seed=61), rand_c(g.shape_zyx, seed=62)])
    fs = [torch.from_numpy(F[0]).cuda(), torch.from_numpy(F[1]).cuda(), torch.from_numpy(Fr).cuda()]
    U = helm3d.solve_group(solvers + [sr], fs)
    for i in range(2):
        for r in range(nrhs[i]):
            assert rel(U[i][r].cpu().numpy(), solvers[i].solve(F[i][r])) < 1e-8
    for r in range(2):
        assert rel(U[2][r].cpu().numpy(), sr.solve(Fr[r])) < 1e-8
    for s in solvers + [sr]:
        s.close()


def test_group_rejects_repeated_context():
    import helm3d
    p = small_problem(16, 14, 12, pml=3, seed=31)
    s = mode_n_solver(p)
    f = rand_c(p.shape, seed=1)
    with pytest.raises(helm3d.Helm3dError):
        helm3d.solve_group([s, s], [f, f])
    s.close()
