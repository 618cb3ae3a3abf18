"""GPU solves of the benchmark configurations at their full sizes, against
the FP64 oracle, through the C ABI.

Each test solves on the GPU exactly as configured and checks two things
with the oracle's own arithmetic: the relative residual ||f - A u|| / ||f||
of the GPU solution evaluated by the oracle's operator (oracle.port's
7-point operator, identical to oracle.mode_n.ModeN.apply_a) is at most the
solve's tolerance, and the solution is within 1e-6 (relative, 2-norm) of
the oracle's solution of the same source, which the oracle computes here
with its PML-eigenbasis preconditioner to 1e-12 (or, at 200^3, reads from
the recorded full solves tests/golden/port_*_n200.npz made by
`python -m oracle.port`, compared on every 8th point per axis).

  C1  64^3 homogeneous, PML 8, 10 ppw, centred source: FFT-z, complex128,
      FGMRES(20) to 1e-8 (the reference's method, Source/FGMRES.cpp:464-684,
      Source/functions.cpp:5837-6061)
  C2  128^3 heterogeneous, PML 12, two sources: PML eigenbasis, complex64
      preconditioner, batched FGMRES(20) to 1e-8
  200^3 heterogeneous, PML 16: the plain complex128 FFT-z path (one source)
      and the headline complex64 eigenbasis path (16 sources in lockstep)
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

TOL = 1e-8
SOL_TOL = 1e-6


def _layered(n, nsrc):
    from oracle import media
    pml = 16 if n >= 200 else 12
    return media.layered_medium(n, n, n, 10.0, pml, 2024, ppw=8.0, n_sources=nsrc)


def _oracle_solution(p, src, tol=1e-12):
    from oracle import port
    with port.PortPreconditioner(p, beta_prec=0.25, z_transform="eigen") as pre:
        pre.factor()
        op = port.PortOperator(p)
        x, its, _, rr, _ = port.fgmres(op, pre.apply, p.rhs(src), tol=tol, m=30, max_iter=3000)
    assert rr <= tol, rr
    return x


def _gpu_solver(p, precision, z_transform, restart=20):
    import helm3d
    g = helm3d.grid_mode_n(p.nx, p.ny, p.nz, p.h, p.pml, p.omega)
    o = helm3d.default_opts(precision=precision, z_transform=z_transform, restart=restart, tol=TOL, beta_prec=0.25,
                            beta_phys=p.beta_phys, max_iter=5000)
    return helm3d.Solver(g, p.s2, o)


def _relres(p, u, f):
    from oracle import port
    op = port.PortOperator(p)
    return float(np.linalg.norm(f - op(u)) / np.linalg.norm(f))


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_c1_fft_z_c128_against_oracle():
    import helm3d
    from oracle import media
    p = media.config_c1()
    f = p.rhs(0)
    s = _gpu_solver(p, helm3d.PREC_C128, helm3d.ZT_FFT)
    u = s.solve(f)
    st = s.last_stats
    s.close()
    assert st.relres <= TOL
    rr = _relres(p, u, f)
    assert rr <= TOL * (1 + 1e-6), rr
    err = _rel(u, _oracle_solution(p, 0))
    print(f"C1 64^3 FFT-z c128: {st.iterations} iterations, oracle relres {rr:.3e}, error {err:.3e}")
    assert err <= SOL_TOL, err


def test_c2_c64_eigen_two_sources_against_oracle():
    import helm3d
    p = _layered(128, 2)
    F = np.stack([p.rhs(0), p.rhs(1)])
    s = _gpu_solver(p, helm3d.PREC_C64, helm3d.ZT_PML_EIGEN)
    U = s.solve(F, nrhs=2)
    st = s.last_stats
    s.close()
    assert st.relres <= TOL
    for r in range(2):
        rr = _relres(p, U[r], F[r])
        assert rr <= TOL * (1 + 1e-6), (r, rr)
        err = _rel(U[r], _oracle_solution(p, r))
        print(f"C2 128^3 c64 eigenbasis, source {r}: oracle relres {rr:.3e}, error {err:.3e}")
        assert err <= SOL_TOL, (r, err)


def _record(kind):
    path = os.path.join(GOLDEN, f"port_{kind}_n200.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} not recorded")
    d = np.load(path)
    return {k: d[k] for k in d.files}


def _sample(u, rec):
    s = int(rec["stride"])
    return np.asarray(u)[::s, ::s, ::s]


def test_n200_fp64_plain_against_port_record():
    """The plain complex128 FFT-z path at 200^3 against the port's full solve
    of the same source with the same method: the same iteration count up to
    the Gram-Schmidt variant (DCGS2 here, CGS2 in the port), and the same
    solution."""
    import torch

    import helm3d
    fft = _record("fftz")
    eig = _record("eigen")
    p = _layered(200, 1)
    f = p.rhs(0)
    s = _gpu_solver(p, helm3d.PREC_C128, helm3d.ZT_FFT)
    fd = torch.from_numpy(f).cuda()
    u = s.solve(fd).cpu().numpy()
    st = s.last_stats
    s.close()
    its_port = int(fft["iterations"])
    assert st.relres <= TOL
    assert abs(st.iterations - its_port) <= max(10, 0.03 * its_port), (st.iterations, its_port)
    rr = _relres(p, u, f)
    assert rr <= TOL * (1 + 1e-6), rr
    e_fft = _rel(_sample(u, fft), fft["sample"])
    e_eig = _rel(_sample(u, eig), eig["sample"])
    print(f"200^3 FFT-z c128: {st.iterations} iterations (port {its_port}), oracle relres {rr:.3e}, "
          f"error vs port FFT-z solve {e_fft:.3e}, vs 1e-12 solve {e_eig:.3e}")
    assert e_fft <= SOL_TOL and e_eig <= SOL_TOL, (e_fft, e_eig)


def test_n200_c64_eigen_batched_against_oracle():
    """The headline path at 200^3: 16 sources in lockstep, complex64
    PML-eigenbasis preconditioner; source 0 against the oracle's 1e-12
    solve, every source's residual by the oracle's operator."""
    import torch

    import helm3d
    eig = _record("eigen")
    p = _layered(200, 16)
    s = _gpu_solver(p, helm3d.PREC_C64, helm3d.ZT_PML_EIGEN)
    F = torch.from_numpy(np.stack([p.rhs(r) for r in range(16)])).cuda()
    U = s.solve(F, nrhs=16)
    st = s.last_stats
    s.close()
    assert st.relres <= TOL
    Uh = U.cpu().numpy()
    Fh = F.cpu().numpy()
    del U, F
    worst = max(_relres(p, Uh[r], Fh[r]) for r in (0, 5, 15))
    assert worst <= TOL * (1 + 1e-6), worst
    err = _rel(_sample(Uh[0], eig), eig["sample"])
    print(f"200^3 c64 eigenbasis x16: {st.iterations / 16:.1f} iterations per source, oracle relres <= "
          f"{worst:.3e}, error vs 1e-12 solve {err:.3e}")
    assert err <= SOL_TOL, err
