"""Builders shared by the tests: oracle problems -> helm3d solvers."""
import numpy as np

from oracle import grid as ogrid
from oracle import media, mode_n, mode_r


def mode_r_case(n_nopml, pml, spg, beta=0.5, media_kind="homo"):
    """Reference (mode R) grid + oracle state, HOMO by default as the
    reference's default build."""
    g = ogrid.reference_grid(n_nopml, pml, spg)
    st = mode_r.setup(g, beta=beta, media=media_kind)
    return g, st


def mode_r_solver(g, st, beta=0.5, media_kind="homo", **kw):
    import helm3d
    G = helm3d.grid_mode_r(g.x.n, g.y.n, g.z.n, g.x.h, g.z.h, g.x.pml_pts, g.z.spg_pts, g.z.l, g.omega)
    s2 = 1.0 / (st.c3d ** 2)
    o = helm3d.default_opts(mode=helm3d.MODE_R, precision=helm3d.PREC_C128, kz_symbol=helm3d.KZ_REFERENCE,
                            beta_prec=beta, quirk_q1=1, restart=30, max_iter=600, tol=1e-11)
    if media_kind == "homo":
        o.s2_l0 = 1.0 / (mode_r.C_Z ** 2)
    for k, v in kw.items():
        setattr(o, k, v)
    return helm3d.Solver(G, s2, o)


def mode_n_solver(p, precision=1, beta_prec=0.25, kz_symbol=0, **kw):
    import helm3d
    G = helm3d.grid_mode_n(p.nx, p.ny, p.nz, p.h, p.pml, p.omega)
    o = helm3d.default_opts(mode=helm3d.MODE_N, precision=precision, kz_symbol=kz_symbol, beta_prec=beta_prec,
                            beta_phys=p.beta_phys, restart=20, max_iter=3000, tol=1e-10)
    for k, v in kw.items():
        setattr(o, k, v)
    return helm3d.Solver(G, p.s2, o)


def small_problem(nx, ny, nz, pml=4, seed=11, ppw=8.0):
    """A small heterogeneous mode N problem of arbitrary (uneven) size."""
    p = media.layered_medium(nx, ny, nz, 10.0, pml, seed, ppw=ppw, amp=0.2)
    return p


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def rand_c(shape, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
