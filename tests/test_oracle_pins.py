"""The oracle against the reference itself (golden fixtures) and against the
reference's own test properties.  CPU only."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN
from oracle import grid, mode_r

CASES = ["n10p4s3", "n11p4s3", "n16p6s4"]


def _load(kind, tag):
    return np.load(os.path.join(GOLDEN, f"ref_{kind}_{tag}.npz"))


@pytest.mark.parametrize("tag", CASES)
def test_setup_matches_reference(tag):
    """sound2D (quirk q1), deltaL and the base 5-point PML matrix
    (Source/FGMRES.cpp:79-151) equal the reference's to rounding."""
    z = _load("setup", tag)
    n, pml, spg, beta = z["params"]
    g = grid.reference_grid(int(n), int(pml), int(spg))
    st = mode_r.setup(g, beta=float(beta), media="homo", factor=False)
    assert np.abs(z["sound2D"].real - st.c2d).max() <= 1e-13 * st.c2d.max()
    assert np.abs(z["sound2D"].imag).max() == 0.0
    assert np.abs(z["deltaL"] - st.dl).max() <= 1e-12 * np.abs(st.dl).max()
    n2 = g.size2d
    A_ref = sp.csr_matrix((z["csr_values"], z["csr_ja"] - 1, z["csr_ia"] - 1), shape=(n2, n2))
    A = mode_r.assemble_2d(g, np.zeros((g.y.n, g.x.n)))
    assert abs(A_ref - A).max() <= 1e-14 * abs(A).max()


@pytest.mark.parametrize("tag", CASES)
def test_fgmres_matches_reference(tag):
    """The reference's FGMRES (q5 Arnoldi, zgels every step, exit at
    phys. rel. residual 1e-4): same residual history and same solution."""
    z = _load("fgmres", tag)
    n, pml, spg, beta, niter, rest = z["params"]
    g = grid.reference_grid(int(n), int(pml), int(spg))
    st = mode_r.setup(g, beta=float(beta), media="homo")
    f = mode_r.point_source_rhs(g)
    assert np.array_equal(f, z["f"])
    log = mode_r.fgmres_reference(st, f, m=int(niter), rest=int(rest), arnoldi="reference")
    conv = z["conv"]
    assert len(log.rows) == conv.shape[0]
    for row, ref in zip(log.rows, conv):
        assert row[1] == pytest.approx(ref[1], rel=1e-5)   # printed with %e (7 digits)
        assert row[2] == pytest.approx(ref[2], rel=1e-5)
    err = np.linalg.norm(log.u - z["x_sol"]) / np.linalg.norm(z["x_sol"])
    assert err < 1e-11


@pytest.mark.parametrize("tag", CASES)
def test_bcgstab_nine_point_matrix_is_the_five_point_one(tag):
    """BCGSTAB assembles its 2D systems with GenSparseMatrixOnline2DwithPMLand9Pts
    (Source/BcGSTAB.cpp:143, Source/functions.cpp:3532-3679).  With the
    coefficients that routine uses (a = c = 1, d = 0, Source/functions.cpp:
    3557-3559) its entries at the four diagonal neighbours are exactly zero
    (Source/functions.cpp:2497-2512) and the rest are the 5-point ones:
    the reference's 9-point CSR equals the 5-point matrix the oracle and the
    GPU factor, and its diagonal positions are where FGMRES adds the shifts."""
    z = _load("setup9", tag)
    n, pml, spg = z["params"]
    g = grid.reference_grid(int(n), int(pml), int(spg))
    n2 = g.size2d
    ia, ja, v = z["csr_ia"] - 1, z["csr_ja"] - 1, z["csr_values"]
    assert len(v) == ((g.x.n + (g.x.n - 1) * 2) * g.y.n + 2 * (n2 - g.x.n) + 4 * (g.x.n - 1) * (g.y.n - 1))
    A9 = sp.csr_matrix((v, ja, ia), shape=(n2, n2))
    z5 = _load("setup", tag)
    A5_ref = sp.csr_matrix((z5["csr_values"], z5["csr_ja"] - 1, z5["csr_ia"] - 1), shape=(n2, n2))
    assert abs(A9 - A5_ref).max() == 0.0            # bit for bit the reference's 5-point matrix
    A5 = mode_r.assemble_2d(g, np.zeros((g.y.n, g.x.n)))
    assert abs(A9 - A5).max() <= 1e-14 * abs(A5).max()
    rows = np.repeat(np.arange(n2), np.diff(ia))
    diag_nb = np.abs(np.abs(ja - rows) - g.x.n) == 1      # (i +- 1, j +- 1)
    assert diag_nb.sum() == 4 * (g.x.n - 1) * (g.y.n - 1) and np.all(v[diag_nb] == 0)
    assert np.array_equal(ja[z["freqs"]], np.arange(n2))


@pytest.mark.parametrize("tag", CASES)
def test_bcgstab_matches_reference(tag):
    """The reference's BCGSTAB (shadow residual 2 r0, iterate kept in u-space,
    true residual through L0 u and K, exit on the absolute physical residual
    1e-8): the same residual history and the same solution, on the RHS
    scaled as the fixture was made (the scale sets the iteration count)."""
    z = _load("bcgstab", tag)
    n, pml, spg, beta, niter, fscale = z["params"]
    g = grid.reference_grid(int(n), int(pml), int(spg))
    st = mode_r.setup(g, beta=float(beta), media="homo")
    f = mode_r.point_source_rhs(g) * fscale
    assert np.array_equal(f, z["f"])
    x, rows = mode_r.bicgstab_reference(st, f, m=int(niter))
    conv = z["conv"]
    assert len(rows) == conv.shape[0] and len(rows) >= 5
    for row, ref in zip(rows, conv):
        assert row[1] == pytest.approx(ref[1], rel=1e-5)   # printed with %e (7 digits)
        assert row[2] == pytest.approx(ref[2], rel=1e-5)
    # the HOMO build zeroes the source cross of its solution (Source/BcGSTAB.cpp:532)
    x = mode_r.nullify_source_cross(g, x)
    err = np.linalg.norm(x - z["x_sol"]) / np.linalg.norm(z["x_sol"])
    # n16p6s4 stops at its 16-iteration cap while BiCGStab stagnates, where
    # rounding differences grow from step to step
    assert err < (1e-11 if conv[-1, 1] < 1e-8 else 1e-8), err


def test_pml_symmetry_invariant():
    """A_2D / (alpha_x alpha_y) is symmetric (Source/Tests.cpp:686-757)."""
    g = grid.reference_grid(12, 5, 3)
    A = mode_r.assemble_2d(g, np.zeros((g.y.n, g.x.n))).tocsr()
    ax = np.array([grid.alpha(g.x, float(i), g.omega) for i in range(g.x.n)])
    ay = np.array([grid.alpha(g.y, float(j), g.omega) for j in range(g.y.n)])
    scale = (ay[:, None] * ax[None, :]).ravel()
    S = sp.diags(1.0 / scale) @ A
    assert abs(S - S.T).max() <= 1e-12 * abs(S).max()


def test_inverse_traversal_identity():
    """A_R (L0^{-1} g) = g - dL L0^{-1} g, i.e. K = A_R L0^{-1}
    (Source/Tests.cpp:444-684)."""
    g = grid.reference_grid(10, 4, 3)
    st = mode_r.setup(g, beta=0.5, media="homo")
    rng = np.random.default_rng(1)
    v = rng.standard_normal(g.shape_zyx) + 1j * rng.standard_normal(g.shape_zyx)
    lhs = st.apply_a(st.l0_solve(v))
    rhs = st.apply_k(v)
    assert np.linalg.norm(lhs - rhs) <= 1e-11 * np.linalg.norm(rhs)


def test_fgmres_savemem_matches_reference():
    """The reference built with SAVE_MEM (Source/FGMRES.cpp:197-206: modes
    with kww >= 5 k2 neither factored nor solved, their solution set to
    zero): the oracle's skip rule picks the same modes, and its FGMRES gives
    the same residual history and solution (every 2nd point per axis)."""
    z = np.load(os.path.join(GOLDEN, "ref_fgmres_savemem_n50p4s4.npz"))
    n, pml, spg, beta, niter, rest = z["params"]
    g = grid.reference_grid(int(n), int(pml), int(spg))
    st = mode_r.setup(g, beta=float(beta), media="homo", kz_skip_ratio=5.0)
    assert np.flatnonzero(st.skip).tolist() == z["skipped"].tolist()
    f = mode_r.point_source_rhs(g)
    log = mode_r.fgmres_reference(st, f, m=int(niter), rest=int(rest), arnoldi="reference")
    conv = z["conv"]
    assert len(log.rows) == conv.shape[0]
    for row, ref in zip(log.rows, conv):
        assert row[1] == pytest.approx(ref[1], rel=1e-5)
        assert row[2] == pytest.approx(ref[2], rel=1e-5)
    sub = log.u[::2, ::2, ::2]
    err = np.linalg.norm(sub - z["x_sol_sub"]) / np.linalg.norm(z["x_sol_sub"])
    assert err < 1e-11
