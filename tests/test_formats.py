"""Result files and convergence-order tools (helm3d.formats) against the
reference's own result files (names and lines from HETERO/, committed as
tests/golden/formats_golden.json by tests/golden/make_formats_golden.py)
and against loop restatements of the reference's arithmetic on small grids."""
import json
import math
import os
import re

import numpy as np
import pytest

from helm3d import formats

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "formats_golden.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def test_convergence_file_names(golden):
    """Source/FGMRES.cpp:50: N, PML, Lx, FREQ, the sponge width (%6.lf) and beta (%5.3lf)."""
    for name in golden["convergence"]:
        m = re.match(r"convergence_N(\d+)_PML(\d+)_Lx(\d+)_FREQ(\d+)_SPG\s*(\d+)_BETA([\d.]+)_FGMRES\.dat", name)
        assert m, name
        n, pml, lx, fr, spg, beta = m.groups()
        assert formats.convergence_filename(int(n), int(pml), float(lx), float(fr), float(spg), float(beta)) == name


def test_convergence_lines_byte_exact(golden):
    """Every line of the reference's logs re-printed from its parsed values."""
    nlines = 0
    for name, lines in golden["convergence"].items():
        for line in lines:
            it, res, relres, ch = line.split()
            assert formats.convergence_line(int(it), float(res), float(relres), float(ch)) == line
            nlines += 1
    assert nlines >= 100


def test_convergence_write_read(tmp_path, golden):
    name, lines = next(iter(golden["convergence"].items()))
    rows = [(int(a), float(b), float(c), float(d)) for a, b, c, d in (l.split() for l in lines)]
    p = tmp_path / name
    formats.write_convergence(str(p), rows)
    assert p.read_text() == "".join(lines)
    back = formats.read_convergence(str(p))
    assert [r[0] for r in back] == [r[0] for r in rows]
    assert math.isinf(back[0][3])


def test_convergence_rows_from_history():
    rows = formats.convergence_rows([0.5, 0.25, 1e-9], 4.0, start=3)
    assert [r[0] for r in rows] == [3, 4, 5]
    assert rows[1][1] == 1.0 and rows[1][2] == 0.25
    assert all(math.isnan(r[3]) for r in rows)
    assert formats.convergence_line(*rows[0]) == "3 2.000000e+00 5.000000e-01 nan\n"


def test_beta_file_names_and_lines(golden):
    for name, lines in golden["beta"].items():
        m = re.match(r"beta_3D_norm2_Nx(\d+)Ny(\d+)_SPG(\d+)\.dat", name)
        assert m, name
        assert formats.beta_filename(*(int(g) for g in m.groups())) == name
        for line in lines:
            a, b = line.split()
            assert formats.beta_line(float(a), float(b)) == line


def test_sol3d_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    u = rng.standard_normal(60) + 1j * rng.standard_normal(60)
    p = tmp_path / formats.sol3d_filename(7)
    assert p.name == "sol3D_N7.dat"
    formats.write_sol3d(str(p), u)
    first = p.read_text().splitlines()[0]
    assert first == "%18.16f %18.16f" % (u[0].real, u[0].imag)
    back = formats.read_sol3d(str(p))
    assert np.max(np.abs(back - u)) < 1e-15


def _reduce_pml_loops(u, nx, ny, nz, px, py, sz):
    """reducePML3D (Source/functions.cpp:238-264) as loops over l."""
    out = []
    for l in range(nx * ny * nz):
        k, rem = divmod(l, nx * ny)
        j, i = divmod(rem, nx)
        if px <= i < nx - px and py <= j < ny - py and sz <= k < nz - sz:
            out.append(u[l])
    return np.array(out)


def test_physical_matches_reduce_pml():
    nx, ny, nz = 9, 8, 7
    u = np.arange(nx * ny * nz) * (1 + 0.5j)
    got = formats.physical(u, nx, ny, nz, 2, 1, 2)
    assert np.array_equal(got, _reduce_pml_loops(u, nx, ny, nz, 2, 1, 2))


def _inject_loops(fine, nf, nc):
    s = (nf + 1) // (nc + 1)
    out = np.zeros(nc ** 3, dtype=complex)
    for k in range(nc):
        for j in range(nc):
            for i in range(nc):
                out[i + nc * j + nc * nc * k] = fine[s * (i + 1) - 1 + nf * (s * (j + 1) - 1) + nf * nf * (s * (k + 1) - 1)]
    return out


def _smooth(n, h, e):
    c = (np.arange(n) + 1) * h
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    return (np.sin(x) * np.cos(0.7 * y) * np.exp(0.3j * z) + e * h * h).reshape(-1)


def test_runge_ratio_matches_loops():
    """Runge (Source/functions.cpp:932-1146, dim 3): injections of the finest
    solution minus the coarser ones, IntegralNorm3D (sum |v| h)."""
    n1, n2, n3 = 3, 7, 15
    L = 1.0
    h1, h2, h3 = L / (n1 + 1), L / (n2 + 1), L / (n3 + 1)
    u1, u2, u3 = _smooth(n1, h1, 0.3), _smooth(n2, h2, 0.3), _smooth(n3, h3, 0.3)
    f1, f2, ratio = formats.runge_ratio(u1, u2, u3, n1, n2, n3, h1, h2)
    g1 = sum(abs(v) for v in _inject_loops(u3, n3, n1) - u1) * h1
    g2 = sum(abs(v) for v in _inject_loops(u3, n3, n2) - u2) * h2
    assert abs(f1 - g1) <= 1e-12 * g1 and abs(f2 - g2) <= 1e-12 * g2
    assert abs(ratio - g1 / g2) <= 1e-12 * ratio


def test_shell_errors_match_loops():
    """Beta3D's shells (Source/functions.cpp:629-670, :1290-1304)."""
    n1 = 7
    n2 = 2 * (n1 + 1) - 1
    L = 1.0
    h1, h2 = L / (n1 + 1), L / (n2 + 1)
    uc, uf = _smooth(n1, h1, 0.5), _smooth(n2, h2, 0.5)
    src = (0.5, 0.5, 0.5)
    rows = formats.shell_errors(uc, uf, n1, h1, src)
    ref = _inject_loops(uf, n2, n1)
    assert [r[0] for r in rows] == [i * h1 for i in range(2, n1)]
    for i, (rad, err) in zip(range(2, n1), rows):
        num = den = 0.0
        for k in range(n1):
            for j in range(n1):
                for q in range(n1):
                    x, y, z = (q + 1) * h1 - src[0], (j + 1) * h1 - src[1], (k + 1) * h1 - src[2]
                    r = math.sqrt(x * x + y * y + z * z)
                    if 2 * h1 <= r <= i * h1:
                        l = q + n1 * j + n1 * n1 * k
                        num += abs(uc[l] - ref[l]) ** 2
                        den += abs(ref[l]) ** 2
        if den == 0:
            assert math.isnan(err) or math.isinf(err)
        else:
            assert abs(err - math.sqrt(num / den)) <= 1e-12 * max(1.0, err)
