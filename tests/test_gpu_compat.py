"""The reference-shaped FGMRES and BCGSTAB (include/helm3d_compat.h) called
from C++ the way the reference's main calls them, against the reference's
own output (tests/golden, made by the reference's sources compiled here)."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, PKG_DIR, REPO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = tmp_path_factory.mktemp("compat") / "compat_main"
    libdir = os.path.join(PKG_DIR, "helm3d")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "compat_main.cpp"), "-L", libdir, "-lhelm3d",
                    f"-Wl,-rpath,{libdir}", "-o", str(out)], check=True)
    return str(out)


@pytest.mark.parametrize("tag", ["n10p4s3", "n11p4s3"])
def test_compat_fgmres_against_reference(driver, tag):
    z = np.load(os.path.join(GOLDEN, f"ref_fgmres_{tag}.npz"))
    n, pml, spg, beta, niter, rest = z["params"]
    with tempfile.TemporaryDirectory() as d:
        z["f"].astype(np.complex128).tofile(os.path.join(d, "f.bin"))
        r = subprocess.run([driver, "fgmres", str(int(n)), str(int(pml)), str(int(spg)), str(float(beta)),
                            str(int(niter)), str(int(rest)), d], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        u = np.fromfile(os.path.join(d, "x_sol.bin"), dtype=np.complex128).reshape(z["x_sol"].shape)
    # both stop near a relative residual of 1e-4 (the reference on the
    # physical domain, the shim on the whole grid)
    err = np.linalg.norm(u - z["x_sol"]) / np.linalg.norm(z["x_sol"])
    assert err < 5e-3, err


@pytest.mark.parametrize("tag", ["n10p4s3", "n11p4s3", "n16p6s4"])
def test_compat_bcgstab_against_reference(driver, tag):
    """BCGSTAB with the reference's prototype: the same iteration count
    (exit on the absolute physical residual 1e-8, or the cap), the same
    final physical-domain residual and the same solution, source cross
    zeroed as the reference's HOMO build does."""
    z = np.load(os.path.join(GOLDEN, f"ref_bcgstab_{tag}.npz"))
    n, pml, spg, beta, niter, fscale = z["params"]
    conv = z["conv"]
    with tempfile.TemporaryDirectory() as d:
        z["f"].astype(np.complex128).tofile(os.path.join(d, "f.bin"))
        r = subprocess.run([driver, "bcgstab", str(int(n)), str(int(pml)), str(int(spg)), str(float(beta)),
                            str(int(niter)), d], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        u = np.fromfile(os.path.join(d, "x_sol.bin"), dtype=np.complex128).reshape(z["x_sol"].shape)
    m = re.search(r"helm3d BCGSTAB: (\d+) iterations, relative residual (\S+) \(physical domain (\S+)\)", r.stdout)
    assert m, r.stdout
    assert int(m.group(1)) == conv.shape[0]
    # the final physical-domain residual (the reference's RelRes column)
    assert float(m.group(3)) == pytest.approx(conv[-1, 2], rel=1e-4 if conv[-1, 1] < 1e-8 else 1e-2)
    err = np.linalg.norm(u - z["x_sol"]) / np.linalg.norm(z["x_sol"])
    assert err < (1e-9 if conv[-1, 1] < 1e-8 else 1e-6), err
