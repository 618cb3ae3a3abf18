"""Generate the golden fixtures in this directory from the reference itself.

Runs oracle/_ref/ref_driver (the reference's own FGMRES sources compiled
against the MKL stand-in, built by ``make -C oracle``) on small grids and
stores what the reference computed:

  ref_setup_<tag>.npz   sound2D, deltaL, base 2D CSR matrix (values/ia/ja)
  ref_fgmres_<tag>.npz  f, x_sol (u = L0^{-1} w), convergence rows
                        (iteration, Res_phys, RelRes_phys, analytic error)
  ref_setup9_<tag>.npz  BCGSTAB's base 2D matrix (9-point CSR, values/ia/ja,
                        diagonal positions freqs)
  ref_bcgstab_<tag>.npz f (the RHS scaled by fscale), x_sol, convergence rows
                        (iteration, Res_phys, RelRes_phys, analytic error)
  ref_fgmres_savemem_<tag>.npz
                        the reference's FGMRES with its SAVE_MEM switch on
                        (oracle/_ref/ref_driver_savemem: kz systems with
                        kww >= 5 k2 neither factored nor solved,
                        Source/FGMRES.cpp:197-206): convergence rows, the
                        skipped modes, x_sol on every 2nd point per axis

The reference is compiled in its default configuration (HOMO, nu = 4 Hz,
c_z = 1280 m/s, LENGTH = 3200 m, REL_RES_EXIT = 1e-4).  Needs the reference
sources, so it runs in the development container only; the fixtures travel.

    python tests/golden/make_golden.py [--savemem-only]
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(REPO, "oracle", "_ref", "ref_driver")
DRIVER_SAVEMEM = os.path.join(REPO, "oracle", "_ref", "ref_driver_savemem")

# (tag, n_nopml, pml, spg, beta, niter, restart)
CASES = [
    ("n10p4s3", 10, 4, 3, 0.5, 10, 5),
    ("n11p4s3", 11, 4, 3, 0.5, 10, 5),     # odd sizes: source at (n-1)/2
    ("n16p6s4", 16, 6, 4, 0.25, 8, 4),
]
# BCGSTAB stops on an absolute residual (RES_EXIT = 1e-8); the RHS scale
# sets how many iterations it runs: (tag, n_nopml, pml, spg, beta, niter, fscale)
BCG_CASES = [
    ("n10p4s3", 10, 4, 3, 0.5, 40, 1e8),
    ("n11p4s3", 11, 4, 3, 0.5, 40, 1e8),
    ("n16p6s4", 16, 6, 4, 0.25, 16, 1e8),   # stops at the iteration cap (BiCGStab stagnates here)
]
# SAVE_MEM: nz = 58 so that some |kz| reach sqrt(5) k (modes 26..32 skipped)
SAVEMEM_CASES = [("n50p4s4", 50, 4, 4, 0.5, 10, 5)]


def run(args, cwd, driver=DRIVER):
    res = subprocess.run([driver] + [str(a) for a in args], cwd=cwd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(res.stdout[-2000:] + res.stderr[-2000:])
    return res.stdout


def savemem_cases():
    for tag, n, pml, spg, beta, niter, rest in SAVEMEM_CASES:
        with tempfile.TemporaryDirectory() as d:
            log = run(["fgmres", n, pml, spg, beta, niter, rest, d], d, DRIVER_SAVEMEM)
            solved = sorted({int(t.split()[3].rstrip(".")) for t in log.splitlines()
                             if t.startswith("Solved k = ")})
            nx = n + 2 * pml
            nz = n + 2 * spg
            skipped = np.array([k for k in range(nz) if k not in solved], dtype=np.int32)
            conv = np.loadtxt(glob.glob(os.path.join(d, "convergence_*"))[0], ndmin=2)
            x_sol = np.fromfile(os.path.join(d, "x_sol.bin"), dtype=np.complex128).reshape(nz, nx, nx)
            np.savez_compressed(
                os.path.join(HERE, f"ref_fgmres_savemem_{tag}.npz"),
                params=np.array([n, pml, spg, beta, niter, rest]),
                skipped=skipped,
                x_sol_sub=x_sol[::2, ::2, ::2],
                conv=conv,
            )
        print("wrote savemem", tag, "skipped", skipped.tolist(), file=sys.stderr)


def main():
    if not os.path.exists(DRIVER) or not os.path.exists(DRIVER_SAVEMEM):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "-j8"], check=True)
    if "--savemem-only" in sys.argv:
        savemem_cases()
        return
    for tag, n, pml, spg, beta, niter, rest in CASES:
        nx = n + 2 * pml
        nz = n + 2 * spg
        with tempfile.TemporaryDirectory() as d:
            run(["setup", n, pml, spg, beta, d], d)
            ia = np.fromfile(os.path.join(d, "csr_ia.bin"), dtype=np.int32)
            np.savez_compressed(
                os.path.join(HERE, f"ref_setup_{tag}.npz"),
                params=np.array([n, pml, spg, beta]),
                sound2D=np.fromfile(os.path.join(d, "sound2D.bin"), dtype=np.complex128).reshape(nx, nx),
                deltaL=np.fromfile(os.path.join(d, "deltaL.bin"), dtype=np.complex128).reshape(nz, nx, nx),
                csr_values=np.fromfile(os.path.join(d, "csr_values.bin"), dtype=np.complex128),
                csr_ia=ia,
                csr_ja=np.fromfile(os.path.join(d, "csr_ja.bin"), dtype=np.int32),
            )
        with tempfile.TemporaryDirectory() as d:
            run(["fgmres", n, pml, spg, beta, niter, rest, d], d)
            conv = np.loadtxt(glob.glob(os.path.join(d, "convergence_*"))[0], ndmin=2)
            np.savez_compressed(
                os.path.join(HERE, f"ref_fgmres_{tag}.npz"),
                params=np.array([n, pml, spg, beta, niter, rest]),
                f=np.fromfile(os.path.join(d, "f.bin"), dtype=np.complex128).reshape(nz, nx, nx),
                x_sol=np.fromfile(os.path.join(d, "x_sol.bin"), dtype=np.complex128).reshape(nz, nx, nx),
                conv=conv,
            )
        print("wrote", tag, file=sys.stderr)
    for tag, n, pml, spg, beta, niter, fscale in BCG_CASES:
        nx = n + 2 * pml
        nz = n + 2 * spg
        with tempfile.TemporaryDirectory() as d:
            run(["setup9", n, pml, spg, d], d)
            np.savez_compressed(
                os.path.join(HERE, f"ref_setup9_{tag}.npz"),
                params=np.array([n, pml, spg]),
                csr_values=np.fromfile(os.path.join(d, "csr9_values.bin"), dtype=np.complex128),
                csr_ia=np.fromfile(os.path.join(d, "csr9_ia.bin"), dtype=np.int32),
                csr_ja=np.fromfile(os.path.join(d, "csr9_ja.bin"), dtype=np.int32),
                freqs=np.fromfile(os.path.join(d, "csr9_freqs.bin"), dtype=np.int32),
            )
        with tempfile.TemporaryDirectory() as d:
            run(["bcgstab", n, pml, spg, beta, niter, fscale, d], d)
            conv = np.loadtxt(glob.glob(os.path.join(d, "convergence_*BCGSTAB*"))[0], ndmin=2)
            np.savez_compressed(
                os.path.join(HERE, f"ref_bcgstab_{tag}.npz"),
                params=np.array([n, pml, spg, beta, niter, fscale]),
                f=np.fromfile(os.path.join(d, "f.bin"), dtype=np.complex128).reshape(nz, nx, nx),
                x_sol=np.fromfile(os.path.join(d, "x_sol.bin"), dtype=np.complex128).reshape(nz, nx, nx),
                conv=conv,
            )
        print("wrote bcgstab", tag, file=sys.stderr)
    savemem_cases()


if __name__ == "__main__":
    main()
