"""CPU FP64 oracle for the 3D Helmholtz solve (test infrastructure only).

This package restates, in NumPy/SciPy, the reference's FFT-z preconditioned
Krylov solve (dklyuchinskiy/Iterative-Helmholtz-solver-with-PARDISO,
``Source/FGMRES.cpp``, ``Source/functions.cpp``) and the 7-point
PML-stretched operator built on the same PML function.  It is the checker
for the CUDA path and the CPU baseline timed by ``bench.py``; the product
library never imports it.

Pinning status (what ties this restatement to the reference itself):
  * the reference's own sources, compiled here by oracle/Makefile into
    oracle/_ref/ref_driver against a stand-in for the ~20 MKL routines its
    FGMRES path calls (oracle/mkl_standin/), produced the golden fixtures
    tests/golden/ref_setup_*.npz and ref_fgmres_*.npz (made by
    tests/golden/make_golden.py): ``mode_r`` reproduces the reference's
    sound2D and dL (to 1e-15), its 2D CSR matrix (exactly), every row of its
    FGMRES residual history (to the printed digits) and its final solution
    (to 1e-11) on three grids (tests/test_oracle_pins.py);
  * the PML symmetry invariant (``Source/Tests.cpp:686-757``) and the
    inverse-traversal identity (``Source/Tests.cpp:444-684``) are checked as
    properties;
  * the histories recorded under ``HETERO/`` come from an earlier code
    version with unknown settings and are not used as pins;
  * PARDISO and MKL DFTI themselves (MKL, not vendored, version unpinned;
    ``run_one_node.sh:16`` loads intel/2017.4.196) are replaced by
    ``scipy.sparse.linalg.splu`` and ``numpy.fft``; both are exact
    solves/transforms, so they agree with the reference to rounding.

``oracle.port`` is the same arithmetic spread over every host core (the
CPU baseline); ``tests/golden/port_fftz_n200.npz`` is its full 200^3 solve.
"""
