"""CPU FP64 oracle for the 3D Helmholtz solve (test infrastructure only).

This package restates, in NumPy/SciPy, the reference's FFT-z preconditioned
Krylov solve (dklyuchinskiy/Iterative-Helmholtz-solver-with-PARDISO,
``Source/FGMRES.cpp``, ``Source/functions.cpp``) and the 7-point
PML-stretched operator built on the same PML function.  It is the checker
for the CUDA path and the CPU baseline timed by ``bench.py``; the product
library never imports it.

Pinning status (what ties this restatement to the reference itself):
  * the reference's recorded FGMRES convergence histories
    (``HETERO/0127/convergence_N49_*_FGMRES.dat``) are reproduced by
    ``mode_r`` with the reference's own settings (tests/test_oracle_pins.py);
  * the PML symmetry invariant (``Source/Tests.cpp:686-757``), the
    inverse-traversal identity (``Source/Tests.cpp:444-684``) and the block
    Schur recurrence identity (``Source/HODLR/TestsHODLR.cpp:2923-2989``)
    are checked as properties;
  * PARDISO and MKL DFTI themselves (MKL, not vendored, version unpinned;
    ``run_one_node.sh:16`` loads intel/2017.4.196) are replaced by
    ``scipy.sparse.linalg.splu`` and ``numpy.fft``; both are exact
    transforms/solves, so they agree with the reference to rounding.
"""
