"""The C-ABI library loads and exports every entry point include/helm3d.h
declares; argument validation works without a GPU.  CPU only."""
import ctypes
import os
import re

import numpy as np

from conftest import REPO


def _declared():
    hdr = open(os.path.join(REPO, "include", "helm3d.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(helm3d_[a-z_0-9]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    import helm3d
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(helm3d.lib, n), n
    assert set(helm3d.EXPORTS) <= set(names)


def test_default_opts_and_status_strings():
    import helm3d
    o = helm3d.default_opts()
    assert o.mode == helm3d.MODE_N and o.precision == helm3d.PREC_C64
    assert o.restart == 20 and abs(o.tol - 1e-8) < 1e-20
    assert helm3d.lib.helm3d_status_string(helm3d.ERR_SINGULAR).decode() == "singular block in the factor"


def test_create_rejects_bad_arguments():
    import helm3d
    g = helm3d.grid_mode_n(8, 8, 8, 10.0, 2, 10.0)
    o = helm3d.default_opts()
    h = ctypes.c_void_p()
    s2 = np.full(512, 1e-6)
    # PML wider than half the grid
    bad = helm3d.grid_mode_n(8, 8, 8, 10.0, 4, 10.0)
    assert helm3d.lib.helm3d_create(ctypes.byref(bad), s2.ctypes.data, ctypes.byref(o), ctypes.byref(h)) \
        == helm3d.ERR_ARG
    # null medium
    assert helm3d.lib.helm3d_create(ctypes.byref(g), None, ctypes.byref(o), ctypes.byref(h)) == helm3d.ERR_ARG
    o2 = helm3d.default_opts(restart=0)
    assert helm3d.lib.helm3d_create(ctypes.byref(g), s2.ctypes.data, ctypes.byref(o2), ctypes.byref(h)) \
        == helm3d.ERR_ARG


def test_create_without_gpu_reports_no_device():
    import torch
    import helm3d
    if torch.cuda.is_available():
        return
    g = helm3d.grid_mode_n(8, 8, 8, 10.0, 2, 10.0)
    o = helm3d.default_opts()
    h = ctypes.c_void_p()
    s2 = np.full(512, 1e-6)
    rc = helm3d.lib.helm3d_create(ctypes.byref(g), s2.ctypes.data, ctypes.byref(o), ctypes.byref(h))
    assert rc == helm3d.ERR_NO_DEVICE
    assert helm3d.lib.helm3d_destroy(None) == 0
