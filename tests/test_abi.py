"""The C-ABI library builds for sm_100a, loads without a GPU, and exports
every entry point include/vlasolve_b200.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "vlasolve_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vls_[a-z0-9_]+)\s*\(", text)))


def test_header_parses():
    names = header_functions()
    assert "vls_create" in names and "vls_step" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from vlasolve_b200 import _lib
    from vlasolve_b200.build import build
    build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding declares exactly the header's entry points
    assert sorted(set(_lib.EXPORTED)) == header_functions()


def test_library_is_sm100a_only():
    from vlasolve_b200.build import ARCH
    assert ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_create_without_gpu_fails_loudly():
    """Without a usable sm_100 device the library reports VLS_ECUDA instead of
    falling back to any CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from vlasolve_b200 import _lib
    L = _lib.load()
    assert L.vls_device_ok(0) == _lib.VLS_ECUDA
    g, s = _lib.GridDesc(), _lib.SolverDesc()
    g.Pmin, g.Pmax, g.Pres, g.Pscale = 0.01, 25, 16, 1
    g.Umin[0], g.Umin[1], g.Umax[0], g.Umax[1] = -2, 0, 2, 1.6
    g.Ures[0], g.Ures[1], g.Uscale[0], g.Uscale[1] = 16, 8, 0, 2
    s.G, s.dt = 1.0, 0.005
    h = ctypes.c_void_p()
    rc = L.vls_create(ctypes.byref(g), ctypes.byref(s), ctypes.byref(h))
    assert rc == _lib.VLS_ECUDA
    assert b"CUDA" in L.vls_last_error(None) or b"device" in L.vls_last_error(None)


def _driver():
    from vlasolve_b200.build import DRIVER, build
    build()
    return DRIVER


def test_driver_rejects_bad_options(tmp_path):
    """The command-line driver parses the reference's -group.param options and
    parameter files before touching the GPU."""
    import subprocess
    d = _driver()
    r = subprocess.run([d, "-solver.kernelType", "foo"], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 1 and "invalid kernel type" in r.stderr
    r = subprocess.run([d, "missing.ini"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "could not read parameter file" in r.stderr
    r = subprocess.run([d, "-init.type", "King"], cwd=tmp_path, capture_output=True,
                       text=True)
    assert r.returncode == 1 and "unknown initial conditions" in r.stderr


def test_driver_without_gpu_fails_loudly(tmp_path):
    import subprocess
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    (tmp_path / "p.ini").write_text("init.type Plummer\ngrid.Pres 16\n")
    r = subprocess.run([_driver(), "p.ini"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 2 and "device" in r.stderr
