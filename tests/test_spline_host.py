"""Host-side pieces of the spline-level surface that need no GPU:
interpolSpline::createInit (interpol_spline.hxx:49-91) through the C-ABI,
against a numpy restatement of its grid (genScale, the last node moved 1e-10
of a cell outwards, the ends rescaled)."""
import ctypes

import numpy as np
import pytest

from vlasolve_b200 import _lib


def _init(**kw):
    L = _lib.load()
    ini = _lib.InterpInit()
    a = dict(xstart=0.01, xstop=25.0, Nx=40, ystart=-2.0, ystop=2.0, Ny=32, xbctL=4, xbctR=4,
             ybctL=4, ybctR=4, xscaleType=1, yscaleType=0, vltype=1, useLog=0, xbcvL=0.0,
             xbcvR=0.0, ybcvL=0.0, ybcvR=0.0)
    a.update(kw)
    rc = L.vls_interp_create_init(*a.values(), ctypes.byref(ini))
    return rc, ini


def test_create_init_grid_and_nudge():
    rc, ini = _init()
    assert rc == 0
    assert (ini.nx, ini.ny) == (41, 33)
    assert ini.rescaleNeeded == 1 and ini.useLog == 0
    R = np.exp(np.linspace(np.log(0.01), np.log(25.0), 41))
    assert ini.xstart == pytest.approx(np.log(0.01), abs=1e-14)
    assert ini.xend == pytest.approx(np.log(25.0 + (25.0 - R[-2]) * 1e-10), abs=1e-14)
    assert ini.xend > np.log(25.0)
    U = np.linspace(-2.0, 2.0, 33)
    assert ini.ystart == -2.0
    assert ini.yend == pytest.approx(2.0 + (U[-1] - U[-2]) * 1e-10, abs=1e-15)
    assert list(ini.xbc) == [4, 4] and list(ini.ybc) == [4, 4]


def test_create_init_linear_grids_need_no_rescale():
    rc, ini = _init(xscaleType=0, xstart=0.0, xstop=1.0, Nx=8)
    assert rc == 0 and ini.rescaleNeeded == 0 and ini.nx == 9
    assert ini.xend == pytest.approx(1.0 + 0.125e-10, abs=1e-16)


def test_create_init_rejects_unknown_scale():
    rc, _ = _init(xscaleType=7)
    assert rc == _lib.VLS_EINVAL
    assert b"scale" in _lib.load().vls_interp_last_error(None)
