"""The allocation-free radial-mass entry point (vls_radial_mass_noalloc).

Some callers own all device memory and cannot let a library allocate (an
application with its own pool, or a budget reserved at start-up); they pass
their own device grid and output buffers.  This test calls that entry point
through the C-ABI on a device grid held in torch memory and checks it against
vls_moments, the allocating path, on two calls in a row (the second call runs
on scratch left over from the first).  It lives in its own file so that
pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_noalloc_radial_mass_matches_vls_moments(prec):
    import torch
    from vlasolve_b200 import VlasovSolver21Spline, _lib

    _, cfg = load_golden("plummer_small")
    s = VlasovSolver21Spline(cfg, precision=prec)
    bins_ref, Mr_ref, mtot_ref = s.moments()
    R, U, J, JV = s.coords()
    dtype = torch.float64 if prec == "fp64" else torch.float32
    f_dev = torch.tensor(s.f, dtype=dtype, device="cuda").contiguous()
    L = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for call in range(2):
        bins = torch.full((s.nr,), float("nan"), dtype=torch.float64, device="cuda")
        Mr = torch.full((s.nr,), float("nan"), dtype=torch.float64, device="cuda")
        mtot = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.vls_radial_mass_noalloc(_ptr(f_dev), _lib.PRECISIONS[prec], s.nr, s.nu, s.nj,
                                       dp(R), dp(U), dp(J), dp(JV), _ptr(bins), _ptr(Mr),
                                       _ptr(mtot), ctypes.c_void_p(stream), 0)
        assert rc == 0, L.vls_noalloc_last_error().decode()
        torch.cuda.synchronize()
        scale = abs(mtot_ref)
        np.testing.assert_allclose(bins.cpu().numpy(), bins_ref, rtol=1e-12, atol=1e-15 * scale)
        np.testing.assert_allclose(Mr.cpu().numpy(), Mr_ref, rtol=1e-12, atol=1e-15 * scale)
        assert mtot.item() == pytest.approx(mtot_ref, rel=1e-13)


def test_noalloc_rejects_oversized_grid():
    import torch
    from vlasolve_b200 import _lib
    L = _lib.load()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    big = np.zeros(4096)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rc = L.vls_radial_mass_noalloc(_ptr(x), 0, 4096, 8, 1, dp(big), dp(big), dp(big), dp(big),
                                   _ptr(x), _ptr(x), _ptr(x), None, 0)
    assert rc == _lib.VLS_EINVAL
    assert b"2048" in L.vls_noalloc_last_error()
