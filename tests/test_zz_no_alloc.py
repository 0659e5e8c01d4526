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


def _moments_numpy(f, R, U, J, JV):
    """Radial bins and enclosed mass of an FP64 grid [j][u][r], restated in
    numpy: bins[r] = dR[r]/4 (T[r] + T[r+1]) with T[r] = sum_j w_j sum_u b_u
    f[j][u][r] (quadrature21.hxx:111-119), Mr the exclusive prefix sum
    (grid_handler.hxx:387-407)."""
    nr, nu, nj = len(R), len(U), len(J)
    dR = np.append(np.diff(R), 0.0)
    dU = np.append(np.diff(U), 0.0)
    bu = dU + np.concatenate([[0.0], dU[:-1]])
    dJ = np.where(np.arange(nj) >= nu - 1, 0.0, np.diff(JV))
    wj = 8 * np.pi * np.pi * J * dJ
    T = np.einsum("j,u,jur->r", wj, bu, f)
    bins = np.zeros(nr)
    bins[:-1] = dR[:-1] * 0.25 * (T[:-1] + T[1:])
    Mr = np.concatenate([[0.0], np.cumsum(bins)[:-1]])
    return bins, Mr, bins.sum()


def test_noalloc_largest_r_extent_two_calls():
    """N_r at the scratch limit (2048 r vertices: two r per thread in the scan,
    64 r strips), 37 J cells (several slices per slice group) and a seeded
    random FP64 grid, against a numpy restatement of the moment, on two calls
    in a row."""
    import torch
    from vlasolve_b200 import _lib

    nr, nu, nj = 2048, 40, 37
    rng = np.random.default_rng(20261203)
    R = np.exp(np.linspace(np.log(0.01), np.log(25.0), nr))
    U = np.linspace(-2.0, 2.0, nu)
    JV = np.linspace(0.0, 1.6, nj + 1) ** 2 / 1.6
    J = 0.5 * (JV[:-1] + JV[1:])
    f = rng.random((nj, nu, nr))
    bins_ref, Mr_ref, mtot_ref = _moments_numpy(f, R, U, J, JV)
    f_dev = torch.tensor(f, dtype=torch.float64, device="cuda").contiguous()
    L = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    dp = lambda a: np.ascontiguousarray(a).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    keep = [np.ascontiguousarray(a) for a in (R, U, J, JV)]
    for call in range(2):
        bins = torch.full((nr,), float("nan"), dtype=torch.float64, device="cuda")
        Mr = torch.full((nr,), float("nan"), dtype=torch.float64, device="cuda")
        mtot = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.vls_radial_mass_noalloc(_ptr(f_dev), _lib.PRECISIONS["fp64"], nr, nu, nj,
                                       *[dp(a) for a in keep], _ptr(bins), _ptr(Mr),
                                       _ptr(mtot), ctypes.c_void_p(stream), 0)
        assert rc == 0, L.vls_noalloc_last_error().decode()
        torch.cuda.synchronize()
        scale = abs(mtot_ref)
        np.testing.assert_allclose(bins.cpu().numpy(), bins_ref, rtol=1e-12, atol=1e-15 * scale)
        np.testing.assert_allclose(Mr.cpu().numpy(), Mr_ref, rtol=1e-12, atol=1e-15 * scale)
        assert mtot.item() == pytest.approx(mtot_ref, rel=1e-12)


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
