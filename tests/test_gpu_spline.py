"""The spline-level surface (LocalSpline2 = localSpline<2>, InterpolSpline =
interpolSpline) through the C-ABI against the oracle's restatement of the
reference's prefilter (create_2D, localSpline.hxx:1238-1258) and gathers
(evaluateC :381-398, evaluateNxPy :423-441).

Tolerances: FP64 coefficients and values 1e-12 of their largest magnitude (the
GPU solves the same systems in another operation order); FP32 storage 1e-6;
integer decompositions (pos2Coord) bit-exact."""
import numpy as np
import pytest

from oracle import vls_oracle as vo

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-6


def smooth_slices(ns, dim0, dim1, seed=20261203):
    """Seeded smooth data [slice][dim1][dim0] with a little noise."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, 1.0, dim0)
    y = np.linspace(-1.0, 1.0, dim1)
    out = np.empty((ns, dim1, dim0))
    for s in range(ns):
        a, b = rng.uniform(1, 4, 2)
        out[s] = (np.exp(-a * x[None, :]) * np.cos(b * y[:, None]) + 0.3
                  + 1e-3 * rng.standard_normal((dim1, dim0)))
    return out


def make(dim0, dim1, ns=3, precision="fp64", scale0="logarithmic"):
    from vlasolve_b200.spline import LocalSpline2
    sp = LocalSpline2(start=(0.01, -2.0), stop=(25.0, 2.0), N=(dim0 - 1, dim1 - 1),
                      scale=(scale0, "linear"), nslices=ns, precision=precision)
    assert sp.dim == (dim0, dim1)
    data = smooth_slices(ns, dim0, dim1)
    sp.assign(data)
    sp.build()
    coefs = [vo.prefilter2d(data[s], sp.step_inv[0], sp.step_inv[1]) for s in range(ns)]
    return sp, data, coefs


# (dim0, dim1): register chunks in both directions; a single-chunk u line;
# r lines of 2048 values (beyond the register layouts: shared-memory
# segments)
SHAPES = [(41, 33), (200, 150), (33, 8), (2048, 40)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "%dx%d" % s)
def test_coefficients_match_oracle(shape):
    sp, data, coefs = make(*shape)
    for s in range(sp.nslices):
        c = sp.coefficients(s)
        ref = coefs[s]
        assert c.shape == ref.shape
        assert np.abs(c - ref).max() <= FP64_TOL * np.abs(ref).max(), s


@pytest.mark.parametrize("shape", SHAPES[:3], ids=lambda s: "%dx%d" % s)
def test_evaluate_c_and_nxpy_match_oracle(shape):
    sp, data, coefs = make(*shape)
    dim0, dim1 = shape
    rng = np.random.default_rng(7)
    n = 2000
    sl = rng.integers(0, sp.nslices, n)
    Nx = rng.integers(0, dim0 - 1, n).astype(np.int32)
    Ny = rng.integers(0, dim1 - 1, n).astype(np.int32)
    x, y = rng.random(n), rng.random(n)
    v = sp.evaluateC(Nx, x, Ny, y, slices=sl)
    ref = np.concatenate([vo.evaluate_c(coefs[s], Nx[sl == s], x[sl == s], Ny[sl == s],
                                        y[sl == s]) for s in range(sp.nslices)])
    got = np.concatenate([v[sl == s] for s in range(sp.nslices)])
    assert np.abs(got - ref).max() <= FP64_TOL * np.abs(ref).max()
    # evaluateNxPy: node Nx along dim0, a position along dim1 (linear scale)
    yy = rng.uniform(-2.0, 2.0 - 1e-9, n)
    v = sp.evaluateNxPy(Nx, yy, slices=sl)
    NyP, yP = sp.pos2Coord(yy, 1)
    ipart = np.floor((yy - sp.start[1]) * sp.step_inv[1])
    np.testing.assert_array_equal(NyP, ipart.astype(np.int32))
    ref = np.concatenate([vo.evaluate_nxpy(coefs[s], Nx[sl == s], NyP[sl == s], yP[sl == s])
                          for s in range(sp.nslices)])
    got = np.concatenate([v[sl == s] for s in range(sp.nslices)])
    assert np.abs(got - ref).max() <= FP64_TOL * np.abs(ref).max()
    # the nodes themselves are interpolated: evaluateNxPy at the data rows
    rows = rng.integers(0, dim1 - 1, 200)
    cols = rng.integers(0, dim0, 200).astype(np.int32)
    U = np.linspace(-2.0, 2.0, dim1)
    v = sp.evaluateNxPy(cols, U[rows], slices=0)
    np.testing.assert_allclose(v, data[0, rows, cols], rtol=1e-11, atol=1e-13)


def test_evaluate_positions_on_a_log_scale():
    """evaluate(x, y): pos2Coord on the log-scaled dim0 and the linear dim1,
    then the gather; at the vertices it returns the data."""
    sp, data, coefs = make(41, 33, ns=1)
    rng = np.random.default_rng(11)
    xx = np.exp(rng.uniform(np.log(0.01), np.log(25.0) - 1e-9, 500))
    yy = rng.uniform(-2.0, 2.0 - 1e-9, 500)
    v = sp.evaluate(xx, yy)
    Nx, fx = sp.pos2Coord(xx, 0)
    Ny, fy = sp.pos2Coord(yy, 1)
    assert np.all((Nx >= 0) & (Nx < 40) & (Ny >= 0) & (Ny < 32))
    ref = vo.evaluate_c(coefs[0], Nx, fx, Ny, fy)
    assert np.abs(v - ref).max() <= FP64_TOL * np.abs(ref).max()
    R = np.exp(np.linspace(np.log(0.01), np.log(25.0), 41))
    U = np.linspace(-2.0, 2.0, 33)
    ii, jj = rng.integers(0, 40, 100), rng.integers(0, 32, 100)
    np.testing.assert_allclose(sp.evaluate(R[ii], U[jj]), data[0, jj, ii], rtol=1e-9)


def test_fp32_storage():
    sp, data, coefs = make(200, 150, precision="fp32")
    for s in range(sp.nslices):
        assert np.abs(sp.coefficients(s) - coefs[s]).max() <= FP32_TOL * np.abs(coefs[s]).max()
    rng = np.random.default_rng(3)
    Nx = rng.integers(0, 199, 300).astype(np.int32)
    Ny = rng.integers(0, 149, 300).astype(np.int32)
    x, y = rng.random(300), rng.random(300)
    v = sp.evaluateC(Nx, x, Ny, y, slices=1)
    ref = vo.evaluate_c(coefs[1], Nx, x, Ny, y)
    assert np.abs(v - ref).max() <= FP32_TOL * np.abs(ref).max()


def test_spline_errors():
    from vlasolve_b200 import _lib
    from vlasolve_b200.spline import LocalSpline2
    with pytest.raises(_lib.VlsError) as e:
        LocalSpline2((0, 0), (1, 1), (10, 10), bc=("flat", "natural"))
    assert e.value.code == _lib.VLS_EINVAL
    sp = LocalSpline2((0, 0), (1, 1), (10, 10))
    with pytest.raises(_lib.VlsError) as e:
        sp.evaluateC([0], [0.5], [0], [0.5])
    assert e.value.code == _lib.VLS_ESTATE
    sp.assign(np.ones((11, 11)))
    sp.build()
    with pytest.raises(_lib.VlsError) as e:
        sp.evaluateC([11], [0.5], [0], [0.5])  # outside the nodes
    assert e.value.code == _lib.VLS_EINVAL
    # a constant is reproduced everywhere (the weights sum to 36)
    np.testing.assert_allclose(sp.evaluate(np.linspace(0, 0.999, 50), np.linspace(0, 0.999, 50)),
                               1.0, rtol=1e-14)


def _interp_case(useLog=False):
    from vlasolve_b200.spline import InterpolSpline
    ini = InterpolSpline.createInit(0.01, 25.0, 40, -2.0, 2.0, 32, xscaleType="logarithmic",
                                    useLog=useLog)
    data = smooth_slices(1, 41, 33)[0]
    if useLog:
        data = np.exp(data)  # positive values for the log-valued spline
    return ini, data, InterpolSpline.create(ini, data)


def _interp_ref(ini, coef, x, y):
    """The reference's evaluation restated: rescale, clamp, decompose on the
    nudged uniform grid, evaluateC on the natural-BC coefficients."""
    px = np.clip(np.log(x), ini.xstart, ini.xend)
    py = np.clip(y, ini.ystart, ini.yend)
    ux = (px - ini.xstart) * ((ini.nx - 1) / (ini.xend - ini.xstart))
    uy = (py - ini.ystart) * ((ini.ny - 1) / (ini.yend - ini.ystart))
    Ix, Iy = np.floor(ux), np.floor(uy)
    return vo.evaluate_c(coef, Ix.astype(int), ux - Ix, Iy.astype(int), uy - Iy)


def test_interpol_spline_init_and_values():
    ini, data, sp = _interp_case()
    assert (ini.nx, ini.ny) == (41, 33) and ini.rescaleNeeded == 1 and ini.useLog == 0
    R = np.exp(np.linspace(np.log(0.01), np.log(25.0), 41))
    assert abs(ini.xstart - np.log(R[0])) < 1e-14
    # the last node sits 1e-10 of a cell past the data's (interpol_spline.hxx:62)
    assert abs(ini.xend - np.log(25.0 + (25.0 - R[-2]) * 1e-10)) < 1e-14
    assert ini.xend > np.log(25.0)
    coef = vo.prefilter2d(data, 1.0, 1.0)  # natural ends: the spacing cancels
    rng = np.random.default_rng(5)
    x = np.exp(rng.uniform(np.log(0.01), np.log(25.0), 400))
    y = rng.uniform(-2.0, 2.0, 400)
    v = sp.evaluate(x, y)
    ref = _interp_ref(ini, coef, x, y)
    assert np.abs(v - ref).max() <= 1e-11 * np.abs(ref).max()
    # points outside the grid are clamped to it
    vo_ = sp.evaluate(np.array([1e-4, 1e3]), np.array([-5.0, 5.0]))
    np.testing.assert_allclose(vo_, sp.evaluate(np.array([0.01, np.exp(ini.xend)]),
                                                np.array([-2.0, ini.yend])), rtol=1e-13)


def test_interpol_spline_derivatives():
    """Gradient (d/dy, d/dx) and Hessian (yy, yx, xy, xx) in rescaled
    coordinates against central differences of the values."""
    ini, data, sp = _interp_case()
    rng = np.random.default_rng(9)
    lx = rng.uniform(np.log(0.02), np.log(20.0), 100)
    y = rng.uniform(-1.8, 1.8, 100)
    v, g, h = sp.evaluate(np.exp(lx), y, hess=True)
    e = 1e-5
    dvx = (sp.evaluate(np.exp(lx + e), y) - sp.evaluate(np.exp(lx - e), y)) / (2 * e)
    dvy = (sp.evaluate(np.exp(lx), y + e) - sp.evaluate(np.exp(lx), y - e)) / (2 * e)
    scale = np.abs(g).max()
    assert np.abs(g[:, 1] - dvx).max() <= 1e-6 * scale
    assert np.abs(g[:, 0] - dvy).max() <= 1e-6 * scale
    _, gxp = sp.evaluate(np.exp(lx + e), y, grad=True)
    _, gxm = sp.evaluate(np.exp(lx - e), y, grad=True)
    _, gyp = sp.evaluate(np.exp(lx), y + e, grad=True)
    _, gym = sp.evaluate(np.exp(lx), y - e, grad=True)
    hs = np.abs(h).max()
    assert np.abs(h[:, 3] - (gxp[:, 1] - gxm[:, 1]) / (2 * e)).max() <= 1e-5 * hs
    assert np.abs(h[:, 0] - (gyp[:, 0] - gym[:, 0]) / (2 * e)).max() <= 1e-5 * hs
    assert np.abs(h[:, 1] - (gxp[:, 0] - gxm[:, 0]) / (2 * e)).max() <= 1e-5 * hs
    np.testing.assert_array_equal(h[:, 1], h[:, 2])


def test_interpol_spline_log_values_and_errors():
    from vlasolve_b200 import _lib
    from vlasolve_b200.spline import InterpolSpline
    ini, data, sp = _interp_case(useLog=True)
    coef = vo.prefilter2d(np.log(data), 1.0, 1.0)
    rng = np.random.default_rng(13)
    x = np.exp(rng.uniform(np.log(0.01), np.log(25.0), 200))
    y = rng.uniform(-2.0, 2.0, 200)
    v, g = sp.evaluate(x, y, grad=True)
    ref = np.exp(_interp_ref(ini, coef, x, y))
    assert np.all(np.isfinite(ref)) and np.all(ref > 0)
    np.testing.assert_allclose(v, ref, rtol=1e-11)
    # the gradient of a log-valued spline is -g v with g that of the spline
    # of the logarithms (interpol_spline.hxx:151-152, the reference's formula)
    ini2 = InterpolSpline.createInit(0.01, 25.0, 40, -2.0, 2.0, 32, xscaleType="logarithmic")
    _, gl = InterpolSpline.create(ini2, np.log(data)).evaluate(x, y, grad=True)
    np.testing.assert_allclose(g, -gl * v[:, None], rtol=1e-10, atol=1e-14)
    with pytest.raises(_lib.VlsError) as e:
        sp.evaluate(x, y, hess=True)
    assert e.value.code == _lib.VLS_EINVAL
    bad = InterpolSpline.createInit(0.0, 1.0, 8, 0.0, 1.0, 8, xbctL="flat")
    with pytest.raises(_lib.VlsError) as e:
        InterpolSpline.create(bad, np.ones(81))
    assert e.value.code == _lib.VLS_EINVAL
