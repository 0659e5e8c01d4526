"""Python mirror of the reference's spline classes, backed by the CUDA library.

LocalSpline2 follows localSpline<2, double> (localSpline.hxx:60-503): init,
assign, build, evaluateC, evaluateNxPy, evaluate, pos2Coord, over a batch of
slices resident on the GPU; every evaluation takes arrays of points.
InterpolSpline follows interpolSpline (interpol_spline.hxx:49-189):
createInit, create, evaluate (value, gradient, Hessian), destroy.  Only the
natural boundary condition is built (VLS_EINVAL otherwise).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_P = ctypes.POINTER


def _d(a):
    return a.ctypes.data_as(_P(ctypes.c_double))


def _i32(a):
    return a.ctypes.data_as(_P(ctypes.c_int32))


def _i64(a):
    return a.ctypes.data_as(_P(ctypes.c_int64))


class LocalSpline2:
    """nslices 2D cubic B-splines on one device (localSpline<2>).

    start, stop, N, scale ("linear", "logarithmic", "quadratic"), vertex
    (True: values at vertices) per dimension, dimension 0 fastest in the data;
    precision "fp64" or "fp32" (FP32 storage, FP64 solves)."""

    def __init__(self, start, stop, N, scale=("linear", "linear"), vertex=(True, True),
                 nslices: int = 1, precision: str = "fp64", device: int = 0,
                 bc=("natural", "natural")):
        L = _lib.load()
        self._L = L
        d = _lib.Spline2dDesc()
        for k in range(2):
            d.start[k], d.stop[k], d.N[k] = float(start[k]), float(stop[k]), int(N[k])
            d.scaleType[k] = _lib.SCALES[scale[k]]
            d.vlType[k] = 1 if vertex[k] else 0
            d.bCond[k][0] = d.bCond[k][1] = _lib.BC[bc[k]]
        d.precision = _lib.PRECISIONS[precision]
        d.device = device
        h = ctypes.c_void_p()
        rc = L.vls_spline2d_create(ctypes.byref(d), int(nslices), ctypes.byref(h))
        if rc != 0:
            raise _lib.VlsError(rc, L.vls_spline2d_last_error(None).decode())
        self._h = h
        d0, d1, ns = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        L.vls_spline2d_dims(h, ctypes.byref(d0), ctypes.byref(d1), ctypes.byref(ns))
        self.dim = (d0.value, d1.value)
        self.nslices = ns.value
        st, hi = np.empty(2), np.empty(2)
        L.vls_spline2d_scale(h, _d(st), _d(hi))
        self.start, self.step_inv = st, hi

    def close(self):
        if getattr(self, "_h", None):
            self._L.vls_spline2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != 0:
            raise _lib.VlsError(rc, self._L.vls_spline2d_last_error(self._h).decode())

    def assign(self, data):
        """Values [slice][dim1][dim0] (or [dim1][dim0] for one slice)."""
        v = np.ascontiguousarray(data, dtype=np.float64)
        if v.size != self.nslices * self.dim[0] * self.dim[1]:
            raise ValueError("assign: size mismatch")
        self._ck(self._L.vls_spline2d_assign(self._h, _d(v), self.nslices))

    def build(self):
        self._ck(self._L.vls_spline2d_build(self._h))

    def coefficients(self, slice_: int = 0) -> np.ndarray:
        """Padded coefficients (dim1 + 2, dim0 + 2) of one slice."""
        out = np.empty((self.dim[1] + 2, self.dim[0] + 2))
        self._ck(self._L.vls_spline2d_coefficients(self._h, int(slice_), _d(out)))
        return out

    def pos2Coord(self, p, dir_: int):
        p = np.ascontiguousarray(p, dtype=np.float64).ravel()
        I, F = np.empty(p.size, np.int32), np.empty(p.size)
        self._ck(self._L.vls_spline2d_pos2coord(self._h, int(dir_), p.size, _d(p), _i32(I),
                                                _d(F)))
        return I, F

    @staticmethod
    def _sl(slices, n):
        if slices is None:
            return None
        s = np.ascontiguousarray(np.broadcast_to(slices, (n,)), dtype=np.int64)
        return s

    def evaluateC(self, Nx, x, Ny, y, slices=None):
        Nx = np.ascontiguousarray(Nx, dtype=np.int32).ravel()
        Ny = np.ascontiguousarray(Ny, dtype=np.int32).ravel()
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = np.ascontiguousarray(y, dtype=np.float64).ravel()
        n = Nx.size
        sl = self._sl(slices, n)
        v = np.empty(n)
        self._ck(self._L.vls_spline2d_evaluate_c(self._h, n, _i64(sl) if sl is not None else None,
                                                 _i32(Nx), _d(x), _i32(Ny), _d(y), _d(v)))
        return v

    def evaluateNxPy(self, Nx, yy, slices=None):
        Nx = np.ascontiguousarray(Nx, dtype=np.int32).ravel()
        yy = np.ascontiguousarray(yy, dtype=np.float64).ravel()
        n = Nx.size
        sl = self._sl(slices, n)
        v = np.empty(n)
        self._ck(self._L.vls_spline2d_evaluate_nxpy(
            self._h, n, _i64(sl) if sl is not None else None, _i32(Nx), _d(yy), _d(v)))
        return v

    def evaluate(self, xx, yy, slices=None):
        xx = np.ascontiguousarray(xx, dtype=np.float64).ravel()
        yy = np.ascontiguousarray(yy, dtype=np.float64).ravel()
        n = xx.size
        sl = self._sl(slices, n)
        v = np.empty(n)
        self._ck(self._L.vls_spline2d_evaluate(self._h, n, _i64(sl) if sl is not None else None,
                                               _d(xx), _d(yy), _d(v)))
        return v


class InterpolSpline:
    """interpolSpline: createInit(...) returns the init struct, create(ini, data)
    an instance, evaluate(x, y[, grad[, hess]]) values (and derivatives in
    rescaled coordinates, einspline's order: d/dy first)."""

    @staticmethod
    def createInit(xstart, xstop, Nx, ystart, ystop, Ny, xbctL="natural", xbctR="natural",
                   ybctL="natural", ybctR="natural", xscaleType="linear", yscaleType="linear",
                   vltype=True, useLog=False, xbcvL=0.0, xbcvR=0.0, ybcvL=0.0, ybcvR=0.0):
        L = _lib.load()
        ini = _lib.InterpInit()
        rc = L.vls_interp_create_init(
            float(xstart), float(xstop), int(Nx), float(ystart), float(ystop), int(Ny),
            _lib.EBC[xbctL], _lib.EBC[xbctR], _lib.EBC[ybctL], _lib.EBC[ybctR],
            _lib.SCALES[xscaleType], _lib.SCALES[yscaleType], 1 if vltype else 0,
            1 if useLog else 0, xbcvL, xbcvR, ybcvL, ybcvR, ctypes.byref(ini))
        if rc != 0:
            raise _lib.VlsError(rc, L.vls_interp_last_error(None).decode())
        return ini

    def __init__(self, ini, data, device: int = 0):
        L = _lib.load()
        self._L = L
        self.ini = ini
        v = np.ascontiguousarray(data, dtype=np.float64)
        if v.size != ini.nx * ini.ny:
            raise ValueError("create: data must hold ny x nx values")
        h = ctypes.c_void_p()
        rc = L.vls_interp_create(ctypes.byref(ini), _d(v), int(device), ctypes.byref(h))
        if rc != 0:
            raise _lib.VlsError(rc, L.vls_interp_last_error(None).decode())
        self._h = h

    @classmethod
    def create(cls, ini, data, device: int = 0):
        return cls(ini, data, device)

    def evaluate(self, x, y, grad: bool = False, hess: bool = False):
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = np.ascontiguousarray(y, dtype=np.float64).ravel()
        n = x.size
        v = np.empty(n)
        g = np.empty((n, 2)) if (grad or hess) else None
        h = np.empty((n, 4)) if hess else None
        rc = self._L.vls_interp_evaluate(self._h, n, _d(x), _d(y), _d(v),
                                         _d(g) if g is not None else None,
                                         _d(h) if h is not None else None)
        if rc != 0:
            raise _lib.VlsError(rc, self._L.vls_interp_last_error(self._h).decode())
        if hess:
            return v, g, h
        return (v, g) if grad else v

    def destroy(self):
        if getattr(self, "_h", None):
            self._L.vls_interp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
