"""ctypes wrapper of the CPU oracle (oracle/vls_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by ``bench.py``'s CPU-baseline leg.  The product package
never imports this module.

The oracle restates the reference step (vlasovSolver21_spline::makeOneStep,
vlasovSolver21_spline.hxx:680-801, and everything it calls) in FP64 and in
the reference's operation order; see vls_oracle.c for per-function citations.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libvls_oracle.so")

SCALES = {"linear": 0, "logarithmic": 1, "quadratic": 2}
PROFILES = {"UDF": 0, "PLDF": 1, "Plummer": 2, "Hernquist": 3}
KERNELS = {"delayed": 0, "reflective": 1}


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (no FMA contraction, like the reference)."""
    src = os.path.join(_HERE, "vls_oracle.c")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.check_call([
            "gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
            "-o", _SO, src, "-lm"])
    return _SO


class _Params(ctypes.Structure):
    _fields_ = [
        ("Pmin", ctypes.c_double), ("Pmax", ctypes.c_double),
        ("Pres", ctypes.c_int), ("Pscale", ctypes.c_int),
        ("Umin", ctypes.c_double * 2), ("Umax", ctypes.c_double * 2),
        ("Ures", ctypes.c_int * 2), ("Uscale", ctypes.c_int * 2),
        ("G", ctypes.c_double), ("dt", ctypes.c_double),
        ("noLinking", ctypes.c_int), ("kernelType", ctypes.c_int),
        ("kernelBufferSize", ctypes.c_int),
        ("initType", ctypes.c_int),
        ("M", ctypes.c_double), ("R0", ctypes.c_double),
        ("alpha", ctypes.c_double), ("smoothingRadius", ctypes.c_double),
        ("gap0", ctypes.c_double), ("gap1", ctypes.c_double),
        ("eta", ctypes.c_double), ("n", ctypes.c_double),
        ("Ra", ctypes.c_double), ("R0_given", ctypes.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        P = ctypes.POINTER
        d, i64, i32, u8 = (ctypes.c_double, ctypes.c_int64, ctypes.c_int32,
                           ctypes.c_uint8)
        L.vlo_create.restype = ctypes.c_void_p
        L.vlo_create.argtypes = [P(_Params)]
        L.vlo_destroy.argtypes = [ctypes.c_void_p]
        L.vlo_dims.argtypes = [ctypes.c_void_p, P(ctypes.c_long), P(ctypes.c_long),
                               P(ctypes.c_long)]
        L.vlo_coords.argtypes = [ctypes.c_void_p, P(d), P(d), P(d), P(d)]
        L.vlo_spline_consts.argtypes = [ctypes.c_void_p, P(d), P(d)]
        L.vlo_kernel_radius.restype = d
        L.vlo_kernel_radius.argtypes = [ctypes.c_void_p]
        L.vlo_get_f.argtypes = [ctypes.c_void_p, P(d)]
        L.vlo_set_f.argtypes = [ctypes.c_void_p, P(d)]
        L.vlo_get_footpoints.argtypes = [ctypes.c_void_p, P(d), P(d), P(u8), P(i32),
                                         P(d), P(i32), P(d)]
        L.vlo_chain_counts.argtypes = [ctypes.c_void_p, P(ctypes.c_long),
                                       P(ctypes.c_long)]
        L.vlo_get_chains.argtypes = [ctypes.c_void_p, P(i64), P(i64), P(i32), P(d),
                                     P(d), P(d)]
        L.vlo_set_chain_vals.argtypes = [ctypes.c_void_p, P(d)]
        L.vlo_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.vlo_moments.restype = d
        L.vlo_moments.argtypes = [ctypes.c_void_p, P(d), P(d)]
        L.vlo_stats.argtypes = [ctypes.c_void_p, P(d)]
        L.vlo_prefilter2d.argtypes = [ctypes.c_long, ctypes.c_long, d, d, P(d), P(d)]
        L.vlo_evaluate_c.argtypes = [P(d), ctypes.c_long, ctypes.c_int, d, ctypes.c_int, d]
        L.vlo_evaluate_c.restype = d
        L.vlo_evaluate_nxpy.argtypes = [P(d), ctypes.c_long, ctypes.c_int, ctypes.c_int, d]
        L.vlo_evaluate_nxpy.restype = d
        L.vlo_kick.argtypes = [ctypes.c_void_p, P(d)]
        L.vlo_drift.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _ptr(a, ct=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def make_params(cfg: dict) -> _Params:
    """cfg uses the reference's option names (grid.*, solver.*, init.*)."""
    p = _Params()
    p.Pmin, p.Pmax = cfg["Pmin"], cfg["Pmax"]
    p.Pres, p.Pscale = cfg["Pres"], SCALES[cfg["Pscale"]]
    p.Umin[0], p.Umin[1] = cfg["Umin"]
    p.Umax[0], p.Umax[1] = cfg["Umax"]
    p.Ures[0], p.Ures[1] = cfg["Ures"]
    p.Uscale[0], p.Uscale[1] = SCALES[cfg["Uscale"][0]], SCALES[cfg["Uscale"][1]]
    p.G, p.dt = cfg.get("G", 1.0), cfg["dt"]
    p.noLinking = int(cfg.get("noLinking", 0))
    p.kernelType = KERNELS[cfg.get("kernelType", "delayed")]
    p.kernelBufferSize = int(cfg.get("kernelBufferSize", 0))
    p.initType = PROFILES[cfg["type"]]
    p.M = cfg.get("M", 1.0)
    p.R0 = cfg.get("R0", 2.0 if cfg["type"] == "UDF" else 1.0)
    p.alpha = cfg.get("alpha", 0.5 if cfg["type"] == "UDF" else 2.0)
    p.smoothingRadius = cfg.get("smoothingRadius", 0.5)
    gap = cfg.get("gap", (0.0, 0.0))
    p.gap0, p.gap1 = gap
    p.eta = cfg.get("eta", 0.1)
    p.n = cfg.get("n", 1.0)
    p.Ra = cfg.get("Ra", -1.0)
    p.R0_given = int("R0" in cfg)
    return p


class ReferenceHalt(RuntimeError):
    """The reference run ends during set-up for this configuration."""


class Oracle:
    """One oracle solver instance (FP64 CPU restatement of the reference)."""

    def __init__(self, cfg: dict):
        self._p = make_params(cfg)
        self._c = lib().vlo_create(ctypes.byref(self._p))
        if not self._c:
            # advanceParticleDrift reached the branch where the reference
            # prints and exits (vlasovSolver21.hxx:389-391)
            raise ReferenceHalt("the reference terminates in generateDisplacement "
                                "for this set-up (vlasovSolver21.hxx:389-391)")
        nr, nu, nj = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
        lib().vlo_dims(self._c, ctypes.byref(nr), ctypes.byref(nu), ctypes.byref(nj))
        self.nr, self.nu, self.nj = nr.value, nu.value, nj.value
        self.shape = (self.nj, self.nu, self.nr)

    def __del__(self):
        if getattr(self, "_c", None):
            lib().vlo_destroy(self._c)
            self._c = None

    def coords(self):
        R = np.empty(self.nr); U = np.empty(self.nu)
        J = np.empty(self.nj); JV = np.empty(self.nj + 1)
        lib().vlo_coords(self._c, _ptr(R), _ptr(U), _ptr(J), _ptr(JV))
        return R, U, J, JV

    def spline_consts(self):
        s = np.empty(2); h = np.empty(2)
        lib().vlo_spline_consts(self._c, _ptr(s), _ptr(h))
        return s, h

    def kernel_radius(self):
        return lib().vlo_kernel_radius(self._c)

    @property
    def f(self):
        out = np.empty(self.shape)
        lib().vlo_get_f(self._c, _ptr(out))
        return out

    @f.setter
    def f(self, val):
        v = np.ascontiguousarray(val, dtype=np.float64).reshape(self.shape)
        lib().vlo_set_f(self._c, _ptr(v))

    def footpoints(self):
        n = self.nr * self.nu * self.nj
        dR = np.empty(n); dU = np.empty(n); out = np.empty(n, np.uint8)
        rI = np.empty(n, np.int32); uI = np.empty(n, np.int32)
        rF = np.empty(n); uF = np.empty(n)
        lib().vlo_get_footpoints(self._c, _ptr(dR), _ptr(dU), _ptr(out, ctypes.c_uint8),
                                 _ptr(rI, ctypes.c_int32), _ptr(rF),
                                 _ptr(uI, ctypes.c_int32), _ptr(uF))
        return dict(driftR=dR, driftU=dU, out=out, rI=rI, rF=rF, uI=uI, uF=uF)

    def chains(self):
        nc, ne = ctypes.c_long(), ctypes.c_long()
        lib().vlo_chain_counts(self._c, ctypes.byref(nc), ctypes.byref(ne))
        nc, ne = nc.value, ne.value
        cell = np.empty(nc, np.int64); start = np.empty(nc, np.int64)
        ln = np.empty(nc, np.int32)
        R = np.empty(ne); U = np.empty(ne); val = np.empty(ne)
        lib().vlo_get_chains(self._c, _ptr(cell, ctypes.c_int64), _ptr(start, ctypes.c_int64),
                             _ptr(ln, ctypes.c_int32), _ptr(R), _ptr(U), _ptr(val))
        return dict(cell=cell, start=start, len=ln, R=R, U=U, val=val)

    def set_chain_vals(self, val):
        v = np.ascontiguousarray(val, dtype=np.float64)
        lib().vlo_set_chain_vals(self._c, _ptr(v))

    def step(self, n=1):
        lib().vlo_step(self._c, int(n))

    def moments(self):
        b = np.empty(self.nr); M = np.empty(self.nr)
        tot = lib().vlo_moments(self._c, _ptr(b), _ptr(M))
        return b, M, tot

    def stats(self):
        out = np.empty(7)
        lib().vlo_stats(self._c, _ptr(out))
        return dict(zip(["Mass", "E", "Ek", "Ep", "S", "L1", "L2"], out))

    def kick(self, shift):
        s = np.ascontiguousarray(shift, dtype=np.float64)
        lib().vlo_kick(self._c, _ptr(s))

    def drift(self):
        lib().vlo_drift(self._c)


def prefilter2d(f_slice, hi_r, hi_u):
    """Padded natural-BC coefficients of one (nu, nr) slice."""
    f = np.ascontiguousarray(f_slice, dtype=np.float64)
    nu, nr = f.shape
    out = np.empty((nu + 2, nr + 2))
    lib().vlo_prefilter2d(nr, nu, hi_r, hi_u, _ptr(f), _ptr(out))
    return out


def evaluate_c(coef, Nx, x, Ny, y):
    """localSpline::evaluateC on padded coefficients (nu + 2, nr + 2), per point."""
    c = np.ascontiguousarray(coef, dtype=np.float64)
    s1 = c.shape[1]
    return np.array([lib().vlo_evaluate_c(_ptr(c), s1, int(a), float(b), int(e), float(f))
                     for a, b, e, f in zip(Nx, x, Ny, y)])


def evaluate_nxpy(coef, Nx, Ny, y):
    """evaluateNxPy's sum at node Nx and the decomposed (Ny, y), per point."""
    c = np.ascontiguousarray(coef, dtype=np.float64)
    s1 = c.shape[1]
    return np.array([lib().vlo_evaluate_nxpy(_ptr(c), s1, int(a), int(e), float(f))
                     for a, e, f in zip(Nx, Ny, y)])
