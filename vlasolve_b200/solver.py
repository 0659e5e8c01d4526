"""Host-side mirror of the reference solver for the spherical (r, v_r, J) path.

``VlasovSolver21Spline`` keeps the surface of the reference's
``vlasovSolver21_spline`` (vlasovSolver21_spline.hxx:16) and its base classes:
``init`` from ``-group.param`` options (vlasovSolver.hxx:61-102),
``makeOneStep`` (vlasovSolver21_spline.hxx:680-801), ``statistics``
(vlasovSolver21.hxx:644-690), ``snapshot`` (vlasovSolver21.hxx:585-598) and
``run`` (vlasovSolver.hxx:134-190).  Every computation goes through the CUDA
C-ABI library; nothing here computes on the CPU.

Defaults follow each profile's ``defaultGridParams`` / ``defaultSolverParams``
(initGen_UniformDensitySphere.hxx:82-112, initGen_PowerLawDensitySphere.hxx:92-136,
initGen_Plummer.hxx:52-85, initGen_Hernquist.hxx:58-93).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from .params import ParamsParser

_P = ctypes.POINTER


def _dptr(a):
    return a.ctypes.data_as(_P(ctypes.c_double))


# ------------------------------------------------------------------ defaults
def _pldf_sigma2(init):
    n, M, eta, alpha = init["n"], init["M"], init["eta"], init["alpha"]
    R0 = init["R0"] if init["R0_given"] else 1.0 / eta
    sigO2 = (3.0 - n) / (5.0 - 2 * n) * (M * eta) / (R0 * (alpha * 0.5 + 1))
    sigR2 = sigO2 * 0.5 * alpha
    return sigO2 + 2 * sigR2


def default_grid(init_type, init):
    if init_type == "UDF":
        return dict(Pmin=0.01, Pmax=25.0, Pres=200, Pscale="logarithmic",
                    Umin=(-2.0, 0.0), Umax=(2.0, 1.6), Ures=(200, 200),
                    Uscale=("linear", "quadratic"))
    if init_type == "PLDF":
        s = math.sqrt(_pldf_sigma2(init))
        return dict(Pmin=0.01, Pmax=200.0, Pres=200, Pscale="logarithmic",
                    Umin=(-16 * s, 0.0), Umax=(16 * s, 1.6), Ures=(200, 200),
                    Uscale=("linear", "quadratic"))
    if init_type == "Plummer":
        return dict(Pmin=0.01, Pmax=25.0 * 4, Pres=45 * 4, Pscale="logarithmic",
                    Umin=(-1.45, 0.0), Umax=(1.45, 3.24), Ures=(40 * 2, 20 * 4),
                    Uscale=("linear", "quadratic"))
    if init_type == "Hernquist":
        return dict(Pmin=0.01, Pmax=25.0 * 10, Pres=45 * 2, Pscale="logarithmic",
                    Umin=(-1.45, 1.0e-4), Umax=(1.45, 3.24 * 4), Ures=(40 * 2, 20 * 4),
                    Uscale=("linear", "logarithmic"))
    raise ValueError(f"ERROR: unknown initial conditions type {init_type}")


def default_solver(init_type):
    if init_type in ("UDF", "PLDF"):
        return dict(G=1.0, T0=0.0, dt=0.005, Tmax=60.0)
    if init_type == "Plummer":
        return dict(G=1.0, T0=0.0, Tmax=62.0, dt=0.1)
    if init_type == "Hernquist":
        return dict(G=1.0, T0=0.0, Tmax=62.0, dt=0.025)
    raise ValueError(f"ERROR: unknown initial conditions type {init_type}")


def default_init(init_type):
    if init_type == "UDF":
        return dict(M=1.0, R0=2.0, alpha=0.5, smoothingRadius=0.5, gap=(0.0, 0.0),
                    eta=0.1, n=1.0, Ra=-1.0, R0_given=1)
    if init_type == "PLDF":
        return dict(M=1.0, R0=10.0, alpha=2.0, smoothingRadius=0.5, gap=(0.0, 0.0),
                    eta=0.1, n=1.0, Ra=-1.0, R0_given=0)
    if init_type in ("Plummer", "Hernquist"):
        return dict(M=1.0, R0=1.0, alpha=0.5, smoothingRadius=0.5, gap=(0.0, 0.0),
                    eta=0.1, n=1.0, Ra=-1.0, R0_given=1)
    raise ValueError(f"ERROR: unknown initial conditions type {init_type}")


@dataclass
class Config:
    """Resolved grid.*, solver.* and init.* options."""
    init_type: str
    grid: dict
    solver: dict
    init: dict


def config_from_params(params: ParamsParser) -> Config:
    """Resolve options exactly as vlasovSolver::init and gridHandler do."""
    t = params.get("type", "init", "UDF")
    ini = default_init(t)
    for k in ("M", "alpha", "smoothingRadius", "eta", "n", "Ra"):
        ini[k] = params.get(k, "init", ini[k], 0 if t in ("UDF", "PLDF") else -1,
                            typ=float)
    if params.is_defined("R0", "init"):
        ini["R0"] = params.get("R0", "init", ini["R0"], 0, typ=float)
        ini["R0_given"] = 1
    ini["gap"] = (params.get("gap", "init", 0.0, 0, typ=float),
                  params.get("gap", "init", 0.0, 1, typ=float))
    sol = default_solver(t)
    for k in ("G", "T0", "Tmax", "dt"):
        sol[k] = params.get(k, "solver", sol[k], typ=float)
    sol["statsEvery"] = params.get("statsEvery", "solver", 25, typ=int)
    sol["snapshotEvery"] = params.get("snapshotEvery", "solver", 500, typ=int)
    sol["restartEvery"] = params.get("restartEvery", "solver", 5000, typ=int)
    sol["noLinking"] = params.get("noLinking", "solver", False, typ=bool)
    sol["kernelType"] = params.get("kernelType", "solver", "delayed")
    sol["kernelBufferSize"] = params.get("kernelBufferSize", "solver", 0, typ=int)
    if sol["kernelType"] not in _lib.KERNELS:
        raise ValueError(f"invalid kernel type '{sol['kernelType']}'")
    g = default_grid(t, ini)
    g["Pmin"] = params.get("Pmin", "grid", g["Pmin"], 0, typ=float)
    g["Pmax"] = params.get("Pmax", "grid", g["Pmax"], 0, typ=float)
    g["Pres"] = params.get("Pres", "grid", g["Pres"], 0, typ=int)
    g["Pscale"] = params.get("Pscale", "grid", g["Pscale"], 0, typ=str)
    g["Umin"] = tuple(params.get("Umin", "grid", g["Umin"][i], i, typ=float) for i in (0, 1))
    g["Umax"] = tuple(params.get("Umax", "grid", g["Umax"][i], i, typ=float) for i in (0, 1))
    g["Ures"] = tuple(params.get("Ures", "grid", g["Ures"][i], i, typ=int) for i in (0, 1))
    g["Uscale"] = tuple(params.get("Uscale", "grid", g["Uscale"][i], i, typ=str)
                        for i in (0, 1))
    for s in (g["Pscale"],) + g["Uscale"]:
        if s not in _lib.SCALES:  # scale names are lowercase (scale.hxx:25-29)
            raise ValueError(f"invalid scale type '{s}'")
    return Config(t, g, sol, ini)


def config_from_dict(d: dict) -> Config:
    """Same as config_from_params, from a flat dict using the option names."""
    args = []
    for k, v in d.items():
        if k == "type":
            args += ["-init.type", str(v)]
            continue
        cat = ("grid" if k in ("Pmin", "Pmax", "Pres", "Pscale", "Umin", "Umax", "Ures",
                               "Uscale") else
               "solver" if k in ("G", "T0", "Tmax", "dt", "statsEvery", "snapshotEvery",
                                 "restartEvery", "noLinking", "kernelType",
                                 "kernelBufferSize") else "init")
        vals = v if isinstance(v, (tuple, list)) else [v]
        args += [f"-{cat}.{k}"] + [repr(x) if isinstance(x, float) else str(x)
                                   for x in vals]
    return config_from_params(ParamsParser(args))


def _descs(cfg: Config, precision: str, device: int):
    g = _lib.GridDesc()
    gg = cfg.grid
    g.Pmin, g.Pmax, g.Pres = gg["Pmin"], gg["Pmax"], gg["Pres"]
    g.Pscale = _lib.SCALES[gg["Pscale"]]
    g.Umin[0], g.Umin[1] = gg["Umin"]
    g.Umax[0], g.Umax[1] = gg["Umax"]
    g.Ures[0], g.Ures[1] = gg["Ures"]
    g.Uscale[0], g.Uscale[1] = (_lib.SCALES[x] for x in gg["Uscale"])
    s = _lib.SolverDesc()
    ss = cfg.solver
    s.G, s.T0, s.Tmax, s.dt = ss["G"], ss["T0"], ss["Tmax"], ss["dt"]
    s.noLinking = int(ss["noLinking"])
    s.kernelType = _lib.KERNELS[ss["kernelType"]]
    s.kernelBufferSize = ss["kernelBufferSize"]
    s.precision = _lib.PRECISIONS[precision]
    s.device = device
    i = _lib.InitDesc()
    ii = cfg.init
    i.type = _lib.PROFILES[cfg.init_type]
    i.M, i.R0, i.alpha, i.smoothingRadius = ii["M"], ii["R0"], ii["alpha"], ii["smoothingRadius"]
    i.gap[0], i.gap[1] = ii["gap"]
    i.eta, i.n, i.Ra, i.R0_given = ii["eta"], ii["n"], ii["Ra"], int(ii["R0_given"])
    return g, s, i


class VlasovSolver21Spline:
    """One resident phase-space grid on one B200 and its step.

    precision: "fp64" (every value FP64) or "fp32" (FP32 f, coefficients and
    gathers; FP64 recursions, indexing, moments and statistics).
    layout: kernel layouts (vls_layout_desc), None for the defaults: a dict
    with any of prefilter ("auto", "segment"), drift ("auto", "window",
    "strip2", "strip1"), slices_per_batch, streams, drift_wait_spins.
    """

    def __init__(self, cfg: Config | ParamsParser | dict, precision: str = "fp64",
                 device: int = 0, init: bool = True, layout: dict | None = None):
        L = _lib.load()
        if isinstance(cfg, ParamsParser):
            cfg = config_from_params(cfg)
        elif isinstance(cfg, dict):
            cfg = config_from_dict(cfg)
        self.cfg = cfg
        self.precision = precision
        self._L = L
        gd, sd, idesc = _descs(cfg, precision, device)
        self._init_desc = idesc
        h = ctypes.c_void_p()
        lay = None
        if layout:
            lay = _lib.LayoutDesc()
            for k, v in layout.items():
                if k == "prefilter":
                    v = _lib.PREFILTERS[v] if isinstance(v, str) else v
                elif k == "drift":
                    v = _lib.DRIFTS[v] if isinstance(v, str) else v
                elif k not in ("slices_per_batch", "streams", "drift_wait_spins"):
                    raise ValueError(f"unknown layout field '{k}'")
                setattr(lay, k, int(v))
        _lib.check(L.vls_create_layout(ctypes.byref(gd), ctypes.byref(sd),
                                       ctypes.byref(lay) if lay is not None else None,
                                       ctypes.byref(h)))
        self._h = h
        nr, nu, nj = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        L.vls_dims(h, ctypes.byref(nr), ctypes.byref(nu), ctypes.byref(nj))
        self.nr, self.nu, self.nj = nr.value, nu.value, nj.value
        self.shape = (self.nj, self.nu, self.nr)
        self.ncells = self.nr * self.nu * self.nj
        self.mass_before = None
        if init:
            self.init_profile()

    def layout(self) -> dict:
        """The kernel layouts this solver uses (vls_get_layout)."""
        d = _lib.LayoutDesc()
        self._ck(self._L.vls_get_layout(self._h, ctypes.byref(d)))
        pre = {v: k for k, v in _lib.PREFILTERS.items()}
        drift = {v: k for k, v in _lib.DRIFTS.items()}
        return dict(prefilter=pre.get(d.prefilter, d.prefilter),
                    drift=drift.get(d.drift, d.drift),
                    slices_per_batch=d.slices_per_batch, streams=d.streams,
                    drift_wait_spins=d.drift_wait_spins, u_chunk_rows=d.u_chunk_rows,
                    r_chunk_rows=d.r_chunk_rows)

    # -- life cycle -------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._L.vls_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, code):
        _lib.check(code, self._h)

    def init_profile(self):
        mb = ctypes.c_double()
        self._ck(self._L.vls_init_profile(self._h, ctypes.byref(self._init_desc),
                                          ctypes.byref(mb)))
        self.mass_before = mb.value

    # -- data ---------------------------------------------------------------
    def coords(self):
        R, U = np.empty(self.nr), np.empty(self.nu)
        J, JV = np.empty(self.nj), np.empty(self.nj + 1)
        self._ck(self._L.vls_coords(self._h, _dptr(R), _dptr(U), _dptr(J), _dptr(JV)))
        return R, U, J, JV

    @property
    def f(self) -> np.ndarray:
        out = np.empty(self.shape)
        self._ck(self._L.vls_get_f(self._h, _dptr(out), out.size))
        return out

    @f.setter
    def f(self, val):
        v = np.ascontiguousarray(val, dtype=np.float64).reshape(self.shape)
        self._ck(self._L.vls_set_f(self._h, _dptr(v), v.size))

    def get_f_into(self, out: np.ndarray):
        self._ck(self._L.vls_get_f(self._h, _dptr(out), out.size))

    def set_f_from(self, arr: np.ndarray):
        self._ck(self._L.vls_set_f(self._h, _dptr(arr), arr.size))

    def footpoints(self):
        n = self.ncells
        rI, uI = np.empty(n, np.int32), np.empty(n, np.int32)
        rF, uF, dR = np.empty(n), np.empty(n), np.empty(n)
        out = np.empty(n, np.uint8)
        i32 = _P(ctypes.c_int32)
        self._ck(self._L.vls_get_footpoints(
            self._h, rI.ctypes.data_as(i32), _dptr(rF), uI.ctypes.data_as(i32), _dptr(uF),
            out.ctypes.data_as(_P(ctypes.c_uint8)), _dptr(dR)))
        return dict(rI=rI, rF=rF, uI=uI, uF=uF, out=out, driftR=dR)

    def chains(self):
        nc, ne = ctypes.c_int64(), ctypes.c_int64()
        N = _P(ctypes.c_int64)
        self._ck(self._L.vls_get_chains(self._h, ctypes.byref(nc), ctypes.byref(ne),
                                        None, None, None, None, None, None))
        nc, ne = nc.value, ne.value
        cell, start = np.empty(nc, np.int64), np.empty(nc, np.int64)
        ln = np.empty(nc, np.int32)
        R, U, val = np.empty(ne), np.empty(ne), np.empty(ne)
        self._ck(self._L.vls_get_chains(
            self._h, None, None, cell.ctypes.data_as(N), start.ctypes.data_as(N),
            ln.ctypes.data_as(_P(ctypes.c_int32)), _dptr(R), _dptr(U), _dptr(val)))
        return dict(cell=cell, start=start, len=ln, R=R, U=U, val=val)

    def set_chain_values(self, val):
        v = np.ascontiguousarray(val, dtype=np.float64)
        self._ck(self._L.vls_set_chain_values(self._h, _dptr(v), v.size))

    # -- step -----------------------------------------------------------------
    def makeOneStep(self, t: float | None = None):
        self._ck(self._L.vls_step(self._h, 1))

    def step(self, n: int = 1):
        self._ck(self._L.vls_step(self._h, int(n)))

    def sync(self):
        self._ck(self._L.vls_sync(self._h))

    def kernel_launches(self) -> int:
        n = ctypes.c_int64()
        self._ck(self._L.vls_kernel_launches(self._h, ctypes.byref(n)))
        return n.value

    def stream_ptr(self) -> int:
        """cudaStream_t (as an integer) every launch of this solver goes to."""
        p = ctypes.c_void_p()
        self._ck(self._L.vls_stream(self._h, ctypes.byref(p)))
        return p.value or 0

    def set_profiling(self, on: bool = True):
        self._ck(self._L.vls_set_profiling(self._h, int(on)))

    def profile_read(self) -> dict:
        """Summed device milliseconds and launch counts per kernel kind since
        the last read (requires set_profiling(True))."""
        nk = len(_lib.KERNEL_KINDS)
        ms = np.zeros(nk)
        cnt = np.zeros(nk, np.int64)
        self._ck(self._L.vls_profile_read(self._h, _dptr(ms),
                                          cnt.ctypes.data_as(_P(ctypes.c_int64)), nk))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_lib.KERNEL_KINDS)
                if cnt[i]}

    def last_mass(self) -> float:
        m = ctypes.c_double()
        self._ck(self._L.vls_last_mass(self._h, ctypes.byref(m)))
        return m.value

    def last_mass_into(self, out: np.ndarray, index: int):
        """Queue the copy of the most recent step's mass into out[index]
        (vls_last_mass_async): out is a float64 array, ideally in page-locked
        memory; the value is there after the next synchronising call."""
        if out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array")
        if not 0 <= index < out.size:
            raise IndexError(index)
        ptr = ctypes.cast(out.ctypes.data + 8 * index, _P(ctypes.c_double))
        self._ck(self._L.vls_last_mass_async(self._h, ptr))

    def moments(self):
        b, M, t = np.empty(self.nr), np.empty(self.nr), ctypes.c_double()
        self._ck(self._L.vls_moments(self._h, _dptr(b), _dptr(M), ctypes.byref(t)))
        return b, M, t.value

    def stats(self) -> dict:
        o = _lib.StatsOut()
        self._ck(self._L.vls_stats(self._h, ctypes.byref(o)))
        return dict(time=o.time, step=o.step, Mass=o.Mass, E=o.E, Ek=o.Ek, Ep=o.Ep,
                    S=o.S, L1=o.L1, L2=o.L2)

    @property
    def time(self):
        t, s = ctypes.c_double(), ctypes.c_int64()
        self._ck(self._L.vls_get_time(self._h, ctypes.byref(t), ctypes.byref(s)))
        return t.value

    def set_time(self, time: float, step: int = 0):
        self._ck(self._L.vls_set_time(self._h, float(time), int(step)))

    @property
    def stepCount(self):
        t, s = ctypes.c_double(), ctypes.c_int64()
        self._ck(self._L.vls_get_time(self._h, ctypes.byref(t), ctypes.byref(s)))
        return s.value

    def shell_volumes(self) -> np.ndarray:
        """(4 pi / 3)(R_{r+1}^3 - R_r^3) for the N_r - 1 radial shells."""
        R = self.coords()[0]
        return (4.0 * np.pi / 3.0) * (R[1:] ** 3 - R[:-1] ** 3)

    def radial_density(self) -> np.ndarray:
        """Mass of each radial shell (the moment's bins) over its volume; the
        last bin, of zero width, is dropped."""
        bins = self.moments()[0]
        return bins[:-1] / self.shell_volumes()

    # -- adjoint --------------------------------------------------------------
    def adjoint_forward(self, nsteps: int, checkpoint_every: int):
        """Runs nsteps steps keeping a state every checkpoint_every steps
        (vls_adjoint_forward)."""
        self._ck(self._L.vls_adjoint_forward(self._h, int(nsteps), int(checkpoint_every)))

    def adjoint_backward(self, dbins):
        """dL/dbins of the final radial bins -> (dL/df0 [j][u][r], dL/dchain0)
        for the initial grid and initial chain values (vls_adjoint_backward)."""
        db = np.ascontiguousarray(dbins, dtype=np.float64)
        df0 = np.empty(self.shape)
        nc, ne = ctypes.c_int64(), ctypes.c_int64()
        self._ck(self._L.vls_get_chains(self._h, ctypes.byref(nc), ctypes.byref(ne),
                                        None, None, None, None, None, None))
        dch = np.empty(ne.value)
        self._ck(self._L.vls_adjoint_backward(
            self._h, _dptr(db), db.size, _dptr(df0), df0.size,
            _dptr(dch) if ne.value else None, ne.value))
        return df0, dch

    def adjoint_set_inner(self, inner_every: int = 0):
        """Second-level checkpoint spacing of the backward pass (0: chosen
        from free device memory; vls_adjoint_set_inner)."""
        self._ck(self._L.vls_adjoint_set_inner(self._h, int(inner_every)))

    def init_desc(self, **kw) -> "_lib.InitDesc":
        """A copy of the handle's init.* parameters with some changed."""
        d = _lib.InitDesc()
        ctypes.pointer(d)[0] = self._init_desc
        for k, v in kw.items():
            if not hasattr(d, k):
                raise KeyError(k)
            setattr(d, k, v)
            if k == "R0":
                d.R0_given = 1
        return d

    def adjoint_init_dot(self, plus: dict, minus: dict):
        """(<dL/df0, f(plus) - f(minus)>, <dL/dc0, c(plus) - c(minus)>) for the
        last adjoint_backward and the initial states of two sets of init.*
        parameters (vls_adjoint_init_dot)."""
        dg, dc = ctypes.c_double(), ctypes.c_double()
        self._ck(self._L.vls_adjoint_init_dot(self._h, ctypes.byref(self.init_desc(**plus)),
                                              ctypes.byref(self.init_desc(**minus)),
                                              ctypes.byref(dg), ctypes.byref(dc)))
        return dg.value, dc.value

    def adjoint_inner_used(self) -> int:
        """Second-level spacing the last backward pass used (0: one level)."""
        v = ctypes.c_int32()
        self._ck(self._L.vls_adjoint_inner_used(self._h, ctypes.byref(v)))
        return v.value

    def device_bytes(self) -> int:
        """Device memory the handle holds (vls_device_bytes); also its peak."""
        v = ctypes.c_size_t()
        self._ck(self._L.vls_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    def set_init_params(self, **kw):
        """Changes init.* parameters (R0, alpha, smoothingRadius, M, eta, n, Ra)
        and regenerates the initial state."""
        for k, v in kw.items():
            if not hasattr(self._init_desc, k):
                raise KeyError(k)
            setattr(self._init_desc, k, v)
            if k == "R0":
                self._init_desc.R0_given = 1
        self.init_profile()

    # -- output ---------------------------------------------------------------
    def snapshot(self, fname: str | None = None):
        """vlasovSolver21::snapshot: writes snapshot_%4.4f.ND (vlasovSolver21.hxx:585-598)."""
        if fname is None:
            fname = "snapshot_%4.4f.ND" % self.time
        self._ck(self._L.vls_write_ndfield(self._h, fname.encode()))
        return fname

    def write_restart(self, fname: str, snapshot_every: int = 500, restart_every: int = 5000,
                      stats_every: int = 25):
        """vlasovSolver::write: the .vls restart file of the current state."""
        self._ck(self._L.vls_write_restart(self._h, fname.encode(), int(snapshot_every),
                                           int(restart_every), int(stats_every)))
        return fname

    def read_restart(self, fname: str):
        """Loads the grid, chain values, time and step count of a .vls file
        (the reference's or write_restart's) into this solver."""
        self._ck(self._L.vls_read_restart(self._h, fname.encode()))

    def load_snapshot(self, fname: str):
        self._ck(self._L.vls_read_ndfield(self._h, fname.encode()))

    def statistics(self, reset: bool = False, fname: str = "statistics.txt"):
        """Appends the row of vlasovSolver21::statistics (vlasovSolver21.hxx:679-689)."""
        s = self.stats()
        mode = "w" if reset else "a"
        with open(fname, mode) as fh:
            if reset:
                fh.write("# Time Step Mass E Ek Ep S L1 L2\n")
            fh.write("%.10g %d %10.10g %10.10g %10.10g %10.10g %10.10g %10.10g %10.10g\n" % (
                s["time"], s["step"], s["Mass"], s["E"], s["Ek"], s["Ep"], s["S"],
                s["L1"], s["L2"]))
        return s

    def run(self, outdir: str = "."):
        """vlasovSolver::run (vlasovSolver.hxx:134-190) without restart dumps."""
        sp = self.cfg.solver
        dt, tmax = sp["dt"], sp["Tmax"]

        def check_timer(every, n):
            return every >= 0 and n % every == 0

        def check_time():
            t = self.time
            return tmax <= 0 or (t < tmax and abs(t - tmax) > dt / 100)

        if not check_time():
            return
        while True:
            n = self.stepCount
            if check_timer(sp["snapshotEvery"], n):
                self.snapshot(os.path.join(outdir, "snapshot_%4.4f.ND" % self.time))
            if check_timer(sp["statsEvery"], n):
                self.statistics(n == 0, os.path.join(outdir, "statistics.txt"))
            self.makeOneStep(self.time)
            if not check_time():
                break
        if check_timer(sp["snapshotEvery"], self.stepCount):
            self.snapshot(os.path.join(outdir, "snapshot_%4.4f.ND" % self.time))


def restart_info(fname: str) -> dict:
    """Grid and solver parameters, output intervals, time and step count stored
    in a .vls restart file (vls_restart_info; the J minimum is not stored)."""
    L = _lib.load()
    g, sd = _lib.GridDesc(), _lib.SolverDesc()
    every = (ctypes.c_int64 * 3)()
    t, st = ctypes.c_double(), ctypes.c_int64()
    _lib.check(L.vls_restart_info(fname.encode(), ctypes.byref(g), ctypes.byref(sd), every,
                                  ctypes.byref(t), ctypes.byref(st)))
    scales = {v: k for k, v in _lib.SCALES.items()}
    kernels = {v: k for k, v in _lib.KERNELS.items()}
    return {"Pmin": g.Pmin, "Pmax": g.Pmax, "Pres": g.Pres, "Pscale": scales[g.Pscale],
            "Umin": (g.Umin[0], g.Umin[1]), "Umax": (g.Umax[0], g.Umax[1]),
            "Ures": (g.Ures[0], g.Ures[1]), "Uscale": (scales[g.Uscale[0]], scales[g.Uscale[1]]),
            "G": sd.G, "T0": sd.T0, "Tmax": sd.Tmax, "dt": sd.dt,
            "noLinking": sd.noLinking, "kernelType": kernels[sd.kernelType],
            "kernelBufferSize": sd.kernelBufferSize, "snapshotEvery": every[0],
            "restartEvery": every[1], "statsEvery": every[2], "time": t.value,
            "step": st.value}
