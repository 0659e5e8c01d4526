"""Benchmark of the split semi-Lagrangian step on B200.

Default workload: Hernquist (M=1, a=1) on the 512x512x256 grid (513 x 513 x
256 = 67,371,264 cells), r log-scaled on [0.01, 50], v_r linear on [-3, 3],
J quadratic on [0, 3], dt = 0.0025, FP32-bulk path; the FP64 path is timed on
the same grid for the FP32/FP64 ratio.  Metric: phase-space cell updates per
second (N_r N_u N_J steps / device time).  The grid (269 MB FP32) is larger
than L2 (126 MB), so no flush is needed between steps.

Arms:
  python bench.py [--gpus N --steps K --warmup W]      this library (CUDA)
  python bench.py --impl reference ...                   the reference's own
      CPU implementation (OpenMP, all host cores) on the same workload
Multi-GPU: replicas only (one independent grid per rank, weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

WORKLOAD = dict(type="Hernquist", Pmin=0.01, Pmax=50.0, Pres=512, Pscale="logarithmic",
                Umin=(-3.0, 0.0), Umax=(3.0, 3.0), Ures=(512, 256),
                Uscale=("linear", "quadratic"), dt=0.0025)
WORKLOAD_NAME = "hernquist_512x512x256"
# smaller case of the same kernels for ncu captures (f = 135 MB FP32, > L2)
WORKLOADS = {
    "hernquist_512x512x256": WORKLOAD,
    "hernquist_512x512x128": dict(WORKLOAD, Ures=(512, 128)),
}
METRIC = "phase-space cell updates/s"
REF_BIN = os.path.join(HERE, "oracle", "_ref", "vlasolve")


def cells_of(w):
    return (w["Pres"] + 1) * (w["Ures"][0] + 1) * w["Ures"][1]


def config_json(w, precision):
    return {"workload": WORKLOAD_NAME, "grid": [w["Pres"] + 1, w["Ures"][0] + 1, w["Ures"][1]],
            "cells": cells_of(w), "profile": w["type"], "dt": w["dt"],
            "precision": precision, "l2": "inputs larger than L2 (f is 269 MB FP32)",
            "parallelism": "replicas"}


def ref_args(w):
    return ["-init.type", w["type"], "-grid.Pmin", repr(w["Pmin"]), "-grid.Pmax",
            repr(w["Pmax"]), "-grid.Pres", str(w["Pres"]), "-grid.Pscale", w["Pscale"],
            "-grid.Umin", repr(w["Umin"][0]), repr(w["Umin"][1]),
            "-grid.Umax", repr(w["Umax"][0]), repr(w["Umax"][1]),
            "-grid.Ures", str(w["Ures"][0]), str(w["Ures"][1]),
            "-grid.Uscale", w["Uscale"][0], w["Uscale"][1], "-solver.dt", repr(w["dt"])]


def run_reference(w, steps, threads):
    """Time the reference binary's own loop ('Computed N timesteps in Ts',
    vlasovSolver.hxx:184-186); returns (cell updates/s, seconds, steps)."""
    tmp = tempfile.mkdtemp(prefix="vls_ref_")
    try:
        args = [REF_BIN, "-threads_per_node", str(threads), "-verbose", "0"] + ref_args(w) + [
            "-solver.Tmax", repr(w["dt"] * steps), "-solver.statsEvery", "-1",
            "-solver.snapshotEvery", "-1", "-solver.restartEvery", "-1"]
        out = subprocess.run(args, cwd=tmp, capture_output=True, text=True, timeout=1800)
        m = re.search(r"Computed (\d+) timesteps in ([0-9.eE+-]+)s", out.stdout)
        if out.returncode != 0 or not m:
            raise RuntimeError("reference run failed: " + out.stdout[-500:] + out.stderr[-500:])
        n, t = int(m.group(1)), float(m.group(2))
        return cells_of(w) * n / t, t, n
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def cpu_info():
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count() or 1


# ------------------------------------------------------------------ clocks
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.p = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi") is None:
            return self
        fd, self.path = tempfile.mkstemp(prefix="vls_clk_", suffix=".csv")
        os.close(fd)
        self.p = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
             "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ GPU arm
def measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def max_over_ranks(x, dist, device="cuda"):
    """The largest of the ranks' values of x (every rank takes the same
    collective); x itself without a process group."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, cells, steps, seconds):
    """Whole-job cell updates/s of `world` replicas that each advanced `cells`
    cells `steps` times, the slowest in `seconds`."""
    return world * cells * steps / seconds


def time_steps(solver, steps, warmup, torch, dist):
    """Device time of `steps` steps on the solver's stream (CUDA events)."""
    stream = torch.cuda.ExternalStream(solver.stream_ptr())
    solver.step(warmup)
    solver.sync()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = solver.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.step(steps)
    e1.record(stream)
    solver.sync()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = solver.kernel_launches() - l0
    if dist is not None:
        ms = max_over_ranks(ms, dist)
        dist.barrier()
    return ms, launches


def gpu_arm(args):
    import numpy as np
    import torch
    from vlasolve_b200 import VlasovSolver21Spline

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    w = dict(WORKLOADS[args.workload])
    cells = cells_of(w)
    K, W = args.steps, args.warmup
    peak, peak_kind = measured_peaks()
    if args.quick:
        # timing only (used under ncu): no FP64 arm, statistics or end-to-end run
        s = VlasovSolver21Spline(w, precision=args.precision, device=local)
        ms, launches = time_steps(s, K, W, torch, dist)
        out = {"workload": args.workload, "precision": args.precision,
               "ms_per_step": ms / K, "launches": launches}
        if args.kernels:
            s.set_profiling(True)
            s.step(min(K, 20))
            prof = s.profile_read()
            s.set_profiling(False)
            out["kernels_ms_per_step"] = {k: v[0] / max(v[1], 1) for k, v in prof.items()}
        if rank == 0:
            print(json.dumps(out), flush=True)
        s.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    res = {}
    precs = [args.precision] + [p for p in ("fp32all", "fp64") if p != args.precision]
    for prec in precs:
        s = VlasovSolver21Spline(w, precision=prec, device=local)
        st0 = s.stats()
        with ClockSampler(local) as clk:
            ms, launches = time_steps(s, K, W, torch, dist)
        st1 = s.stats()
        # per-kernel device times from the library's event profile (1 extra step set)
        s.set_profiling(True)
        s.step(min(K, 20))
        prof = s.profile_read()
        s.set_profiling(False)
        res[prec] = dict(ms=ms, launches=launches, clocks=clk.summary(), prof=prof,
                         dE=(st1["E"] - st0["E"]) / abs(st0["E"]), steps_done=s.stepCount,
                         solver=s)
        if prec != args.precision:
            s.close()
            res[prec].pop("solver")

    main = res[args.precision]
    ms = main["ms"]
    value = replica_value(world, cells, K, ms * 1e-3)
    esize = 8 if args.precision == "fp64" else 4
    # dominant kernel and its roofline: algorithmic bytes = one read of its input
    # field + one write of its output field per cell (8 B FP32 / 16 B FP64)
    prof = main["prof"]
    dom = max(prof, key=lambda k: prof[k][0])
    dom_ms = prof[dom][0] / prof[dom][1]
    algo_bytes = 2 * esize * cells
    achieved = algo_bytes / (dom_ms * 1e-3) / 1e9
    step_achieved = 4 * esize * cells * K / (ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(HERE, "profiles", "traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get(dom)

    # end to end through the C-ABI with pinned host buffers: upload the state,
    # K steps each copying the step's mass to the host (queued on the
    # solver's stream, no stall between steps), download the state (which
    # waits for everything before it)
    s = main["solver"]
    host = torch.empty(cells, dtype=torch.float64).pin_memory()
    hnp = host.numpy()
    masses = torch.zeros(K, dtype=torch.float64).pin_memory().numpy()
    s.get_f_into(hnp)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.set_f_from(hnp)
    for i in range(K):
        s.step(1)
        s.last_mass_into(masses, i)
    s.get_f_into(hnp)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist)
    e2e = replica_value(world, cells, K, e2e_s)
    s.close()
    # every step's mass arrived on the host
    if not (np.all(np.isfinite(masses)) and np.all(masses > 0)):
        raise RuntimeError("end-to-end leg: a step's mass did not reach the host")

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        model, ncores = cpu_info()
        if os.path.exists(REF_BIN):
            v, t, n = run_reference(w, args.cpu_steps, ncores)
            cpu = {"value": v, "unit": "cell updates/s", "cores": ncores, "kind": "reference",
                   "sample": f"{n} steps of the full {WORKLOAD_NAME} grid, OpenMP "
                             f"{ncores} threads, {model}; reference's own loop timer",
                   "seconds": t}
        else:
            cpu = {"value": None, "unit": "cell updates/s", "cores": 0, "kind": "reference",
                   "sample": "reference binary not built"}
    line = {
        "metric": METRIC, "value": value, "unit": "cell updates/s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32",
        "data": "synthetic (analytic Hernquist distribution function)",
        "config": config_json(w, args.precision),
        "gpu_launches": main["launches"],
        "clocks": main["clocks"],
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": algo_bytes,
                     "step_achieved": step_achieved, "step_frac": step_achieved / peak},
        "kernels_ms_per_step": {k: v[0] / min(K, 20) for k, v in prof.items()},
        "e2e": {"value": e2e, "unit": "cell updates/s",
                "h2d_bytes_per_step": cells * 8 / K,
                "d2h_bytes_per_step": (cells * 8 + 8 * K) / K},
        "energy_drift_rel": {p: res[p]["dE"] for p in res},
        "cpu_baseline": cpu,
    }
    for p in res:
        if p == args.precision:
            continue
        v = world * cells * K / (res[p]["ms"] * 1e-3)
        line[p] = {"value": v, "ms_per_step": res[p]["ms"] / K,
                   "kernels_ms_per_step": {k: x[0] / min(K, 20)
                                           for k, x in res[p]["prof"].items()}}
    if "fp64" in line:
        line["fp32_over_fp64"] = value / line["fp64"]["value"]
    if world == 1 and not args.no_accuracy:
        line["configs"] = configs_block(100)
        line["accuracy"] = accuracy_block(args.accuracy_steps)
    if world == 1 and not args.no_adjoint:
        line["adjoint"] = adjoint_block(args.adjoint_steps, args.adjoint_every)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# accuracy run: Plummer M=1, a=1 on 257 x 257 x 128, dt = 0.005, 2000 steps
ACCURACY = dict(type="Plummer", Pmin=0.01, Pmax=25.0, Pres=256, Pscale="logarithmic",
                Umin=(-3.0, 0.0), Umax=(3.0, 2.0), Ures=(256, 128),
                Uscale=("linear", "quadratic"), dt=0.005)
# adjoint run: UDF theta = (R0, alpha, smoothingRadius) = (2, 0.5, 0.5) on
# 257 x 257 x 128, 500 steps at dt = 0.005, a checkpoint every 50 steps
ADJOINT = dict(type="UDF", Pmin=0.01, Pmax=25.0, Pres=256, Pscale="logarithmic",
               Umin=(-2.0, 0.0), Umax=(2.0, 1.6), Ures=(256, 128),
               Uscale=("linear", "quadratic"), dt=0.005)


# the listed configurations' grids, timed in both storage precisions
CONFIGS = {
    "udf_200x200x200": dict(type="UDF", Pmin=0.01, Pmax=25.0, Pres=200, Pscale="logarithmic",
                            Umin=(-2.0, 0.0), Umax=(2.0, 1.6), Ures=(200, 200),
                            Uscale=("linear", "quadratic"), dt=0.005),
}


def configs_block(steps):
    """Cell updates/s of the FP64 and FP32-bulk step on the UDF 201x201x200
    and Plummer 257x257x128 grids (device time, CUDA events, after 5 warm-up
    steps)."""
    import torch
    from vlasolve_b200 import VlasovSolver21Spline
    out = {}
    for name, w in (("udf_200x200x200", CONFIGS["udf_200x200x200"]),
                    ("plummer_256x256x128", ACCURACY)):
        out[name] = {}
        for prec in ("fp64", "fp32"):
            s = VlasovSolver21Spline(w, precision=prec)
            ms, _ = time_steps(s, steps, 5, torch, None)
            cells = s.nr * s.nu * s.nj
            out[name][prec] = {"ms_per_step": ms / steps, "value": cells * steps / (ms * 1e-3),
                               "cells": cells}
            s.close()
        out[name]["fp32_over_fp64"] = out[name]["fp32"]["value"] / out[name]["fp64"]["value"]
    return out


def accuracy_block(steps):
    """Mass and energy drift of each precision over `steps` steps, and the L2
    distance of the FP32 modes' final f from the FP64 path's (the FP64 path
    matches the oracle to 1e-12 per step)."""
    import numpy as np
    from vlasolve_b200 import VlasovSolver21Spline
    out, f64 = {}, None
    t0 = time.perf_counter()
    for prec in ("fp64", "fp32", "fp32all"):
        s = VlasovSolver21Spline(ACCURACY, precision=prec)
        a = s.stats()
        s.step(steps)
        b = s.stats()
        f = s.f
        if prec == "fp64":
            f64 = f
        out[prec] = {"mass_drift": (b["Mass"] - a["Mass"]) / a["Mass"],
                     "energy_drift": (b["E"] - a["E"]) / abs(a["E"])}
        if prec != "fp64":
            out[prec]["l2_vs_fp64"] = float(np.linalg.norm(f - f64) / np.linalg.norm(f64))
            out[prec]["energy_drift_minus_fp64"] = (out[prec]["energy_drift"]
                                                    - out["fp64"]["energy_drift"])
        s.close()
    return {"workload": "plummer_257x257x128", "steps": steps, "dt": ACCURACY["dt"],
            "reference": "FP64 GPU path", "seconds": time.perf_counter() - t0, **out}


def adjoint_block(nsteps, K):
    """Config of the adjoint: loss ||rho(theta) - rho(theta + dtheta)||_2 of the
    final radial density; gradient by the adjoint (FP64 and FP32 storage)
    against central differences of full FP64 runs (h = 1e-4).  Times: the
    whole backward pass of the autograd function (step adjoint plus the
    initial-state map; median of three, and the first), the step adjoint
    alone (vls_adjoint_backward, with
    its recomputation), and the plain forward of the same steps, the last two
    as device time on the solver's stream (and wall time), medians of three
    runs each; adjoint_over_forward is the step adjoint over that forward."""
    import numpy as np
    import torch
    from vlasolve_b200 import VlasovSolver21Spline
    from vlasolve_b200.adjoint import DensityProblem, final_density
    theta = np.array([2.0, 0.5, 0.5])
    dtheta = np.array([0.05, -0.02, 0.03])
    out = {"workload": "udf_257x257x128", "steps": nsteps, "checkpoint_every": K,
           "theta": theta.tolist(), "loss": "||rho - rho_target||_2, rho_target at theta + "
           + str(dtheta.tolist())}
    t_all = time.perf_counter()
    grads = {}
    for prec in ("fp64", "fp32"):
        p = DensityProblem(ADJOINT, precision=prec, nsteps=nsteps, checkpoint_every=K)
        target = p.run(theta + dtheta) if prec == "fp64" else target
        # the autograd forward and backward three times (wall time; the first
        # backward also builds the inverse footpoint map), the medians reported
        fwd_wall, bwd_wall = [], []
        for rep in range(3):
            th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rho = final_density(th, p)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            L = torch.linalg.norm(rho - torch.as_tensor(target))
            L.backward()
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            fwd_wall.append(t1 - t0)
            bwd_wall.append(t2 - t1)
            if rep == 0:
                grads[prec] = th.grad.numpy().copy()
                repeatable = True
            else:
                repeatable &= bool(np.array_equal(th.grad.numpy(), grads[prec]))
        # the step adjoint alone (recomputation included, initial-state map
        # excluded): three more backward passes with the same seed, and three
        # plain forward runs of the same steps; the medians are reported
        s = p.solver
        dbins = np.zeros(s.nr)
        dbins[:-1] = (torch.as_tensor(rho.detach()) - torch.as_tensor(target)).numpy()
        stream = torch.cuda.ExternalStream(s.stream_ptr())

        def timed_run(fn):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            s.sync()
            w0 = time.perf_counter()
            e0.record(stream)
            fn()
            e1.record(stream)
            s.sync()
            w1 = time.perf_counter()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) * 1e-3, w1 - w0

        def forward():
            s.set_init_params(**dict(zip(p.params, map(float, theta))))
            s.sync()
            return timed_run(lambda: s.step(nsteps))

        adj = [timed_run(lambda: s.adjoint_backward(dbins)) for _ in range(3)]
        fwd = [forward() for _ in range(3)]
        adj_dev = float(np.median([a[0] for a in adj]))
        fwd_dev = float(np.median([f[0] for f in fwd]))
        # device times (CUDA events on the solver's stream) and the wall times
        # around the same calls (host launch overhead included)
        out[prec] = {"grad": grads[prec].tolist(), "loss": float(L.detach()),
                     "forward_checkpointed_s": float(np.median(fwd_wall)),
                     "backward_s": float(np.median(bwd_wall)),
                     "backward_first_s": bwd_wall[0], "grad_bitwise_repeatable": repeatable,
                     "step_adjoint_s": adj_dev, "forward_s": fwd_dev,
                     "step_adjoint_runs_s": [a[0] for a in adj],
                     "forward_runs_s": [f[0] for f in fwd],
                     "step_adjoint_wall_s": float(np.median([a[1] for a in adj])),
                     "forward_wall_s": float(np.median([f[1] for f in fwd])),
                     "adjoint_over_forward": adj_dev / fwd_dev}
        if prec == "fp64":
            fd = np.zeros(3)
            h = 1e-4
            for k in range(3):
                tp, tm = theta.copy(), theta.copy()
                tp[k] += h
                tm[k] -= h
                fd[k] = (np.linalg.norm(p.run(tp) - target)
                         - np.linalg.norm(p.run(tm) - target)) / (2 * h)
            out["fd_grad"] = fd.tolist()
            out["fp64_vs_fd_rel"] = float(np.max(np.abs(grads["fp64"] - fd)) / np.max(np.abs(fd)))
        p.close()
    out["fp32_vs_fp64_rel"] = float(np.max(np.abs(grads["fp32"] - grads["fp64"]))
                                    / np.max(np.abs(grads["fp64"])))
    out["seconds"] = time.perf_counter() - t_all
    return out


# large case: PLDF (M=1, n=1, alpha=1, eta=0.1, smoothingRadius=0.5) on
# 1025 x 1025 x 512 (FP32 f of 2.15 GB), the PLDF default ranges (r log on
# [0.01, 200], v_r within 16 sigma, J quadratic on [0, 1.6]), dt = 0.005;
# the gradient check runs the same problem on 257 x 257 x 128
LARGE = dict(type="PLDF", M=1.0, n=1.0, alpha=1.0, eta=0.1, smoothingRadius=0.5,
             Pres=1024, Ures=(1024, 512), dt=0.005)
LARGE_SUB = dict(LARGE, Pres=256, Ures=(256, 128))
LARGE_PARAMS = ("n", "alpha", "smoothingRadius")


def large_block(nsteps, K):
    """Forward cell updates/s, device memory and the adjoint (checkpoint every
    K steps, second level chosen from free memory) of the 1025 x 1025 x 512
    PLDF case; FP32-storage gradient against the FP64 adjoint on the
    257 x 257 x 128 grid.  Loss ||rho(theta) - rho(theta + dtheta)||_2 of the
    final radial density, theta = (n, alpha, smoothingRadius)."""
    import numpy as np
    import torch
    from vlasolve_b200.adjoint import DensityProblem, final_density
    theta = np.array([1.0, 1.0, 0.5])
    dtheta = np.array([0.05, -0.02, 0.03])
    out = {"workload": "pldf_1024x1024x512", "steps": nsteps, "checkpoint_every": K,
           "params": list(LARGE_PARAMS), "theta": theta.tolist(),
           "loss": "||rho - rho_target||_2, rho_target at theta + " + str(dtheta.tolist())}
    t_all = time.perf_counter()
    free0, total = torch.cuda.mem_get_info()
    t0 = time.perf_counter()
    p = DensityProblem(LARGE, precision="fp32", nsteps=nsteps, checkpoint_every=K,
                       params=LARGE_PARAMS)
    s = p.solver
    s.set_init_params(**dict(zip(LARGE_PARAMS, map(float, theta))))
    s.sync()
    out["setup_s"] = time.perf_counter() - t0
    out["cells"] = s.nr * s.nu * s.nj
    out["grid"] = [s.nr, s.nu, s.nj]
    fwd_bytes = s.device_bytes()
    # plain forward, device time on the solver's stream
    stream = torch.cuda.ExternalStream(s.stream_ptr())
    s.step(3)
    s.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step(nsteps)
    e1.record(stream)
    s.sync()
    ms = e0.elapsed_time(e1)
    out["forward_ms_per_step"] = ms / nsteps
    out["value"] = out["cells"] * nsteps / (ms * 1e-3)
    out["unit"] = "cell updates/s"
    s.set_profiling(True)
    s.step(5)
    prof = s.profile_read()
    s.set_profiling(False)
    out["kernels_ms_per_step"] = {k: v[0] / 5 for k, v in prof.items()}
    # adjoint
    target = p.run(theta + dtheta)
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    t1 = time.perf_counter()
    rho = final_density(th, p)
    s.sync()
    t2 = time.perf_counter()
    L = torch.linalg.norm(rho - torch.as_tensor(target))
    L.backward()
    s.sync()
    t3 = time.perf_counter()
    free1, _ = torch.cuda.mem_get_info()
    # the step adjoint alone (recomputation included, initial-state map
    # excluded): one more backward pass with the same seed
    dbins = np.zeros(s.nr)
    dbins[:-1] = (rho.detach().numpy() - target) / np.linalg.norm(rho.detach().numpy() - target)
    dbins[:-1] /= s.shell_volumes()
    s.sync()
    ta = time.perf_counter()
    e0.record(stream)
    s.adjoint_backward(dbins)
    e1.record(stream)
    s.sync()
    out["step_adjoint_wall_s"] = time.perf_counter() - ta
    out["step_adjoint_s"] = e0.elapsed_time(e1) * 1e-3  # device time on the solver stream
    out["step_adjoint_ms_per_step"] = 1e3 * out["step_adjoint_s"] / nsteps
    out["adjoint_over_forward"] = out["step_adjoint_ms_per_step"] / out["forward_ms_per_step"]
    out["inner_every_used"] = s.adjoint_inner_used()
    # per-kernel device times of a 4-step backward pass (3 recomputed forward
    # steps and 4 transposed steps)
    s.adjoint_forward(4, 4)
    s.set_profiling(True)
    s.adjoint_backward(dbins)
    prof = s.profile_read()
    s.set_profiling(False)
    out["adjoint_pass_4_steps_kernel_ms"] = {k: v[0] for k, v in prof.items() if v[1]}
    out["grad"] = th.grad.numpy().tolist()
    out["loss_value"] = float(L.detach())
    out["forward_checkpointed_s"] = t2 - t1
    out["backward_s"] = t3 - t2
    out["hbm_gb"] = {"step_handle_forward": fwd_bytes / 1e9,
                     "step_handle_with_adjoint": s.device_bytes() / 1e9,
                     "device_used_after_backward": (total - free1) / 1e9,
                     "device_used_before": (total - free0) / 1e9}
    p.close()
    del p
    # gradient of the FP32-storage adjoint against the FP64 adjoint, 257 x 257 x 128
    grads, rhos = {}, {}
    for prec in ("fp64", "fp32"):
        q = DensityProblem(LARGE_SUB, precision=prec, nsteps=nsteps, checkpoint_every=K,
                           params=LARGE_PARAMS)
        if prec == "fp64":
            tgt = q.run(theta + dtheta)
        th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
        rq = final_density(th, q)
        rhos[prec] = rq.detach().numpy().copy()
        Lq = torch.linalg.norm(rq - torch.as_tensor(tgt))
        Lq.backward()
        grads[prec] = th.grad.numpy().copy()
        q.close()
    # the loss differences rho - rho_target, which are 1e-2 of rho, so the FP32
    # storage's error in rho reaches the gradient amplified by
    # ||rho|| / ||rho - rho_target||
    rho_rel = float(np.linalg.norm(rhos["fp32"] - rhos["fp64"]) / np.linalg.norm(rhos["fp64"]))
    resid_rel = float(np.linalg.norm(rhos["fp64"] - tgt) / np.linalg.norm(rhos["fp64"]))
    out["subsample"] = {"workload": "pldf_256x256x128", "grad_fp64": grads["fp64"].tolist(),
                        "grad_fp32": grads["fp32"].tolist(),
                        "fp32_vs_fp64_rel": float(np.max(np.abs(grads["fp32"] - grads["fp64"]))
                                                  / np.max(np.abs(grads["fp64"]))),
                        "rho_fp32_vs_fp64_rel": rho_rel,
                        "residual_over_rho": resid_rel,
                        "amplified_rho_error": rho_rel / resid_rel}
    out["seconds"] = time.perf_counter() - t_all
    return out


def adjoint_kernels_block(grid, nsteps, precision):
    """Per-kernel device times of one backward pass of `nsteps` steps
    (checkpoint every nsteps) on the PLDF case of the large block at grid
    (N_r - 1, N_u - 1, N_J): the recomputed forward steps and the transposed
    steps, divided by nsteps.  A first backward pass builds the inverse
    footpoint map and is not timed."""
    import numpy as np
    from vlasolve_b200 import VlasovSolver21Spline
    s = VlasovSolver21Spline(dict(LARGE, Pres=grid[0], Ures=(grid[1], grid[2])),
                             precision=precision)
    s.adjoint_forward(nsteps, nsteps)
    dbins = np.cos(0.01 * np.arange(s.nr))
    s.adjoint_backward(dbins)
    s.set_profiling(True)
    s.adjoint_backward(dbins)
    prof = s.profile_read()
    s.set_profiling(False)
    out = {"workload": "pldf_%dx%dx%d" % tuple(grid), "grid": [s.nr, s.nu, s.nj],
           "precision": precision, "steps": nsteps,
           "kernel_ms_per_step": {k: v[0] / nsteps for k, v in prof.items() if v[1]}}
    s.close()
    return out


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = dict(WORKLOAD)
    model, ncores = cpu_info()
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference binary oracle/_ref/vlasolve was not built"}))
        return
    # each timed "step" is one reference step on the full grid; the run is
    # bounded to a few minutes of host time
    steps = max(1, min(args.steps, args.ref_max_steps))
    v, t, n = run_reference(w, steps, ncores)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell updates/s",
            "n_gpus": args.gpus, "steps": n, "warmup": 0, "ms_per_step": 1e3 * t / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic Hernquist distribution function)",
            "config": config_json(w, "fp64"),
            "cpu_baseline": {"value": v, "unit": "cell updates/s", "cores": ncores,
                             "kind": "reference",
                             "sample": f"{n} steps (of {args.steps} requested) of the full "
                                       f"grid, {model}"},
            "e2e": {"value": v, "unit": "cell updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp32all", "fp64"])
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--ref-max-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the 2000-step drift comparison of the precisions")
    ap.add_argument("--accuracy-steps", type=int, default=2000)
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint gradient check and timing")
    ap.add_argument("--adjoint-steps", type=int, default=500)
    ap.add_argument("--adjoint-every", type=int, default=50)
    ap.add_argument("--kernels", action="store_true",
                    help="with --quick: also report per-kernel event times")
    ap.add_argument("--quick", action="store_true",
                    help="timing of the chosen precision only (for profiler runs)")
    ap.add_argument("--workload", default=WORKLOAD_NAME, choices=sorted(WORKLOADS))
    ap.add_argument("--large", action="store_true",
                    help="only the 1025 x 1025 x 512 PLDF forward + adjoint block")
    ap.add_argument("--large-steps", type=int, default=1000)
    ap.add_argument("--large-every", type=int, default=100)
    ap.add_argument("--adjoint-kernels", metavar="PRES,NU,NJ",
                    help="only the per-kernel times of a backward pass on this PLDF grid")
    ap.add_argument("--adjoint-kernel-steps", type=int, default=4)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        reference_arm(args)
    elif args.adjoint_kernels:
        grid = [int(x) for x in args.adjoint_kernels.split(",")]
        print(json.dumps({"adjoint_kernels": adjoint_kernels_block(
            grid, args.adjoint_kernel_steps, args.precision)}), flush=True)
    elif args.large:
        print(json.dumps({"large": large_block(args.large_steps, args.large_every)}), flush=True)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
