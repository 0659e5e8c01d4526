"""Generate the golden vectors under tests/golden/ from the reference binary.

The reference binary is built from the reference sources by
``oracle/build_ref.sh`` into ``oracle/_ref/vlasolve`` (FP64, OpenMP, no MPI).
Every case runs it with ``-threads_per_node 1`` (the reference's moment sums
depend on the OpenMP thread count at the 1e-12 level; one thread fixes the
order) and records:

* f at selected steps, read from its NDfield snapshots (whole grid for the
  small cases; a seeded sample of cells plus per-J-slice sums for the
  full-size configurations, whose grids are too large to commit);
* the ``statistics.txt`` rows;
* the delayed-kernel chains (cell, R, U, values) from the restart file written
  at step 0 and from the final restart file;
* two .vls restart files of the smallest case, byte for byte (``restart``);
* one NDfield snapshot of the smallest case, byte for byte (``ndfield``).

Usage:  python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(REPO, "oracle", "_ref", "vlasolve")

SAMPLE_SEED = 20261203
N_SAMPLE = 4096


def case(name, args, steps, save_steps, full_f=True, dt=None):
    return dict(name=name, args=args, steps=steps, save_steps=save_steps,
                full_f=full_f, dt=dt)


def _grid(pres, ures, jres, pmin, pmax, umin, umax, jmin, jmax,
          pscale="logarithmic", uscale="linear", jscale="quadratic"):
    return ["-grid.Pmin", str(pmin), "-grid.Pmax", str(pmax), "-grid.Pres", str(pres),
            "-grid.Pscale", pscale,
            "-grid.Umin", str(umin), str(jmin), "-grid.Umax", str(umax), str(jmax),
            "-grid.Ures", str(ures), str(jres), "-grid.Uscale", uscale, jscale]


CASES = [
    case("udf_tiny", ["-init.type", "UDF"] + _grid(16, 16, 8, 0.01, 25, -2, 2, 0, 1.6),
         10, [0, 1, 2, 5, 10], dt=0.005),
    case("udf_rect_kbuf", ["-init.type", "UDF", "-solver.kernelBufferSize", "2"]
         + _grid(24, 20, 6, 0.01, 25, -2, 2, 0, 1.6), 6, [0, 1, 6], dt=0.01),
    case("udf_nolink", ["-init.type", "UDF", "-solver.noLinking", "1"]
         + _grid(16, 16, 8, 0.01, 25, -2, 2, 0, 1.6), 5, [0, 1, 5], dt=0.005),
    case("udf_gap", ["-init.type", "UDF", "-init.gap", "0.5", "1.0", "-init.alpha", "0.8"]
         + _grid(20, 18, 6, 0.01, 25, -2, 2, 0, 1.6), 4, [0, 1, 4], dt=0.005),
    case("plummer_small", ["-init.type", "Plummer"] + _grid(20, 16, 8, 0.01, 25, -3, 3, 0, 2),
         5, [0, 1, 5], dt=0.005),
    case("hernquist_small", ["-init.type", "Hernquist"]
         + _grid(20, 16, 8, 0.01, 50, -3, 3, 0, 3), 5, [0, 1, 5], dt=0.0025),
    case("hernquist_aniso", ["-init.type", "Hernquist", "-init.Ra", "1.5"]
         + _grid(18, 14, 6, 0.01, 50, -3, 3, 0, 3), 3, [0, 3], dt=0.0025),
    case("pldf_small", ["-init.type", "PLDF", "-init.alpha", "1", "-init.eta", "0.1",
                        "-init.n", "1", "-init.smoothingRadius", "0.5"]
         + _grid(20, 16, 8, 0.01, 200, -3, 3, 0, 1.6), 5, [0, 1, 5], dt=0.005),
    case("plummer_linr", ["-init.type", "Plummer"]
         + _grid(20, 16, 8, 0.05, 20, -3, 3, 0, 2, pscale="linear"),
         4, [0, 1, 4], dt=0.01),
    # reflective kernel (kernelType reflective): footpoints that cross the
    # kernel radius R_Val[0] are reflected there (vlasovSolver21.hxx:343-377,
    # :434); with kernelBufferSize > 0 the reference terminates during set-up
    # (:389-391), so the radius stays at the first vertex
    case("udf_reflect", ["-init.type", "UDF", "-solver.kernelType", "reflective"]
         + _grid(20, 18, 6, 0.01, 25, -2, 2, 0, 1.6), 4, [0, 1, 4], dt=0.02),
    # lines of 1025 vertices along r and along v_r (the layouts the
    # 1024 x 1024 x 512 PLDF configuration takes), three J slices (sampled)
    case("pldf_1025", ["-init.type", "PLDF", "-init.alpha", "1", "-init.eta", "0.1",
                       "-init.n", "1", "-init.smoothingRadius", "0.5"]
         + _grid(1024, 1024, 3, 0.01, 200, -3, 3, 0, 1.6), 2, [0, 1, 2], full_f=False,
         dt=0.005),
    # the north-star configurations at their full sizes (sampled)
    case("udf_cfg1", ["-init.type", "UDF"] + _grid(200, 200, 200, 0.01, 25, -2, 2, 0, 1.6),
         10, [0, 1, 10], full_f=False, dt=0.005),
    case("plummer_cfg2", ["-init.type", "Plummer"] + _grid(256, 256, 128, 0.01, 25, -3, 3, 0, 2),
         3, [0, 1, 3], full_f=False, dt=0.005),
    case("hernquist_cfg3", ["-init.type", "Hernquist"]
         + _grid(512, 512, 256, 0.01, 50, -3, 3, 0, 3), 2, [0, 1, 2], full_f=False,
         dt=0.0025),
]


def read_nd(path):
    """Data block of an NDfield snapshot (NDfield.hxx:308-363): the payload
    is the last record of the file, framed by 4-byte markers."""
    with open(path, "rb") as fh:
        b = fh.read()
    # tag record (4 + 16 + 4 bytes), then the header record: int marker,
    # 80-byte comment, ndims, dims[...]
    off = 4 + 16 + 4 + 4 + 80
    ndims = struct.unpack_from("<i", b, off)[0]
    dims = struct.unpack_from("<%di" % ndims, b, off + 4)
    n = int(np.prod(dims))
    data = np.frombuffer(b[len(b) - 4 - 8 * n: len(b) - 4], dtype="<f8")
    return dims, data


def read_chains(path):
    """Kernel chains of a .vls restart file (sphericalKernel::write,
    sphericalKernel.hxx:88-106; cellChain::write cellChain.hxx:91-98;
    dummyCell21::write dummyCell21_vect.hxx:56-63), sorted by cell index."""
    with open(path, "rb") as fh:
        b = fh.read()
    tag = b"KERNEL_CELLS v0.10"
    pos = b.find(tag)
    if pos < 0:
        return None
    pos += len(tag)
    (nsl,) = struct.unpack_from("<q", b, pos); pos += 8
    chains = []
    for _ in range(nsl):
        (n2,) = struct.unpack_from("<q", b, pos); pos += 8
        for _ in range(n2):
            (key,) = struct.unpack_from("<q", b, pos); pos += 8
            (L,) = struct.unpack_from("<q", b, pos); pos += 8
            els = []
            for _ in range(L):
                R, U = struct.unpack_from("<dd", b, pos); pos += 16
                (nv,) = struct.unpack_from("<i", b, pos); pos += 4
                vals = struct.unpack_from("<%dd" % nv, b, pos); pos += 8 * nv
                els.append((R, U, vals[0]))
            chains.append((key, els))
    chains.sort(key=lambda c: c[0])
    cell = np.array([c[0] for c in chains], np.int64)
    ln = np.array([len(c[1]) for c in chains], np.int32)
    R = np.array([e[0] for c in chains for e in c[1]])
    U = np.array([e[1] for c in chains for e in c[1]])
    V = np.array([e[2] for c in chains for e in c[1]])
    return dict(cell=cell, len=ln, R=R, U=U, val=V)


def read_stats(path):
    rows = []
    with open(path) as fh:
        for line in fh:
            if line.startswith("#") or not line.strip():
                continue
            rows.append([float(x) for x in line.split()])
    return np.array(rows)


def run_case(c):
    tmp = tempfile.mkdtemp(prefix="vls_golden_")
    try:
        dt = c["dt"]
        tmax = dt * c["steps"]
        args = [REF_BIN, "-threads_per_node", "1", "-verbose", "0"] + c["args"] + [
            "-solver.dt", repr(dt), "-solver.Tmax", repr(tmax),
            "-solver.statsEvery", "1", "-solver.snapshotEvery", "1",
            "-solver.restartEvery", "100000"]
        if not c["full_f"]:
            args[args.index("-solver.statsEvery") + 1] = "1"
        with open(os.path.join(tmp, "log.txt"), "w") as log:
            subprocess.check_call(args, cwd=tmp, stdout=log, stderr=subprocess.STDOUT)
        out = {"args": np.array(c["args"]), "dt": dt, "steps": c["steps"]}
        snaps = sorted(x for x in os.listdir(tmp) if x.startswith("snapshot_"))
        # snapshot names carry the time with 4 decimals; map by order
        times = [float(x[len("snapshot_"):-3]) for x in snaps]
        order = np.argsort(times)
        snaps = [snaps[i] for i in order]
        rng = np.random.default_rng(SAMPLE_SEED)
        idx = None
        for s in c["save_steps"]:
            dims, data = read_nd(os.path.join(tmp, snaps[s]))
            shape = tuple(reversed(dims))  # [J][u][r]
            out["shape"] = np.array(shape)
            f = data.reshape(shape)
            if c["full_f"]:
                out["f_%d" % s] = f
            else:
                if idx is None:
                    idx = np.sort(rng.choice(f.size, size=N_SAMPLE, replace=False))
                    out["sample_idx"] = idx
                out["fs_%d" % s] = data[idx]
                out["slicesum_%d" % s] = f.reshape(shape[0], -1).sum(axis=1)
        out["stats"] = read_stats(os.path.join(tmp, "statistics.txt"))
        ch0 = read_chains(os.path.join(tmp, "restart_0.0000.vls"))
        finals = [x for x in os.listdir(tmp) if x.startswith("final_")]
        ch1 = read_chains(os.path.join(tmp, finals[0])) if finals else None
        for tagname, ch in (("chain0", ch0), ("chainN", ch1)):
            if ch is None:
                continue
            if not c["full_f"]:
                # keep the chain layout and a sample of values only
                ch = dict(cell=ch["cell"], len=ch["len"],
                          val_head=ch["val"][:512], R_head=ch["R"][:512],
                          U_head=ch["U"][:512], val_sum=np.array([ch["val"].sum()]))
            for k, v in ch.items():
                out["%s_%s" % (tagname, k)] = v
        np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), **out)
        return c["name"], "ok"
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


# .vls restart files of the reference, kept byte for byte: the udf_tiny case
# dumped after step 2 (restartEvery 2) and its final dump after step 3
RESTART_FILES = {"restart_0.0100.vls": "udf_tiny_restart_step2.vls",
                 "final_0.0150.vls": "udf_tiny_final_step3.vls"}


def make_restart_fixtures():
    tmp = tempfile.mkdtemp(prefix="vls_golden_")
    try:
        c = CASES[0]
        args = [REF_BIN, "-threads_per_node", "1", "-verbose", "0"] + c["args"] + [
            "-solver.dt", "0.005", "-solver.Tmax", "0.0125", "-solver.restartEvery", "2",
            "-solver.statsEvery", "-1", "-solver.snapshotEvery", "-1"]
        with open(os.path.join(tmp, "log.txt"), "w") as log:
            subprocess.check_call(args, cwd=tmp, stdout=log, stderr=subprocess.STDOUT)
        for src, dst in RESTART_FILES.items():
            shutil.copyfile(os.path.join(tmp, src), os.path.join(HERE, dst))
        return "restart", "ok"
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


# an NDfield snapshot written by the reference (Save_NDfield, NDfield.hxx:308-363),
# kept byte for byte: the udf_tiny case after one step
NDFIELD_FILE = ("snapshot_0.0050.ND", "udf_tiny_snapshot_step1.ND")


def make_ndfield_fixture():
    tmp = tempfile.mkdtemp(prefix="vls_golden_")
    try:
        c = CASES[0]
        args = [REF_BIN, "-threads_per_node", "1", "-verbose", "0"] + c["args"] + [
            "-solver.dt", "0.005", "-solver.Tmax", "0.005", "-solver.restartEvery", "100000",
            "-solver.statsEvery", "-1", "-solver.snapshotEvery", "1"]
        with open(os.path.join(tmp, "log.txt"), "w") as log:
            subprocess.check_call(args, cwd=tmp, stdout=log, stderr=subprocess.STDOUT)
        shutil.copyfile(os.path.join(tmp, NDFIELD_FILE[0]), os.path.join(HERE, NDFIELD_FILE[1]))
        return "ndfield", "ok"
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main(names):
    if not os.path.exists(REF_BIN):
        sys.exit("reference binary missing: run oracle/build_ref.sh first")
    if not names or "restart" in names:
        print(*make_restart_fixtures(), flush=True)
    if not names or "ndfield" in names:
        print(*make_ndfield_fixture(), flush=True)
    todo = [c for c in CASES if not names or c["name"] in names]
    if not todo:
        return
    with cf.ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 1)) as ex:
        for name, st in ex.map(run_case, todo):
            print(name, st, flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
