import glob
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a)")
    config.addinivalue_line("markers", "slow: long CPU run, enabled by VLS_SLOW_TESTS=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("VLS_SLOW_TESTS") == "1":
        return
    skip = pytest.mark.skip(reason="set VLS_SLOW_TESTS=1 to run")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


def cfg_from_args(args, dt):
    """Option dict (oracle / solver names) from the reference command line a
    golden case was generated with."""
    a = [str(x) for x in args]
    cfg = {"dt": float(dt)}
    i = 0
    while i < len(a):
        k = a[i][1:]
        vals = []
        i += 1
        while i < len(a) and not (a[i].startswith("-") and not a[i][1:2].isdigit()):
            vals.append(a[i])
            i += 1
        key = k.split(".")[1]
        if key in ("Umin", "Umax", "gap"):
            cfg[key] = tuple(float(v) for v in vals)
        elif key == "Ures":
            cfg[key] = tuple(int(v) for v in vals)
        elif key == "Uscale":
            cfg[key] = tuple(vals)
        elif key in ("Pres", "kernelBufferSize", "noLinking"):
            cfg[key] = int(vals[0])
        elif key in ("Pscale", "type", "kernelType"):
            cfg[key] = vals[0]
        else:
            cfg[key] = float(vals[0])
    return cfg


def golden_cases(full_only=None):
    out = []
    for fn in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        g = np.load(fn)
        full = any(k.startswith("f_") for k in g.files)
        if full_only is None or full == full_only:
            out.append(os.path.basename(fn)[:-4])
    return out


def load_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    return g, cfg_from_args(g["args"], g["dt"])
