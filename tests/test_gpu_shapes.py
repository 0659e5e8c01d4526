"""Grid shapes that exercise the chunking of the register-resident prefilter
(one chunk, a last chunk of one row, exactly full chunks, odd sizes) and the
drift's strip boxes against the oracle, for every prefilter / drift layout
and all three precisions."""

import numpy as np
import pytest

from oracle.vls_oracle import Oracle

pytestmark = pytest.mark.gpu

# (grid.Pres, grid.Ures[0]) -> N_r = Pres + 1 r vertices, N_u = Ures0 + 1 u
# vertices; chunks of 31 rows: 4 -> 1 chunk, 32 -> 2 chunks with a last
# chunk of one row, 62 -> 2 full chunks, 63 -> 3 chunks, 94 -> 4 chunks;
# chunks of 23 rows: 47 -> 2 full chunks and one row, 69 -> 3 full chunks;
# chunks of 19 rows: 47 -> 2 full chunks and 9 rows;
# 701 u vertices: lines too long for 16-line blocks of 15-row chunks, which
# take 23-row chunks by default; 1001 r vertices: FP64 rows whose four
# persistent r-solve tiles exceed a block's shared memory (the plain kernel
# takes them); 2048 r or u vertices, the largest grids a handle takes: lines
# beyond the register layouts, whose shared-memory segment tiles hold half
# the usual lines in FP64
SHAPES = [(3, 31), (31, 32), (32, 61), (61, 62), (62, 93), (93, 3), (150, 40),
          (46, 68), (20, 700), (1000, 8), (2047, 8), (8, 2047)]

FP64_TOL = 1e-12
FP32_L2 = 2e-6
FP32_MAX = 1e-5


def cfg_for(pres, ures0):
    return {"type": "UDF", "Pmin": 0.01, "Pmax": 25.0, "Pres": pres,
            "Pscale": "logarithmic", "Umin": (-2.0, 0.0), "Umax": (2.0, 1.6),
            "Ures": (ures0, 6), "Uscale": ("linear", "quadratic"), "dt": 0.02}


# layout of each kernel choice (vls_layout_desc): the defaults, the
# shared-memory segment prefilter with the windowed drift, and each drift
# kind forced (a strip that does not fit falls back to windows)
IMPLS = {
    "default": None,
    "segment-window": {"prefilter": "segment", "drift": "window"},
    "window": {"drift": "window"},
    "strip2": {"drift": "strip2"},
    "strip1": {"drift": "strip1"},
}


@pytest.fixture(params=sorted(IMPLS))
def impl(request):
    return request.param


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "%dx%d" % (s[0] + 1, s[1] + 1))
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32all"])
def test_shape_steps_match_oracle(shape, precision, impl):
    from vlasolve_b200 import VlasovSolver21Spline
    cfg = cfg_for(*shape)
    s = VlasovSolver21Spline(cfg, precision=precision, layout=IMPLS[impl])
    o = Oracle(cfg)
    for _ in range(3):
        s.step(1)
        o.step(1)
        ref = o.f
        got = s.f
        scale = np.max(np.abs(ref))
        if precision == "fp64":
            assert np.max(np.abs(got - ref)) <= FP64_TOL * scale
        else:
            l2 = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert l2 <= FP32_L2, l2
            assert np.max(np.abs(got - ref)) <= FP32_MAX * scale
