"""The hand-written adjoint of the step against central finite differences of
full forward runs (FP64), against the FP64 adjoint (FP32 modes), and its
checkpointing invariances.

Loss: L(theta) = sum_r (rho_r(theta) - rho*_r)^2, rho the radial density of
the final state and rho* the same forward run at theta + (0.05, -0.02, 0.03),
theta = (R0, alpha, smoothingRadius) of the UDF profile."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

THETA = np.array([2.0, 0.5, 0.5])
DTHETA = np.array([0.05, -0.02, 0.03])
FD_STEP = 1e-4
FD_RTOL = 1e-5       # adjoint vs central differences, FP64
FP32_RTOL = 1e-3     # FP32-storage adjoints vs the FP64 adjoint


def cfg(pres=32, ures=(24, 8), dt=0.02):
    return {"type": "UDF", "Pmin": 0.01, "Pmax": 25.0, "Pres": pres,
            "Pscale": "logarithmic", "Umin": (-2.0, 0.0), "Umax": (2.0, 1.6),
            "Ures": ures, "Uscale": ("linear", "quadratic"), "dt": dt}


def problem(precision="fp64", nsteps=12, K=5, **kw):
    from vlasolve_b200.adjoint import DensityProblem
    return DensityProblem(cfg(**kw), precision=precision, nsteps=nsteps, checkpoint_every=K)


def loss_and_grad(p, target):
    from vlasolve_b200.adjoint import final_density
    th = torch.tensor(THETA, dtype=torch.float64, requires_grad=True)
    rho = final_density(th, p)
    L = ((rho - torch.as_tensor(target)) ** 2).sum()
    L.backward()
    return float(L.detach()), th.grad.numpy().copy()


def test_adjoint_matches_central_differences():
    p = problem()
    target = p.run(THETA + DTHETA)
    L0, g = loss_and_grad(p, target)
    assert L0 > 0
    fd = np.zeros(3)
    for k in range(3):
        tp, tm = THETA.copy(), THETA.copy()
        tp[k] += FD_STEP
        tm[k] -= FD_STEP
        Lp = np.sum((p.run(tp) - target) ** 2)
        Lm = np.sum((p.run(tm) - target) ** 2)
        fd[k] = (Lp - Lm) / (2 * FD_STEP)
    err = np.abs(g - fd) / np.max(np.abs(fd))
    assert np.all(err <= FD_RTOL), (g, fd, err)


@pytest.mark.parametrize("precision", ["fp32", "fp32all"])
def test_fp32_adjoint_matches_fp64_adjoint(precision):
    p64 = problem("fp64")
    target = p64.run(THETA + DTHETA)
    _, g64 = loss_and_grad(p64, target)
    p32 = problem(precision)
    _, g32 = loss_and_grad(p32, target)
    err = np.abs(g32 - g64) / np.max(np.abs(g64))
    assert np.all(err <= FP32_RTOL), (g32, g64, err)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_initial_state_contraction_on_the_device_matches_the_host_grids(precision):
    """vls_adjoint_init_dot (the grids of theta +- h made and contracted with
    dL/df0 on the device, the chain values on the host) against the same
    contractions of the host-made initial states (vls_init_profile) on the
    host, for each parameter; and VLS_ESTATE before a backward pass."""
    from vlasolve_b200 import _lib
    p = problem(precision)
    target = p.run(THETA + DTHETA)
    rho = p.run(THETA)
    with pytest.raises(_lib.VlsError) as e:
        p.solver.adjoint_init_dot(dict(zip(p.params, THETA)), dict(zip(p.params, THETA)))
    assert e.value.code == _lib.VLS_ESTATE
    dbins = np.zeros(p.solver.nr)
    dbins[:-1] = (rho - target) / p.vol
    df0, dch0 = p.solver.adjoint_backward(dbins)
    for k in range(len(p.params)):
        h = p.ic_step * max(1.0, abs(THETA[k]))
        tp, tm = THETA.copy(), THETA.copy()
        tp[k] += h
        tm[k] -= h
        dg, dc = p.solver.adjoint_init_dot(dict(zip(p.params, tp)), dict(zip(p.params, tm)))
        fp, cp = p.initial_state(tp)
        fm, cm = p.initial_state(tm)
        want_g = float(np.vdot(df0, fp - fm))
        want_c = float(np.vdot(dch0, cp - cm))
        assert abs(dg - want_g) <= 1e-7 * abs(want_g), (k, dg, want_g)
        assert abs(dc - want_c) <= 1e-7 * abs(want_c) + 1e-300, (k, dc, want_c)


@pytest.mark.parametrize("K", [1, 4, 12])
def test_checkpoint_interval_does_not_change_gradient(K):
    p_ref = problem(K=5)
    target = p_ref.run(THETA + DTHETA)
    _, g_ref = loss_and_grad(p_ref, target)
    _, g = loss_and_grad(problem(K=K), target)
    np.testing.assert_allclose(g, g_ref, rtol=1e-10, atol=1e-14 * np.max(np.abs(g_ref)))


@pytest.mark.parametrize("inner", [1, 2, 3])
def test_second_level_checkpoints_do_not_change_gradient(inner):
    """Segments of 5 steps split into sub-segments of `inner` steps (the last
    one shorter for 2 and 3) give the gradient of the one-level pass."""
    p_ref = problem(K=5)
    target = p_ref.run(THETA + DTHETA)
    _, g_ref = loss_and_grad(p_ref, target)
    assert p_ref.solver.adjoint_inner_used() == 0
    p = problem(K=5)
    p.solver.adjoint_set_inner(inner)
    _, g = loss_and_grad(p, target)
    assert p.solver.adjoint_inner_used() == inner
    np.testing.assert_allclose(g, g_ref, rtol=1e-10, atol=1e-14 * np.max(np.abs(g_ref)))
    # after a backward pass the handle holds the final state of the forward
    # run (vjp re-initialised this FP64 handle for the initial-state map, so
    # run the forward again first)
    s = p.solver
    p.run(THETA)
    f_final = s.f
    s.adjoint_backward(np.linspace(0.0, 1.0, s.nr))
    np.testing.assert_array_equal(s.f, f_final)


def test_device_bytes_counts_the_adjoint_buffers():
    """vls_device_bytes: at least the grid, coefficients and footpoints after
    set-up; it grows by the checkpoints, stash and FP64 arrays of the adjoint."""
    p = problem(K=5)
    s = p.solver
    cells = s.nr * s.nu * s.nj
    before = s.device_bytes()
    assert before >= 3 * 8 * cells  # f, G, C in FP64 at least
    p.run(THETA)
    s.adjoint_backward(np.linspace(0.0, 1.0, s.nr))
    after = s.device_bytes()
    # 3 checkpoints + final state + 5 stashed states + lam, Cb, Gb (FP64)
    assert after >= before + (3 + 1 + 5) * 8 * cells + 3 * 8 * cells


def test_second_level_rejects_negative_spacing():
    from vlasolve_b200._lib import VlsError
    p = problem()
    with pytest.raises(VlsError):
        p.solver.adjoint_set_inner(-1)


def test_backward_restores_final_state_and_repeats():
    p = problem()
    p.run(THETA)
    s = p.solver
    f_final = s.f
    dbins = np.linspace(0.0, 1.0, s.nr)
    a, ca = s.adjoint_backward(dbins)
    np.testing.assert_array_equal(s.f, f_final)
    b, cb = s.adjoint_backward(dbins)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-14 * np.max(np.abs(a)))
    np.testing.assert_allclose(ca, cb, rtol=1e-12, atol=1e-14 * max(np.max(np.abs(ca), initial=0), 1e-300))
    # linear in the seed
    c, _ = s.adjoint_backward(2.0 * dbins)
    np.testing.assert_allclose(c, 2.0 * a, rtol=1e-12, atol=1e-14 * np.max(np.abs(a)))


def test_adjoint_rejects_nolinking_and_missing_forward():
    from vlasolve_b200 import VlasovSolver21Spline
    from vlasolve_b200._lib import VlsError
    c = dict(cfg(), noLinking=1)
    s = VlasovSolver21Spline(c)
    with pytest.raises(VlsError):
        s.adjoint_forward(3, 1)
    s2 = VlasovSolver21Spline(cfg())
    with pytest.raises(VlsError):
        s2.adjoint_backward(np.zeros(s2.nr))


def test_reinitialising_a_stepped_handle_restores_the_initial_state():
    """vls_init_profile after steps gives the same grid and chain values as
    on a fresh handle (the ring position restarts first)."""
    from vlasolve_b200 import VlasovSolver21Spline
    fresh = VlasovSolver21Spline(cfg())
    s = VlasovSolver21Spline(cfg())
    s.step(7)
    s.init_profile()
    np.testing.assert_array_equal(s.f, fresh.f)
    np.testing.assert_array_equal(s.chains()["val"], fresh.chains()["val"])
    s.step(3)
    fresh.step(3)
    np.testing.assert_array_equal(s.f, fresh.f)


def test_chunked_adjoint_lines_match_one_thread_per_line():
    """The chunked-register transposed solves against the one-thread-per-line
    kernels (the segment prefilter layout selects those for both
    directions)."""
    p_ref = problem("fp64")
    target = p_ref.run(THETA + DTHETA)
    _, g_ref = loss_and_grad(p_ref, target)
    from vlasolve_b200.adjoint import DensityProblem
    p = DensityProblem(cfg(), precision="fp64", nsteps=12, checkpoint_every=5,
                       layout={"prefilter": "segment"})
    assert p.solver.layout()["prefilter"] == "segment"
    _, g = loss_and_grad(p, target)
    np.testing.assert_allclose(g, g_ref, rtol=1e-10)


def test_chunked_adjoint_lines_of_1025_vertices():
    """The same on lines of 1025 vertices in both directions (70-chunk u
    lines, and r lines in the 4-line blocks of the longest layout), cell by
    cell on dL/df0."""
    from vlasolve_b200 import VlasovSolver21Spline
    c = cfg(pres=1024, ures=(1024, 4), dt=0.01)
    out = []
    for layout in (None, {"prefilter": "segment"}):
        s = VlasovSolver21Spline(c, precision="fp64", layout=layout)
        assert s.f.shape == (4, 1025, 1025)
        s.adjoint_forward(3, 3)
        df0, _ = s.adjoint_backward(np.cos(0.01 * np.arange(s.nr)))
        out.append(np.asarray(df0).copy())
        s.close()
    assert np.max(np.abs(out[1])) > 0
    np.testing.assert_allclose(out[0], out[1], rtol=0, atol=1e-10 * np.max(np.abs(out[1])))


def _kbuf_solver(precision):
    """A small grid with delayed-kernel chains (kernel radius at the third r
    vertex) and footpoints far enough to leave the drift strips."""
    from vlasolve_b200 import VlasovSolver21Spline
    c = dict(cfg(pres=40, ures=(28, 10)), kernelBufferSize=2)
    return VlasovSolver21Spline(c, precision=precision)


def _loss(s, f, chv, nsteps, dbins):
    """L = <dbins, bins(f_N)>: the radial bins after nsteps steps from (f, chv)."""
    s.f = f
    s.set_chain_values(chv)
    s.step(nsteps)
    return float(np.dot(dbins, s.moments()[0]))


def test_adjoint_random_directions_match_central_differences():
    """Cell by cell rather than through three parameters: for seeded random
    directions v over the initial grid and w over the initial chain values,
    <dL/df0, v> + <dL/dchain0, w> equals the central difference
    (L(f0 + h v, c0 + h w) - L(f0 - h v, c0 - h w)) / 2h of FP64 forward runs
    (h = 1e-5), to 1e-6 relative.  The grid has chains, so the ring buffers'
    transposes and the chain tails' gathers enter every direction."""
    nsteps, K = 7, 3
    s = _kbuf_solver("fp64")
    f0, c0 = s.f, s.chains()["val"].copy()
    assert len(c0) > 0
    rng = np.random.default_rng(20261203)
    dbins = rng.standard_normal(s.nr)
    s.f = f0
    s.set_chain_values(c0)
    s.adjoint_forward(nsteps, K)
    df0, dch = s.adjoint_backward(dbins)
    df0 = np.asarray(df0).reshape(f0.shape)
    h = 1e-5
    for trial in range(3):
        v = f0 * rng.standard_normal(f0.shape)
        w = c0 * rng.standard_normal(c0.shape)
        pred = float(np.sum(df0 * v) + np.dot(dch, w))
        Lp = _loss(s, f0 + h * v, c0 + h * w, nsteps, dbins)
        Lm = _loss(s, f0 - h * v, c0 - h * w, nsteps, dbins)
        fd = (Lp - Lm) / (2 * h)
        print(f"direction {trial}: adjoint {pred:.12e} fd {fd:.12e}")
        assert abs(pred - fd) <= 1e-6 * abs(fd), (trial, pred, fd)
    # the chain part alone, so that a wrong ring transpose cannot hide behind
    # the much larger grid part.  Its derivative is ~1e-9 of L, below the
    # rounding noise of a difference at h = 1e-5; L depends on the chain
    # values almost linearly (only through their tiny share of the mass), so
    # the central difference takes hc = 0.5
    hc = 0.5
    w = c0 * rng.standard_normal(c0.shape)
    pred = float(np.dot(dch, w))
    fd = (_loss(s, f0, c0 + hc * w, nsteps, dbins) -
          _loss(s, f0, c0 - hc * w, nsteps, dbins)) / (2 * hc)
    print(f"chains only: adjoint {pred:.12e} fd {fd:.12e}")
    assert abs(pred - fd) <= 1e-6 * abs(fd), (pred, fd)


@pytest.mark.parametrize("nj", [72, 136])
def test_adjoint_on_grids_past_the_l2(nj):
    """Grids of 513 x 509 x nj vertices (150 and 284 MB of FP64 adjoint
    field), whose FP32 handles take the entry-ordered gather (16 node rows
    per thread at nj = 72, 32 at nj = 136; the FP64 cell-ordered gather
    takes 32 rows per warp at both): a seeded random direction over every cell
    against central differences of FP64 runs (1e-6 relative), and the
    FP32-storage transpose against the FP64 one on every cell (1e-4 of the
    largest)."""
    from vlasolve_b200 import VlasovSolver21Spline
    c = cfg(pres=512, ures=(508, nj), dt=0.01)
    nsteps = 2
    s = VlasovSolver21Spline(c, precision="fp64")
    f0, c0 = s.f, s.chains()["val"].copy()
    assert f0.shape == (nj, 509, 513)
    rng = np.random.default_rng(20261204 + nj)
    dbins = rng.standard_normal(s.nr)
    s.adjoint_forward(nsteps, nsteps)
    df0, _ = s.adjoint_backward(dbins)
    df0 = np.asarray(df0).reshape(f0.shape)
    v = f0 * rng.standard_normal(f0.shape)
    pred = float(np.sum(df0 * v))
    h = 1e-5
    fd = (_loss(s, f0 + h * v, c0, nsteps, dbins) -
          _loss(s, f0 - h * v, c0, nsteps, dbins)) / (2 * h)
    print(f"adjoint {pred:.12e} fd {fd:.12e}")
    assert abs(pred - fd) <= 1e-6 * abs(fd), (pred, fd)
    s.close()
    s32 = VlasovSolver21Spline(c, precision="fp32")
    s32.adjoint_forward(nsteps, nsteps)
    d32, _ = s32.adjoint_backward(dbins)
    d32 = np.asarray(d32).reshape(f0.shape)
    s32.close()
    assert np.max(np.abs(d32 - df0)) <= 1e-4 * np.max(np.abs(df0))


def test_fp32_adjoint_matches_fp64_adjoint_cell_by_cell():
    """The FP32-storage handle's transposed step (packed footpoint words)
    against the FP64 handle's (FP64 fractions) on every cell of
    dL/df0 and every chain element: the two differ only by the FP32 rounding
    of the forward states they linearise around."""
    out = []
    for prec in ("fp64", "fp32"):
        s = _kbuf_solver(prec)
        s.adjoint_forward(7, 3)
        dbins = np.cos(0.3 * np.arange(s.nr, dtype=np.float64))
        df0, dch = s.adjoint_backward(dbins)
        out.append((np.asarray(df0).ravel().copy(), dch.copy()))
    (a0, ac), (b0, bc) = out
    assert np.max(np.abs(a0)) > 0 and ac.size > 0
    assert np.max(np.abs(b0 - a0)) <= 1e-4 * np.max(np.abs(a0))
    assert np.max(np.abs(bc - ac)) <= 1e-4 * max(np.max(np.abs(ac)), 1e-300)


def _backward_twice(precision):
    s = _kbuf_solver(precision)
    s.adjoint_forward(7, 3)
    dbins = np.cos(0.3 * np.arange(s.nr, dtype=np.float64))
    out = []
    for _ in range(2):
        df0, dch = s.adjoint_backward(dbins)
        out.append((np.asarray(df0).copy(), dch.copy()))
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gather_drift_transpose_is_deterministic(precision):
    """Two backward passes through the gather give the same bits."""
    (a0, ac), (b0, bc) = _backward_twice(precision)
    np.testing.assert_array_equal(a0, b0)
    np.testing.assert_array_equal(ac, bc)


def _set_footpoints(s, fp, rI):
    import ctypes
    i32, u8 = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint8)
    d = ctypes.POINTER(ctypes.c_double)
    assert s._L.vls_set_footpoints(
        s._h, rI.ctypes.data_as(i32), fp["rF"].ctypes.data_as(d),
        fp["uI"].ctypes.data_as(i32), fp["uF"].ctypes.data_as(d),
        fp["out"].ctypes.data_as(u8), fp["driftR"].ctypes.data_as(d)) == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_inverse_map_follows_new_footpoints(precision):
    """vls_set_footpoints after a backward pass: the next gather uses the
    inverse map of the new footpoints (base columns moved by one), as a
    handle that never saw the old footpoints does."""
    dbins = np.cos(0.3 * np.arange(41, dtype=np.float64))
    s = _kbuf_solver(precision)
    f0, c0 = s.f, s.chains()["val"].copy()
    s.adjoint_forward(4, 2)
    s.adjoint_backward(dbins)
    fp = s.footpoints()
    rI = fp["rI"].copy()
    move = (fp["out"] == 0) & (rI >= 1)
    rI[move] -= 1
    _set_footpoints(s, fp, rI)
    s.f = f0
    s.set_chain_values(c0)
    s.adjoint_forward(4, 2)
    g0, gc = s.adjoint_backward(dbins)
    t = _kbuf_solver(precision)
    _set_footpoints(t, fp, rI)
    t.adjoint_forward(4, 2)
    a0, ac = t.adjoint_backward(dbins)
    assert np.max(np.abs(np.asarray(g0) - np.asarray(a0))) == 0.0
    np.testing.assert_array_equal(gc, ac)
