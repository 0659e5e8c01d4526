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


def test_far_cell_layout_keeps_the_adjoint(monkeypatch):
    """With the far-cell pass (packed words FP_FAR + list index) the drift's
    transpose reads the original footpoints from the far list."""
    p_ref = problem("fp32")
    target = p_ref.run(THETA + DTHETA)
    _, g_ref = loss_and_grad(p_ref, target)
    monkeypatch.setenv("VLS_FAR", "1")
    p = problem("fp32")
    _, g = loss_and_grad(p, target)
    np.testing.assert_allclose(g, g_ref, rtol=1e-6)


@pytest.mark.parametrize("layout", ["long", "short"])
def test_other_adjoint_line_layouts_keep_the_gradient(layout, monkeypatch):
    """The chunk layouts the transposed solves take besides the default ones:
    the r layout of lines too long for the default (1025 rows), forced here
    on short lines ("long"), and the 16-line u layout ("short")."""
    p_ref = problem("fp64")
    target = p_ref.run(THETA + DTHETA)
    _, g_ref = loss_and_grad(p_ref, target)
    monkeypatch.setenv("VLS_ADJ_RC", layout)
    for prec in ("fp64", "fp32"):
        p = problem(prec)
        _, g = loss_and_grad(p, target)
        if prec == "fp64":
            np.testing.assert_allclose(g, g_ref, rtol=1e-10)
        else:
            assert np.all(np.abs(g - g_ref) <= FP32_RTOL * np.max(np.abs(g_ref)))


def test_chunked_adjoint_lines_match_one_thread_per_line(monkeypatch):
    """The chunked-register transposed solves against the one-thread-per-line
    kernels (VLS_PREFILTER=segment selects those for both directions)."""
    p_ref = problem("fp64")
    target = p_ref.run(THETA + DTHETA)
    _, g_ref = loss_and_grad(p_ref, target)
    monkeypatch.setenv("VLS_PREFILTER", "segment")
    p = problem("fp64")
    _, g = loss_and_grad(p, target)
    np.testing.assert_allclose(g, g_ref, rtol=1e-10)


def _solver_backward(precision, env, monkeypatch, far=False):
    from vlasolve_b200 import VlasovSolver21Spline
    if far:
        monkeypatch.setenv("VLS_FAR", "1")
    s = VlasovSolver21Spline(cfg(pres=40, ures=(28, 10)), precision=precision)
    s.adjoint_forward(7, 3)
    dbins = np.cos(0.3 * np.arange(s.nr, dtype=np.float64))
    out = []
    for mode in env:
        if mode:
            monkeypatch.setenv("VLS_DRIFT_ADJ", mode)
        else:
            monkeypatch.delenv("VLS_DRIFT_ADJ", raising=False)
        df0, dch = s.adjoint_backward(dbins)
        out.append((df0.copy(), dch.copy()))
    return out


@pytest.mark.parametrize("precision,far", [("fp64", False), ("fp32", False), ("fp32", True)])
def test_gather_drift_transpose_matches_atomic_scatter(precision, far, monkeypatch):
    """The drift transposed as a gather over the inverse footpoint map against
    the scatter with FP64 atomics: the same sums in another order, on every
    cell of dL/df0 and every ring slot of dL/d(chains)."""
    (g0, gc), (a0, ac) = _solver_backward(precision, ["", "atomic"], monkeypatch, far)
    assert np.max(np.abs(a0)) > 0
    np.testing.assert_allclose(g0, a0, rtol=1e-11, atol=1e-13 * np.max(np.abs(a0)))
    assert gc.size == ac.size and gc.size > 0
    np.testing.assert_allclose(gc, ac, rtol=1e-11, atol=1e-13 * max(np.max(np.abs(ac)), 1e-300))


def test_gather_drift_transpose_is_deterministic(monkeypatch):
    """Two backward passes through the gather give the same bits."""
    (a0, ac), (b0, bc) = _solver_backward("fp32", ["", ""], monkeypatch)
    np.testing.assert_array_equal(a0, b0)
    np.testing.assert_array_equal(ac, bc)


def test_inverse_map_follows_new_footpoints(monkeypatch):
    """vls_set_footpoints after a backward pass: the next gather uses the
    inverse map of the new footpoints (base columns moved by one), checked
    against the atomic scatter, which reads the footpoints directly."""
    import ctypes
    from vlasolve_b200 import VlasovSolver21Spline
    s = VlasovSolver21Spline(cfg(pres=40, ures=(28, 10)), precision="fp32")
    dbins = np.cos(0.3 * np.arange(s.nr, dtype=np.float64))
    s.adjoint_forward(4, 2)
    monkeypatch.delenv("VLS_DRIFT_ADJ", raising=False)
    s.adjoint_backward(dbins)
    fp = s.footpoints()
    rI = fp["rI"].copy()
    move = (fp["out"] == 0) & (rI >= 1)
    rI[move] -= 1
    i32, u8 = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint8)
    d = ctypes.POINTER(ctypes.c_double)
    assert s._L.vls_set_footpoints(
        s._h, rI.ctypes.data_as(i32), fp["rF"].ctypes.data_as(d),
        fp["uI"].ctypes.data_as(i32), fp["uF"].ctypes.data_as(d),
        fp["out"].ctypes.data_as(u8), fp["driftR"].ctypes.data_as(d)) == 0
    s.adjoint_forward(4, 2)
    g0, gc = s.adjoint_backward(dbins)
    monkeypatch.setenv("VLS_DRIFT_ADJ", "atomic")
    a0, ac = s.adjoint_backward(dbins)
    np.testing.assert_allclose(g0, a0, rtol=1e-11, atol=1e-13 * np.max(np.abs(a0)))
    np.testing.assert_allclose(gc, ac, rtol=1e-11, atol=1e-13 * max(np.max(np.abs(ac)), 1e-300))


@pytest.mark.parametrize("far", [False, True])
def test_entry_ordered_gather_matches_cell_ordered_gather(far, monkeypatch):
    """FP32 handles: the gather over entry-ordered values and packed words
    against the gather that reads lam and the footpoints through each
    entry's cell index (with the far-cell layout too)."""
    from vlasolve_b200 import VlasovSolver21Spline
    if far:
        monkeypatch.setenv("VLS_FAR", "1")
    s = VlasovSolver21Spline(cfg(pres=40, ures=(28, 10)), precision="fp32")
    s.adjoint_forward(7, 3)
    dbins = np.cos(0.3 * np.arange(s.nr, dtype=np.float64))
    monkeypatch.delenv("VLS_DRIFT_ADJ", raising=False)
    monkeypatch.setenv("VLS_ADJ_GATHER_PERM", "0")
    a0, ac = s.adjoint_backward(dbins)
    monkeypatch.setenv("VLS_ADJ_GATHER_PERM", "1")
    p0, pc = s.adjoint_backward(dbins)
    np.testing.assert_allclose(p0, a0, rtol=1e-13, atol=1e-15 * np.max(np.abs(a0)))
    np.testing.assert_allclose(pc, ac, rtol=1e-13, atol=1e-15 * max(np.max(np.abs(ac)), 1e-300))
