"""GPU parity: the CUDA pair step against the CPU oracle, through the C-ABI.

Tolerances (the parity bar of the plain form): global relative error ||X_gpu - X_oracle|| / ||X_oracle||
<= 1e-12 for positions and velocities, and the per-particle maximum
max|X_gpu - X_oracle| / max|X_oracle| <= 1e-12 at the workloads' step lengths, against
both the FP64 oracle (the reference's CPU path) and its quad-precision evaluation (the
step without rounding noise).  At the reference fixture's dt = 1 the per-particle
maximum is 1e-11 (see test_oracle.py: one pericentre pair is ill-conditioned in the
reference algorithm itself).
"""
import numpy as np
import pytest

import oracle
from bia_3d_gpu_b200 import (BIASolver, METHOD_ALG, METHOD_RKF, METHOD_UNIVERSAL, default_config,
                             find_dxyuv_kernel, initial, invariance_gpu)
from conftest import max_rel_err, rel_err

pytestmark = pytest.mark.gpu


def gpu_run(cuda, state, eps, dt, nsteps, q=None, method=METHOD_ALG, deterministic=1,
            graph=False, disp=False, **cfg_fields):
    t = cuda.tensor(state, dtype=cuda.float64, device="cuda").contiguous()
    qt = cuda.tensor(q, dtype=cuda.float64, device="cuda") if q is not None else None
    cfg = default_config(eps_th=eps, dt=dt, method=method, deterministic=deterministic, **cfg_fields)
    d = cuda.zeros_like(t) if disp else None
    with BIASolver() as s:
        if graph:
            stats = s.run(t, cfg, nsteps, q=qt, graph=True)
        else:
            stats = None
            for _ in range(nsteps):
                stats = s.step(t, cfg, q=qt, disp=d)
        s.stream.synchronize()
    out = t.cpu().numpy()
    return (out, stats, d.cpu().numpy()) if disp else (out, stats)


def oracle_run(state, eps, dt, nsteps, q=None, method=1, quad=False, relerr=0.0, abserr=1e-16):
    s = state
    st = None
    for _ in range(nsteps):
        s, _, st = oracle.bia_step(s, eps, dt, method=method, q=q, quad=quad, relerr=relerr, abserr=abserr)
    return s, st


CLASSES = ("hyperbola", "ellipse", "parabola", "universal", "degenerate", "rkf")


def total_pairs(st):
    return sum(st[k] for k in CLASSES)


def assert_parity(gpu, ref, tol_max=1e-12):
    assert rel_err(gpu[:3], ref[:3]) <= 1e-12
    assert rel_err(gpu[3:], ref[3:]) <= 1e-12
    assert max_rel_err(gpu[:3], ref[:3]) <= tol_max
    assert max_rel_err(gpu[3:], ref[3:]) <= tol_max


def test_gravity_ball_matches_oracle(cuda):
    s, eps = initial.gravity_ball(300, seed=21)
    g, st = gpu_run(cuda, s, eps, 1e-4, 5)
    r, rst = oracle_run(s, eps, 1e-4, 5)
    assert_parity(g, r)
    assert total_pairs(st) == 300 * 299 // 2
    # the universal-variable routing is a threshold on FP64 quantities: allow a flip or two
    for k in ("hyperbola", "ellipse", "universal"):
        assert abs(st[k] - rst[k]) <= 2, k
    assert st["nonfinite"] == 0


@pytest.mark.parametrize("case", ["gravity", "coulomb", "plummer"])
def test_matches_quad_precision_step(cuda, case):
    """Against the exact step (oracle in __float128, FP64 state between steps)."""
    if case == "gravity":
        (s, eps), q, dt = initial.gravity_ball(200, seed=51), None, 1e-4
    elif case == "coulomb":
        s, eps, q = initial.coulomb_cube(200, seed=52)
        dt = 1e-5
    else:
        (s, eps), q, dt = initial.plummer(200, seed=53), None, 1e-4
    g, _ = gpu_run(cuda, s, eps, dt, 2, q=q)
    r, _ = oracle_run(s, eps, dt, 2, q=q, quad=True)
    assert_parity(g, r, tol_max=1e-13)


def test_universal_method_matches_quad(cuda):
    """BIA_METHOD_UNIVERSAL (every pair by Stumpff-function universal variables)."""
    s, eps, q = initial.coulomb_cube(200, seed=54)
    g, st = gpu_run(cuda, s, eps, 1e-5, 2, q=q, method=METHOD_UNIVERSAL)
    r, _ = oracle_run(s, eps, 1e-5, 2, q=q, quad=True)
    assert st["universal"] == 200 * 199 // 2
    assert_parity(g, r, tol_max=1e-13)
    o, _ = oracle_run(s, eps, 1e-5, 2, q=q, method=2)
    assert_parity(g, o, tol_max=1e-13)


def test_coulomb_mixed_classes_match_oracle(cuda):
    """Repulsive pairs on hyperbolae, attractive pairs mostly on ellipses."""
    s, eps, q = initial.coulomb_cube(400, seed=22, dmin=1e-3)
    g, st = gpu_run(cuda, s, eps, 1e-5, 3, q=q)
    r, rst = oracle_run(s, eps, 1e-5, 3, q=q)
    assert st["ellipse"] > 1000 and st["hyperbola"] > 1000
    assert abs(st["ellipse"] - rst["ellipse"]) <= 2
    assert_parity(g, r)


def test_plummer_matches_oracle(cuda):
    s, eps = initial.plummer(384, seed=23)
    g, _ = gpu_run(cuda, s, eps, 1e-4, 4)
    r, _ = oracle_run(s, eps, 1e-4, 4)
    assert_parity(g, r)


@pytest.mark.parametrize("relerr", [0.0, 1e-12])
def test_rkf_mode_matches_oracle(cuda, relerr):
    """Per-pair RKF45 with the reference's tolerances (relerr 0, abserr 1e-16,
    bia/find_dXYUV_RKF.f90:4) and with the scale configuration's relative tolerance 1e-12
    (abserr kept at 1e-16): the same accepted step counts as the oracle, and its step."""
    s, eps, q = initial.coulomb_cube(96, seed=24, dmin=1e-2)
    g, st = gpu_run(cuda, s, eps, 1e-5, 2, q=q, method=METHOD_RKF, rkf_relerr=relerr, rkf_abserr=1e-16)
    r, rst = oracle_run(s, eps, 1e-5, 2, q=q, method=0, relerr=relerr, abserr=1e-16)
    assert st["rkf"] == 96 * 95 // 2 and st["rkf_steps"] == rst["rkf_steps"]
    assert_parity(g, r)


def test_reference_fixture_through_bia_step(cuda, golden, golden_ic):
    """The .BIA record of the reference (dt = 1, eps_th = -6e-7) via the whole-step API."""
    g, st, disp = gpu_run(cuda, golden_ic, -6e-7, 1.0, 1, disp=True)
    ref_disp = golden["bia_disp_aos"].reshape(-1, 6).T
    ref = golden_ic + ref_disp
    assert_parity(g, ref, tol_max=1e-11)
    assert np.abs(disp[3:] - ref_disp[3:]).max() <= 1e-14
    o, _, _ = oracle.bia_step(golden_ic, -6e-7, 1.0)
    assert_parity(g, o, tol_max=1e-11)


def test_reference_fixture_through_dropin_row_entry(cuda, golden, golden_ic):
    """bia/bia.f90:128-204 GPU branch restated over the drop-in find_dxyuv_kernel_."""
    s = golden_ic
    n = s.shape[1]
    X, Y, Z, U, V, W = [np.ascontiguousarray(s[k]) for k in range(6)]
    acc = [np.zeros(n) for _ in range(6)]
    rel = np.zeros(6 * n)
    out = np.zeros(6 * n)
    for I in range(1, n + 1):
        i = I - 1
        for k, a in enumerate((X, Y, Z, U, V, W)):
            rel[k::6] = a[i] - a
        st = find_dxyuv_kernel(1, n, I, -6e-7, 1.0, 18, *acc, rel, out)
        assert st == 0
        assert np.all(out[: 6 * I] == 0)
        acc[0][i] += U[i] * 1.0
        acc[1][i] += V[i] * 1.0
        acc[2][i] += W[i] * 1.0
    disp = np.stack(acc)
    ref_disp = golden["bia_disp_aos"].reshape(-1, 6).T
    assert_parity(s + disp, s + ref_disp, tol_max=1e-11)


def test_deterministic_mode_is_bitwise_reproducible(cuda):
    s, eps, q = initial.coulomb_cube(700, seed=25)
    a, _ = gpu_run(cuda, s, eps, 1e-5, 2, q=q)
    b, _ = gpu_run(cuda, s, eps, 1e-5, 2, q=q)
    assert np.array_equal(a, b)


def test_atomic_mode_matches_deterministic(cuda):
    s, eps = initial.gravity_ball(500, seed=26)
    a, _ = gpu_run(cuda, s, eps, 1e-4, 2, deterministic=1)
    b, _ = gpu_run(cuda, s, eps, 1e-4, 2, deterministic=0)
    assert rel_err(b, a) <= 1e-15


def test_graph_run_equals_stepwise(cuda):
    s, eps = initial.plummer(600, seed=27)
    a, sa = gpu_run(cuda, s, eps, 1e-4, 4, graph=True)
    b, _ = gpu_run(cuda, s, eps, 1e-4, 4, graph=False)
    assert np.array_equal(a, b)
    assert total_pairs(sa) == 4 * 600 * 599 // 2


def test_host_buffer_run_equals_device_run(cuda):
    s, eps, q = initial.coulomb_cube(300, seed=28)
    h = s.copy()
    cfg = default_config(eps_th=eps, dt=1e-5)
    with BIASolver() as solver:
        solver.run_host(h, cfg, 3, q=q)
    d, _ = gpu_run(cuda, s, eps, 1e-5, 3, q=q, graph=True)
    assert np.array_equal(h, d)


@pytest.mark.parametrize("n", [1, 2, 3, 31, 32, 33, 64, 65, 97])
def test_ragged_sizes(cuda, n):
    s, eps = initial.gravity_ball(n, seed=100 + n)
    g, st = gpu_run(cuda, s, eps, 1e-3, 2)
    r, _ = oracle_run(s, eps, 1e-3, 2)
    assert_parity(g, r)
    assert total_pairs(st) == n * (n - 1) // 2


def test_degenerate_and_parabolic_pairs(cuda):
    """g = 0 (cold start), r parallel to g, and an exactly parabolic pair."""
    s = np.zeros((6, 4))
    s[:3, 0] = (0, 0, 0)
    s[:3, 1] = (4, 3, 0)        # |r| = 5 from particle 0
    s[3:, 1] = (0, 0, 1)        # |g| = 1, W = 1 + 2 eps / 5 = 0 with eps = -2.5
    s[:3, 2] = (-3, 0, 0)
    s[3:, 2] = (-0.5, 0, 0)     # r parallel to g relative to particle 0
    s[:3, 3] = (0, 7, 1)        # at rest with particle 0: g = 0
    eps = -2.5
    g, st = gpu_run(cuda, s, eps, 0.01, 1)
    r, rst = oracle_run(s, eps, 0.01, 1)
    assert st["parabola"] == rst["parabola"] == 1
    assert st["degenerate"] == rst["degenerate"] >= 2
    assert st["nonfinite"] == 0
    assert_parity(g, r)


def test_cold_start_all_degenerate(cuda):
    s, eps = initial.cold_ball(200, seed=29)
    g, st = gpu_run(cuda, s, eps, 5e-5, 1)
    r, _ = oracle_run(s, eps, 5e-5, 1)
    assert st["degenerate"] == 200 * 199 // 2
    assert_parity(g, r)


def test_nonfinite_input_is_reported(cuda):
    s, eps = initial.gravity_ball(40, seed=30)
    s[0, 5] = np.nan
    _, st = gpu_run(cuda, s, eps, 1e-4, 1)
    assert st["nonfinite"] >= 39


@pytest.mark.parametrize("method", [METHOD_UNIVERSAL, METHOD_RKF, 3])
def test_nonfinite_pairs_counted_exactly(cuda, method):
    """The universal-variable, RKF45 and learned walks test each warp-block's sums instead of
    each pair and count the pairs again only where a sum is not finite: one NaN particle
    among 40 gives exactly its 39 pairs."""
    s, eps = initial.gravity_ball(40, seed=30)
    s[0, 5] = np.nan
    t = cuda.tensor(s, device="cuda")
    with BIASolver() as solver:
        solver.load_heads()
        st = solver.step(t, default_config(eps_th=eps, dt=1e-4, method=method))
    assert st["nonfinite"] == 39


def test_invalid_arguments_raise(cuda):
    from bia_3d_gpu_b200 import BiaError
    t = cuda.zeros((6, 8), dtype=cuda.float64, device="cuda")
    with BIASolver() as s:
        with pytest.raises(BiaError):
            s.step(t, default_config(itr=0))
        with pytest.raises(BiaError):
            s.step(t, default_config(method=7))
    with pytest.raises(TypeError):
        BIASolver().step(t.float(), default_config())


def test_invariance_matches_oracle(cuda, golden_ic):
    s, eps, q = initial.coulomb_cube(1000, seed=31)
    t = cuda.tensor(s, device="cuda")
    qt = cuda.tensor(q, device="cuda")
    with BIASolver() as solver:
        got = solver.invariance(t, eps, q=qt)
    ref = oracle.invariance(s, eps, q=q, quad=True)
    for k in ("KE", "PE"):
        assert abs(got[k] / ref[k] - 1) <= 1e-13, k
    for k in ("Ua", "Va", "Wa", "Xa", "Ya", "Za", "Lx", "Ly", "Lz"):
        assert abs(got[k] - ref[k]) <= 1e-12 * max(1.0, abs(ref[k])), k
    # drop-in invariance_gpu_ on the fixture (bia/bia.f90:67-68 call shape)
    X, Y, Z, U, V, W = [np.ascontiguousarray(golden_ic[k]) for k in range(6)]
    vals = invariance_gpu(golden_ic.shape[1], -6e-7, X, Y, Z, U, V, W)
    refq = oracle.invariance(golden_ic, -6e-7, quad=True)
    for name, v in zip(("KE", "PE", "Lx", "Ly", "Lz", "Ua", "Va", "Wa", "Xa", "Ya", "Za"), vals):
        assert abs(v - refq[name]) <= 1e-13 * max(1.0, abs(refq[name])), name


@pytest.mark.parametrize("method", [METHOD_ALG, METHOD_UNIVERSAL])
def test_near_radial_pair_far_above_start_guess(cuda, method):
    """Two particles a few microns apart closing at 543 of their 563 relative speed: the
    universal-variable start guess lies far above the root on a hyperbolic branch, where
    plain Newton crawls.  The step must converge and match the quad-precision oracle."""
    s = np.zeros((6, 2))
    s[:3, 0] = [-4.064577389883972e-06, 7.483568417843145e-06, -9.615181365080216e-06]
    s[3:, 0] = [95.72878999340595, -231.02576430088004, 504.2191870037502]
    g, st = gpu_run(cuda, s, -2.0, 1e-5, 1, method=method)
    r, _ = oracle_run(s, -2.0, 1e-5, 1, method=method, quad=True)
    assert st["nonconverged"] == 0 and st["nonfinite"] == 0
    assert st["iter_universal"] < 60
    assert_parity(g, r)


def test_phase_locked_kernel_modes_agree(cuda):
    """N = 8192 takes the phase-locked ALG kernel (more than two 32-warp CTAs per SM):
    deterministic mode is bitwise reproducible, atomic mode agrees to rounding, and
    sampled particles match the oracle."""
    s, eps, q = initial.coulomb_cube(8192, seed=27)
    a, st, da = gpu_run(cuda, s, eps, 1e-5, 1, q=q, disp=True)
    b, _ = gpu_run(cuda, s, eps, 1e-5, 1, q=q)
    c, _ = gpu_run(cuda, s, eps, 1e-5, 1, q=q, deterministic=0)
    assert np.array_equal(a, b)
    assert rel_err(c, a) <= 1e-15
    assert total_pairs(st) == 8192 * 8191 // 2 and st["ellipse"] > 0 and st["universal"] > 0
    sel = np.random.default_rng(3).choice(8192, 24, replace=False)
    ref = oracle.particle_disp(s, eps, 1e-5, sel, q=q)
    got = da[:, sel].T
    assert np.abs(got[:, :3] - ref[:, :3]).max() <= 1e-12 * np.abs(s[:3]).max()
    assert np.abs(got[:, 3:] - ref[:, 3:]).max() <= 1e-12 * np.abs(s[3:]).max()


def test_autotune_picks_a_shape_and_keeps_results(cuda):
    """The autotuner times the ALG pair-kernel shapes on the state without changing it and
    keeps the fastest; every shape computes the same per-block sums in the same order, so
    the step is bitwise the same before and after tuning."""
    s, eps, q = initial.coulomb_cube(8192, seed=28)
    t = cuda.tensor(s, device="cuda")
    qt = cuda.tensor(q, device="cuda")
    cfg = default_config(eps_th=eps, dt=1e-5)
    with BIASolver() as solver:
        a = t.clone()
        solver.step(a, cfg, q=qt)
        var, ms = solver.autotune(t, cfg, q=qt)
        assert cuda.equal(t, cuda.tensor(s, device="cuda"))   # state untouched
        assert var in (0, 1, 2) and len(ms) == 3 and all(v > 0 for v in ms.values())
        assert min(ms, key=ms.get) == ("tiles8", "phase32_lane", "phase32")[var]
        b = t.clone()
        st = solver.step(b, cfg, q=qt)
        assert st["hyperbola"] + st["ellipse"] + st["universal"] + st["parabola"] + st["degenerate"] == 8192 * 8191 // 2
    assert cuda.equal(a, b)


@pytest.mark.parametrize("det", [True, False])
def test_alg_shapes_are_bitwise_equal_on_mixed_classes(cuda, det):
    """The three ALG pair-kernel shapes give bitwise the same step on a system of mixed
    classes (hyperbolae, ellipses, near-unit eccentricity): 8-warp CTAs with per-lane class
    loops, and phase-locked 16- and 32-warp CTAs whose class loops pack the lanes' last pairs
    of a class into shared turns (each row and each column still adds its pairs in the same
    order).  Atomic mode is compared to rounding.  The step matches the oracle."""
    n = 3000
    s, eps, q = initial.coulomb_cube(n, seed=31)
    cfg = default_config(eps_th=eps, dt=1e-5)
    cfg.deterministic = 1 if det else 0
    outs = []
    with BIASolver() as solver:
        qt = cuda.tensor(q, device="cuda")
        for shape in ("tiles8", "phase32_lane", "phase32"):
            solver.set_shape(METHOD_ALG, n, shape, deterministic=det)
            t = cuda.tensor(s, device="cuda")
            st = solver.step(t, cfg, q=qt)
            assert st["hyperbola"] > 0 and st["ellipse"] > 0 and st["universal"] > 0
            outs.append(t.cpu().numpy())
        solver.set_shape(METHOD_ALG, n, None, deterministic=det)
    for o in outs[1:]:
        if det:
            assert np.array_equal(outs[0], o)
        else:
            assert rel_err(o, outs[0]) <= 1e-15
    ref, _, _ = oracle.bia_step(s, eps, 1e-5, q=q)
    assert_parity(outs[0], ref)


def test_set_shape_validates_and_pins(cuda):
    """bia_context_set_shape refuses shapes out of range and methods with one shape, and a
    pinned shape (or the default restored) gives the same step bitwise."""
    from bia_3d_gpu_b200 import capi
    s, eps, q = initial.coulomb_cube(600, seed=32)
    cfg = default_config(eps_th=eps, dt=1e-5)
    outs = []
    with BIASolver() as solver:
        lib = capi.lib()
        assert lib.bia_context_set_shape(solver._ctx, METHOD_ALG, 1, 600, 3) == capi.BIA_ERR_INVALID_ARGUMENT
        assert lib.bia_context_set_shape(solver._ctx, METHOD_ALG, 1, 600, -2) == capi.BIA_ERR_INVALID_ARGUMENT
        assert lib.bia_context_set_shape(solver._ctx, METHOD_UNIVERSAL, 1, 600, 0) == capi.BIA_ERR_INVALID_ARGUMENT
        assert lib.bia_context_set_shape(solver._ctx, METHOD_ALG, 1, 0, 0) == capi.BIA_ERR_INVALID_ARGUMENT
        assert lib.bia_context_set_shape(None, METHOD_ALG, 1, 600, 0) == capi.BIA_ERR_INVALID_ARGUMENT
        qt = cuda.tensor(q, device="cuda")
        for shape in (None, "phase32_lane", None):
            solver.set_shape(METHOD_ALG, 600, shape)
            t = cuda.tensor(s, device="cuda")
            solver.step(t, cfg, q=qt, stats=False)
            outs.append(t.cpu().numpy())
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


def test_bounded_device_wait_reports_timeout(cuda):
    """A device-side wait that nothing completes gives up after its limit and the step API
    reports BIA_ERR_DEVICE_TIMEOUT; the context then runs a normal step."""
    import ctypes
    from bia_3d_gpu_b200 import capi
    s, eps = initial.gravity_ball(64, seed=29)
    with BIASolver() as solver:
        st = capi.lib().bia_selftest_wait_timeout(solver._ctx)
        assert st == capi.BIA_ERR_DEVICE_TIMEOUT
        t = cuda.tensor(s, device="cuda")
        stats = solver.step(t, default_config(eps_th=eps, dt=1e-4))
        assert stats["nonfinite"] == 0 and stats["timeouts"] == 0
    r, _, _ = oracle.bia_step(s, eps, 1e-4)
    assert_parity(t.cpu().numpy(), r)


def test_bia_driver_reproduces_reference_record(cuda, golden, golden_ic, tmp_path):
    """bia/bia.f90 through the driver: the .bbb record in, the .BIA record (t, dX..dW) and
    particle 1's text line out, against the reference's own run."""
    from bia_3d_gpu_b200 import driver, records
    bbb = tmp_path / "0001332_10^0.bbb"
    records.write_bbb(bbb, [golden_ic])
    stats, inv = driver.run_bia(bbb, tmp_path / "0001332_10^0.BIA", tmp_path / "BIA_10^0.0001332",
                                eps_th=-6e-7, time_end=1.0)
    assert stats[0]["nonfinite"] == 0 and inv["KE"] > 0
    (t, d), = records.read_timed(tmp_path / "0001332_10^0.BIA")
    ref_disp = golden["bia_disp_aos"].reshape(-1, 6).T
    assert t == 1.0
    assert_parity(golden_ic + d, golden_ic + ref_disp, tol_max=1e-11)
    line = (tmp_path / "BIA_10^0.0001332").read_text().splitlines()[0]
    vals = [float(line[23 + 24 * k:23 + 24 * (k + 1)]) for k in range(6)]
    assert np.abs(np.array(vals) - golden["bia_p1"][1:]).max() <= 1e-13


def test_universal_solver_against_reference_equations_near_unit_eccentricity(cuda):
    """The universal-variable solver (every pair of BIA_METHOD_UNIVERSAL and of the learned
    form) against the reference's own conic equations (bia/find_hyperbola.f90,
    bia/find_ellipse.f90) evaluated in quad precision, on attractive pairs drawn in
    0.1 < |e^2 - 1| < 0.3: there ALG still takes the reference's equations and they are well
    conditioned, so the quad oracle is their exact step.  One 2-particle system per pair, as an
    ensemble; steps long enough to move the pairs through a good part of their orbits."""
    from bia_3d_gpu_b200 import METHOD_UNIVERSAL
    rng = np.random.default_rng(77)
    eps, dt = -1.0, 0.3
    pairs = []
    while len(pairs) < 200:
        r = rng.standard_normal(3)
        r *= rng.uniform(0.5, 2.0) / np.linalg.norm(r)
        g = rng.standard_normal(3) * rng.uniform(0.2, 2.0)
        rm = np.linalg.norm(r)
        E = g @ g + 2 * eps / rm
        L = np.cross(r, g)
        e2m1 = E * (L @ L) / eps ** 2
        if 0.1 < abs(e2m1) < 0.3:
            pairs.append((r, g))
    states = []
    for r, g in pairs:
        states.append(np.array([[r[0] / 2, -r[0] / 2], [r[1] / 2, -r[1] / 2], [r[2] / 2, -r[2] / 2],
                                [g[0] / 2, -g[0] / 2], [g[1] / 2, -g[1] / 2], [g[2] / 2, -g[2] / 2]]))
    host = np.concatenate(states, axis=1)
    whole = cuda.tensor(host, device="cuda")
    with BIASolver() as solver:
        ens = solver.ensemble([2] * len(pairs), [eps] * len(pairs))
        st = ens.run(whole, default_config(dt=dt, method=METHOD_UNIVERSAL), 1, graph=False)
        solver.stream.synchronize()
        ens.close()
    got = whole.cpu().numpy()
    assert st["nonfinite"] == 0 and st["nonconverged"] == 0
    worst = 0.0
    for k, (r, g) in enumerate(pairs):
        d = got[:, 2 * k] - host[:, 2 * k]
        h = d.copy()
        h[:3] -= host[3:, 2 * k] * dt  # the interaction part of particle i's displacement
        ref, rst = oracle.pair_halfdisp(r, g, eps, dt, method=1, quad=True)
        assert rst["hyperbola"] + rst["ellipse"] == 1  # the reference's equations, not the universal path
        worst = max(worst, np.linalg.norm(h[:3] - ref[:3]) / np.linalg.norm(ref[:3]),
                    np.linalg.norm(h[3:] - ref[3:]) / np.linalg.norm(ref[3:]))
    print(f"universal solver vs the reference's equations in quad, 200 pairs at 0.1 < |e^2-1| < 0.3: "
          f"worst relative error {worst:.2e}")
    assert worst <= 1e-12
