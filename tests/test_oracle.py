"""Pins of the CPU oracle against the reference's own outputs and known answers.

The oracle (oracle/bia_oracle.c) restates the reference's CPU path; these tests check
it before it is trusted as the parity reference for the CUDA kernels.  The same source
is also evaluated in __float128 ("quad"): the BIA step without rounding noise, against
which any FP64 implementation's rounding error is measured.  Pins:
  * the committed fixture OUT/0001332_10^0.{bbb,BIA,DIM} (reference run, N = 1332,
    eps_th = -6e-7, dt = 1; tests/golden/make_golden.py converts it);
  * per-branch identities every two-body solve must satisfy (energy W and angular
    momentum L of the planar relative orbit, bia/find_parabola.f90:102-103) and the
    agreement of the analytic branches with the reference's per-pair RKF45.
"""
import numpy as np
import pytest

import oracle
from conftest import max_rel_err, rel_err

EPS_FIX = -6e-7


@pytest.fixture(scope="module")
def fixture_step(golden_ic):
    new, disp, stats = oracle.bia_step(golden_ic, EPS_FIX, 1.0, method=1, itr=18)
    return new, disp, stats


def test_fixture_is_all_hyperbolic(fixture_step):
    _, _, st = fixture_step
    assert st["hyperbola"] == 1332 * 1331 // 2
    assert st["ellipse"] == st["parabola"] == st["degenerate"] == 0


def test_oracle_matches_reference_bia_record(golden, golden_ic, fixture_step):
    """Oracle step vs the reference's .BIA record (its GPU ALG run).

    Tolerance: global relative error <= 1e-12 in positions and velocities (the parity
    bar of the plain form).  The per-particle maximum is looser, 1e-11 of max|X|: a pair
    that starts at pericentre gets its start angle from acos(1 - delta)
    (bia/find_hyperbola.f90:38), whose conditioning ~1/sqrt(delta) turns one ulp into
    ~1e-11 of displacement at dt = 1; the reference's CPU and GPU paths differ there
    by the same amount."""
    new, disp, _ = fixture_step
    ref_disp = golden["bia_disp_aos"].reshape(-1, 6).T
    ref_new = golden_ic + ref_disp
    assert rel_err(new[:3], ref_new[:3]) <= 1e-12
    assert rel_err(new[3:], ref_new[3:]) <= 1e-12
    assert max_rel_err(new[:3], ref_new[:3]) <= 1e-11
    assert max_rel_err(new[3:], ref_new[3:]) <= 1e-13
    # velocity kicks themselves (no drift term), absolute
    assert np.abs(disp[3:] - ref_disp[3:]).max() <= 1e-14


def test_oracle_particle1_text_line(golden, fixture_step):
    """bia/bia.f90:207 writes particle 1's final state as text (17 significant digits)."""
    new, _, _ = fixture_step
    line = golden["bia_p1"]
    assert line[0] == 1.0
    assert np.abs(new[:, 0] - line[1:]).max() <= 1e-13


def test_oracle_vs_dim_reference_run(golden, fixture_step):
    """BIA vs the direct-integration run: a physics-level agreement check
    (bia/bia.f90:261-278).  The reference's own BIA record is at 3.8e-13 / 8.4e-12."""
    new, _, _ = fixture_step
    dim = golden["dim_final_aos"].reshape(-1, 6).T
    assert rel_err(new[:3], dim[:3]) <= 1e-12
    assert rel_err(new[3:], dim[3:]) <= 2e-11


def test_invariance_fp64_vs_quad(golden_ic):
    """Invariance_CPU vs Invariance_QPU on the fixture IC (bia/bia.f90:70-107)."""
    d = oracle.invariance(golden_ic, EPS_FIX)
    q = oracle.invariance(golden_ic, EPS_FIX, quad=True)
    for k in ("KE", "PE"):
        assert abs(d[k] / q[k] - 1) <= 1e-13, k
    for k in ("Ua", "Va", "Wa", "Lx", "Ly", "Lz"):
        assert abs(d[k] - q[k]) <= 1e-12, k


def _orbit_invariants(Y, eps):
    r = np.hypot(Y[0], Y[1])
    W = Y[2] ** 2 + Y[3] ** 2 + 2 * eps / r
    L = Y[0] * Y[3] - Y[1] * Y[2]
    return W, L


def _random_pairs(rng, count, eps, g_scale, r_scale):
    out = []
    for _ in range(count):
        r = rng.standard_normal(3) * r_scale
        g = rng.standard_normal(3) * g_scale
        out.append((r, g))
    return out


@pytest.mark.parametrize("dt", [1e-4, 1e-2, 1.0])
def test_hyperbola_conserves_W_L_and_matches_rkf(dt):
    rng = np.random.default_rng(11)
    eps = -0.01
    n_checked = 0
    for r, g in _random_pairs(rng, 40, eps, 1.0, 1.0):
        _, _, _, YZ, deg = oracle.frame(r, g)
        assert not deg
        W0, L0 = _orbit_invariants(YZ, eps)
        if W0 <= 0:
            continue
        YN, err, it = oracle.find_hyperbola(eps, dt, YZ)
        W1, L1 = _orbit_invariants(YN, eps)
        assert abs(W1 - W0) <= 1e-11 * abs(W0) + 1e-13
        assert abs(L1 - L0) <= 1e-11 * abs(L0) + 1e-14
        YR, _, ier, _ = oracle.find_dxyuv_rkf(eps, dt, YZ)
        assert ier == 0
        assert np.abs(YN - YR).max() <= 1e-9 * max(1.0, np.abs(YZ).max())
        n_checked += 1
    assert n_checked > 20


@pytest.mark.parametrize("dt", [1e-4, 0.05, 0.7])
def test_ellipse_conserves_W_L_and_matches_rkf(dt):
    rng = np.random.default_rng(12)
    eps = -2.0
    n_checked = 0
    for r, g in _random_pairs(rng, 60, eps, 0.7, 1.0):
        _, _, _, YZ, deg = oracle.frame(r, g)
        W0, L0 = _orbit_invariants(YZ, eps)
        if W0 >= 0:
            continue
        YN, err, it = oracle.find_ellipse(eps, dt, YZ)
        W1, L1 = _orbit_invariants(YN, eps)
        assert abs(W1 - W0) <= 1e-10 * abs(W0)
        assert abs(L1 - L0) <= 1e-10 * abs(L0) + 1e-14
        YR, _, ier, _ = oracle.find_dxyuv_rkf(eps, dt, YZ)
        assert ier == 0
        # close approaches amplify the RKF's own error; compare on regular orbits
        if np.hypot(YN[0], YN[1]) > 0.05:
            assert np.abs(YN - YR).max() <= 1e-7 * np.abs(YZ).max()
        n_checked += 1
    assert n_checked > 20


def test_parabola_exact_zero_energy():
    """W == 0 exactly selects find_parabola (bia/bia.f90:160): |r| = 5, |g| = 1,
    eps = -2.5 gives g^2 + 2 eps / r = 0 with no rounding."""
    r = np.array([4.0, 3.0, 0.0])
    g = np.array([0.0, 0.0, 1.0])
    eps = -2.5
    _, _, _, YZ, deg = oracle.frame(r, g)
    assert not deg
    assert np.dot(g, g) + 2 * eps / np.linalg.norm(r) == 0.0
    h, st = oracle.pair_halfdisp(r, g, eps, 0.3)
    assert st["parabola"] == 1
    YN, err, it = oracle.find_parabola(eps, 0.3, YZ)
    W1, L1 = _orbit_invariants(YN, eps)
    W0, L0 = _orbit_invariants(YZ, eps)
    assert abs(W1) <= 1e-14
    assert abs(L1 - L0) <= 1e-13 * abs(L0)
    YR, _, ier, _ = oracle.find_dxyuv_rkf(eps, 0.3, YZ)
    assert np.abs(YN - YR).max() <= 1e-9


def test_pair_antisymmetry_bitwise():
    rng = np.random.default_rng(5)
    for _ in range(50):
        r, g = rng.standard_normal(3), rng.standard_normal(3)
        h1, _ = oracle.pair_halfdisp(r, g, -0.05, 0.01)
        h2, _ = oracle.pair_halfdisp(-r, -g, -0.05, 0.01)
        assert np.array_equal(h1, -h2)


def test_degenerate_pairs_are_radial():
    """Zero relative velocity or r parallel to g: the reference divides by zero
    (bia/bia.f90:295-296); the oracle advances them with the universal-variable solver,
    which agrees with the per-pair RKF45 along the line of motion."""
    eps, dt = -0.5, 0.01
    r = np.array([1.0, 2.0, 2.0])
    h, st = oracle.pair_halfdisp(r, np.zeros(3), eps, dt)
    assert st["degenerate"] == 1
    assert np.all(np.isfinite(h))
    # displacement along r, attraction pulls i toward j: h_x ~ eps/|r|^3 r dt^2 / 4
    expect = eps / 27.0 * r * dt * dt / 4
    assert np.allclose(h[:3], expect, rtol=1e-3)
    h2, st2 = oracle.pair_halfdisp(r, 0.1 * r, eps, dt)
    assert st2["degenerate"] == 1
    assert np.all(np.isfinite(h2))
    assert abs(np.dot(np.cross(h2[:3], r), np.ones(3))) <= 1e-18


def test_rkf_mode_agrees_with_alg_mode_on_fixture_rows(golden_ic):
    """The reference's two pair methods (bia/bia.f90:149-171) agree on the fixture."""
    rows = [0, 100, 1000]
    alg, npairs, _ = oracle.bia_rows(golden_ic, EPS_FIX, 1.0, rows, method=1)
    rkf, _, st = oracle.bia_rows(golden_ic, EPS_FIX, 1.0, rows, method=0)
    assert st["rkf"] == npairs
    scale = np.abs(golden_ic[:3]).max()
    assert np.abs(alg - rkf)[:3].max() <= 1e-12 * scale
    assert np.abs(alg - rkf)[3:].max() <= 1e-12


def test_rows_omp_matches_sequential(golden_ic):
    d1, n1, _ = oracle.bia_rows(golden_ic[:, :200], EPS_FIX, 1.0, np.arange(200), nthreads=1)
    d4, n4, _ = oracle.bia_rows(golden_ic[:, :200], EPS_FIX, 1.0, np.arange(200), nthreads=4)
    assert n1 == n4 == 200 * 199 // 2
    assert np.abs(d1 - d4).max() <= 1e-15


def test_dim_oracle_conserves_energy_small():
    """dim/rkf_kernel.cu's adaptive RKF45 restated: energy drift at round-off level."""
    s, eps = __import__("bia_3d_gpu_b200.initial", fromlist=["x"]).lattice(NL=1, seed=3)
    y0 = np.ascontiguousarray(s.T).reshape(-1)
    eps_dim = -3e-3
    yn, ier, nacc, nde = oracle.dim_rkf(y0, eps_dim, 0.0, 1.0)
    assert ier == 0 and nacc > 0
    e0 = oracle.invariance(s, 2 * eps_dim, quad=True)
    e1 = oracle.invariance(yn.reshape(-1, 6).T, 2 * eps_dim, quad=True)
    assert abs((e1["KE"] + e1["PE"]) / (e0["KE"] + e0["PE"]) - 1) <= 1e-13


# ---- quad-precision evaluation: rounding noise of the FP64 path ----------------------

def test_fixture_fp64_vs_quad_sampled(golden, golden_ic):
    """On the reference fixture (dt = 1) the FP64 path is within 1e-11 of max|X| of
    the exact step on every sampled particle, including the pericentre pair of
    particles 207/1086 (start angle from acos near 1, bia/find_hyperbola.f90:38), and
    the reference's own record (its GPU run) is within the same band."""
    sel = [0, 207, 1086, 557, 1244] + list(range(3, 1332, 97))
    d = oracle.particle_disp(golden_ic, EPS_FIX, 1.0, sel)
    qd = oracle.particle_disp(golden_ic, EPS_FIX, 1.0, sel, quad=True)
    ref = golden["bia_disp_aos"].reshape(-1, 6).T[:, sel].T
    scale = np.abs(golden_ic[:3]).max()
    assert np.abs(d - qd)[:, :3].max() <= 1e-11 * scale
    assert np.abs(ref - qd)[:, :3].max() <= 1e-11 * scale
    assert np.abs(d - qd)[:, 3:].max() <= 1e-14


@pytest.mark.parametrize("case", ["gravity", "coulomb", "plummer"])
def test_fp64_step_within_1e13_of_quad(case):
    """With the near-unit-eccentricity pairs on the universal-variable solver and the
    unconverged iterations re-solved, the FP64 step is within 1e-13 of the exact step."""
    from bia_3d_gpu_b200 import initial
    if case == "gravity":
        (s, eps), q, dt = initial.gravity_ball(160, seed=41), None, 1e-4
    elif case == "coulomb":
        s, eps, q = initial.coulomb_cube(160, seed=42)
        dt = 1e-5
    else:
        (s, eps), q, dt = initial.plummer(160, seed=43), None, 1e-4
    a, _, st = oracle.bia_step(s, eps, dt, q=q)
    b, _, _ = oracle.bia_step(s, eps, dt, q=q, quad=True)
    assert rel_err(a[:3], b[:3]) <= 1e-13 and max_rel_err(a[:3], b[:3]) <= 1e-13
    assert rel_err(a[3:], b[3:]) <= 1e-13 and max_rel_err(a[3:], b[3:]) <= 1e-13


def test_universal_variables_match_quad_classical():
    """Universal-variable solver (FP64) against the classical formulas evaluated in quad:
    agreement to 1e-12 of the displacement itself on random pairs of every class."""
    rng = np.random.default_rng(8)
    worst = 0.0
    for _ in range(300):
        eps = -10 ** rng.uniform(-4, 0.5) * rng.choice([1, 1, -1])
        r = rng.standard_normal(3) * 10 ** rng.uniform(-1, 0.3)
        g = rng.standard_normal(3) * 10 ** rng.uniform(-1.5, 0.5)
        dt = 10 ** rng.uniform(-6, -1.5)
        hq, _ = oracle.pair_halfdisp(r, g, eps, dt, quad=True)
        hu, st = oracle.pair_halfdisp(r, g, eps, dt, method=2)
        assert st["universal"] == 1
        worst = max(worst, np.abs(hu - hq).max() / np.abs(hq).max())
    assert worst <= 1e-12


def test_near_parabolic_bound_pair_regression():
    """A barely bound pair (W = -3.6e-5, eps = -2): the reference's ellipse formulas give a
    displacement of 1e4 in dt = 1e-5; the guarded path matches the exact step."""
    YZ = np.array([0.3191676, 0.61635585, 0.0, 2.40060326])
    eps = -2.0
    r_abs = np.hypot(YZ[0], YZ[1])
    # set |g| so that W = g^2 + 2 eps / r = -3.6e-5
    gm = np.sqrt(-2 * eps / r_abs - 3.6e-5)
    r = np.array([YZ[0], YZ[1], 0.0])
    g = np.array([0.0, gm, 0.0])
    h, st = oracle.pair_halfdisp(r, g, eps, 1e-5)
    hq, _ = oracle.pair_halfdisp(r, g, eps, 1e-5, quad=True)
    hr, _ = oracle.pair_halfdisp(r, g, eps, 1e-5, method=0, quad=True)
    assert st["universal"] == 1
    assert np.abs(h - hq).max() <= 1e-12 * np.abs(hq).max()
    assert np.abs(hq - hr).max() <= 1e-9 * np.abs(hq).max()


def test_unconverged_ellipse_is_resolved():
    """Pair (365, 179) of coulomb_cube(400, seed 22), a bound pair with e close to 1:
    the reference's Kepler Newton starts from xi_2 + delta_ini (bia/find_ellipse.f90:
    125-129) and ends at ITR unconverged with a displacement of order 10.  The raw
    ellipse branch flags it and re-solves Kepler's equation by bisection-safeguarded
    Newton; the whole pair path sends it to the universal-variable solver
    (|e^2 - 1| < 0.1).  Both agree with the quad-precision per-pair RKF45."""
    from bia_3d_gpu_b200 import initial
    s, eps, q = initial.coulomb_cube(400, seed=22, dmin=1e-3)
    r = s[:3, 365] - s[:3, 179]
    g = s[3:, 365] - s[3:, 179]
    e = eps * q[365] * q[179]
    h, st = oracle.pair_halfdisp(r, g, e, 1e-5)
    hr, _ = oracle.pair_halfdisp(r, g, e, 1e-5, method=0, quad=True)
    assert st["universal"] == 1
    assert np.abs(h - hr).max() <= 1e-9 * np.abs(hr).max()
    _, _, _, YZ, _ = oracle.frame(r, g)
    YN, _, it, fb = oracle.find_ellipse(e, 1e-5, YZ, return_fallback=True)
    YR, _, ier, _ = oracle.find_dxyuv_rkf(e, 1e-5, YZ)
    assert fb == 1 and ier == 0
    assert np.abs(YN - YR).max() <= 1e-9 * np.abs(YZ).max()


def test_attractive_hyperbola_bracket_fallback():
    """An attractive hyperbola whose reference iterate leaves (-theta_0, theta_0)
    (bia/find_hyperbola.f90:98-101): the raw hyperbola branch re-solves the time
    equation by bracketed Newton (decreasing in theta for eps < 0) and matches the
    per-pair RKF45; the pair path sends it to the universal-variable solver
    (|e^2 - 1| = 0.03), which matches as well."""
    r = np.array([0.05477136, 0.29190468, 0.0])
    g = np.array([0.0, 4.50440845, 0.0])
    eps, dt = -2.54, 0.0534
    _, _, _, YZ, _ = oracle.frame(r, g)
    YN, _, it, fb = oracle.find_hyperbola(eps, dt, YZ, return_fallback=True)
    YR, _, ier, _ = oracle.find_dxyuv_rkf(eps, dt, YZ)
    assert fb == 1 and ier == 0
    assert np.abs(YN - YR).max() <= 1e-8 * np.abs(YZ).max()
    h, st = oracle.pair_halfdisp(r, g, eps, dt)
    hr, _ = oracle.pair_halfdisp(r, g, eps, dt, method=0, quad=True)
    assert st["universal"] == 1
    assert np.abs(h - hr).max() <= 1e-8 * np.abs(hr).max()


def test_universal_variables_converge_from_far_above_root():
    """A near-radial attractive pair a few microns apart, approaching at 543 of its 563
    relative speed (from the Coulomb cube after 39 steps): the second-order start guess
    lies 5000x above the root on a hyperbolic branch, where a Newton step moves s by only
    1/sqrt(-beta) ~ 0.014.  Plain Newton stopped at the iteration cap with a position
    displacement of 1e76; the safeguarded iteration (bisection when Newton stalls) must
    converge and agree with the quad-precision solve."""
    r = np.array([-4.064577389883972e-06, 7.483568417843145e-06, -9.615181365080216e-06])
    g = np.array([95.72878999340595, -231.02576430088004, 504.2191870037502])
    for method in (1, 2):
        h, st = oracle.pair_halfdisp(r, g, -2.0, 1e-5, method=method)
        hq, _ = oracle.pair_halfdisp(r, g, -2.0, 1e-5, method=method, quad=True)
        assert st["nonconverged"] == 0 and st["uv_iterations"] < 60
        assert np.abs(h[:3] - hq[:3]).max() <= 1e-12 * np.abs(g).max() * 1e-5
        assert np.abs(h[3:] - hq[3:]).max() <= 1e-12 * np.abs(g).max()
        assert np.abs(h[:3]).max() < np.abs(g).max() * 1e-5
