"""Pins of the CPU oracle against the reference's own outputs and known answers.

The oracle (oracle/bia_oracle.c) restates the reference's CPU path; these tests check
it before it is trusted as the parity reference for the CUDA kernels:
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

    Tolerance: global relative error <= 1e-12 in positions and velocities (the
    north-star bar).  The per-particle maximum is looser, 1e-11 of max|X|: a pair
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
    (bia/bia.f90:295-296); the oracle integrates along the line of motion."""
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
