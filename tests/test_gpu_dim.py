"""The direct-integration (DIM) reference solver on the GPU (dim/rkf_kernel.cu rebuilt).

Checks: against the oracle's CPU restatement of rkf_c_ on small lattices (same adaptive
step sequence, final state to 1e-12), against the reference's own DIM run committed as
OUT/0001332_10^0.DIM (N = 1332, eps_th = -3e-7, 0 -> 1; its adaptive trajectory of
particle 1 in OUT/0001332.DIM has 239 time levels), energy conservation in quad
precision (the reference reports dE/E0 = 1.33e-15 for this run, README.md:41), and the
rkf_c_ drop-in on host arrays.
"""
import numpy as np
import pytest

import oracle
from bia_3d_gpu_b200 import BIASolver, initial, rkf_c
from conftest import max_rel_err, rel_err

pytestmark = pytest.mark.gpu


def _dim_gpu(cuda, s, eps, x0, xe):
    t = cuda.tensor(s, device="cuda")
    with BIASolver() as solver:
        st = solver.dim_integrate(t, eps, x0, xe)
        solver.stream.synchronize()
    return t.cpu().numpy(), st


@pytest.mark.parametrize("NL,eps,xe", [(1, -3e-3, 1.0), (2, -1e-3, 0.5)])
def test_dim_matches_oracle_small(cuda, NL, eps, xe):
    s, _ = initial.lattice(NL=NL, seed=7)
    g, st = _dim_gpu(cuda, s, eps, 0.0, xe)
    y0 = np.ascontiguousarray(s.T).reshape(-1)
    yn, ier, nacc, nde = oracle.dim_rkf(y0, eps, 0.0, xe)
    r = yn.reshape(-1, 6).T
    assert ier == 0 and st["ier"] == 0
    assert st["accepted"] == nacc and st["nde"] == nde
    assert rel_err(g[:3], r[:3]) <= 1e-12 and max_rel_err(g[:3], r[:3]) <= 1e-12
    assert rel_err(g[3:], r[3:]) <= 1e-12 and max_rel_err(g[3:], r[3:]) <= 1e-12


def test_dim_matches_reference_run(cuda, golden, golden_ic):
    g, st = _dim_gpu(cuda, golden_ic, golden["eps_dim"].item(), 0.0, 1.0)
    ref = golden["dim_final_aos"].reshape(-1, 6).T
    assert st["ier"] == 0 and st["x_reached"] == 1.0
    # the reference wrote one trajectory line per accepted step plus the initial one
    assert st["accepted"] == golden["dim_p1_traj"].shape[0] - 1
    assert rel_err(g[:3], ref[:3]) <= 1e-12 and max_rel_err(g[:3], ref[:3]) <= 1e-12
    assert rel_err(g[3:], ref[3:]) <= 1e-12
    # particle 1's final line (dim/dim_3D.f90:31, 17 significant digits)
    assert np.abs(g[:, 0] - golden["dim_p1"][1:]).max() <= 1e-13
    e0 = oracle.invariance(golden_ic, 2 * golden["eps_dim"].item(), quad=True)
    e1 = oracle.invariance(g, 2 * golden["eps_dim"].item(), quad=True)
    assert abs((e1["KE"] + e1["PE"]) / (e0["KE"] + e0["PE"]) - 1) <= 1e-14


def test_rkf_c_dropin(cuda):
    s, _ = initial.lattice(NL=1, seed=9)
    y0 = np.ascontiguousarray(s.T).reshape(-1)
    yh0 = y0.copy()  # rkf_c_ overwrites YH0 with the final state, as the reference does
    out = rkf_c(yh0.size, -3e-3, 0.0, 1.0, yh0, 1, 0.0, 1e-16)
    yn, ier, nacc, nde = oracle.dim_rkf(y0, -3e-3, 0.0, 1.0)
    assert out["IER"] == 0 and out["X0"] == 1.0 and out["INIT"] == 2 and out["NDE"] == nde
    assert np.abs(out["YHN"] - yn).max() <= 1e-12 * np.abs(yn).max()
    assert np.array_equal(out["YH0"], out["YHN"])
    assert np.all(np.isfinite(out["ESE"])) and np.abs(out["ESE"]).max() < 1e-12


def test_dim_driver_reproduces_reference_run(cuda, golden, golden_ic, tmp_path):
    """dim/dim_3D.f90 through the driver on the reference's initial condition: the .DIM
    record and particle 1's text line against the reference's own run."""
    from bia_3d_gpu_b200 import driver, records
    bbb = tmp_path / "0001332_10^0.bbb"
    records.write_bbb(bbb, [golden_ic])
    out = driver.run_dim(bbb, tmp_path / "0001332_10^0.DIM", tmp_path / "DIM_10^0.0001332",
                         eps_th=golden["eps_dim"].item())
    assert out[0][0] == 0
    (t, g), = records.read_timed(tmp_path / "0001332_10^0.DIM")
    ref = golden["dim_final_aos"].reshape(-1, 6).T
    assert t == 1.0
    assert rel_err(g[:3], ref[:3]) <= 1e-12 and rel_err(g[3:], ref[3:]) <= 1e-12
    line = (tmp_path / "DIM_10^0.0001332").read_text().splitlines()[-1]
    vals = [float(line[23 + 24 * k:23 + 24 * (k + 1)]) for k in range(6)]
    assert np.abs(np.array(vals) - golden["dim_p1"][1:]).max() <= 1e-13


def test_dim_against_bia_plummer_8192(cuda):
    """DIM as the physics check of BIA beyond the reference's N = 1332 (the comparison of
    bia/bia.f90:261-278): a seeded Plummer sphere of 8192 particles, one BIA step of
    dt = 1e-4 (the reference's ALG path and the universal-variable form) against DIM
    integrated from 0 to dt with the per-particle coupling eps/2.  The two methods differ by
    the binary approximation itself: ~1e-14 of the state in positions, ~4e-13 in
    velocities (the oracle's BIA and DIM at n = 512 agree to 7e-15 and 4e-13).  The DIM of
    bia_dim_integrate (rsqrt-based inverse cube) also agrees with the rkf_c_ drop-in's DIM
    (the reference's sqrt and division) to 1e-13 with the same accepted steps."""
    from bia_3d_gpu_b200 import METHOD_UNIVERSAL, default_config
    s, eps = initial.plummer(8192, seed=81)
    dt = 1e-4
    g, st = _dim_gpu(cuda, s, eps / 2, 0.0, dt)
    assert st["ier"] == 0 and st["x_reached"] == dt
    y0 = np.ascontiguousarray(s.T).reshape(-1).copy()
    out = rkf_c(y0.size, eps / 2, 0.0, dt, y0, 1, 0.0, 1e-16)
    exact = out["YHN"].reshape(-1, 6).T
    assert out["IER"] == 0
    assert rel_err(g[:3], exact[:3]) <= 1e-13 and rel_err(g[3:], exact[3:]) <= 1e-13
    drift = s[:3] + s[3:] * dt
    for method in (1, METHOD_UNIVERSAL):
        t = cuda.tensor(s, device="cuda")
        with BIASolver() as solver:
            solver.step(t, default_config(eps_th=eps, dt=dt, method=method))
        b = t.cpu().numpy()
        ep, ev = rel_err(b[:3], g[:3]), rel_err(b[3:], g[3:])
        print(f"BIA method {method} vs DIM, n = 8192, dt = 1e-4: positions {ep:.2e}, velocities {ev:.2e}; "
              f"interaction dX {rel_err(b[:3] - drift, g[:3] - drift):.2e}, "
              f"dV {rel_err(b[3:] - s[3:], g[3:] - s[3:]):.2e}; DIM accepted steps {st['accepted']}")
        assert ep <= 1e-12 and ev <= 1e-11
