"""Ensemble engine: independent systems of uneven size in one launch per step.

Each system's result must equal a bia_step of that system alone (same per-block code,
same summation order, so bitwise), and the per-system energies must match the oracle's
quad-precision invariants (bia/Invariance_QPU.f90 per system).
"""
import numpy as np
import pytest

import oracle
from bia_3d_gpu_b200 import BIASolver, METHOD_UNIVERSAL, default_config, initial

pytestmark = pytest.mark.gpu

SIZES = [1, 5, 31, 32, 33, 64, 100, 150, 257]


def _systems(seed=0):
    rng = np.random.default_rng(seed)
    states, eps = [], []
    for k, n in enumerate(SIZES):
        s, e = initial.plummer(n, seed=100 + k) if n > 1 else (rng.standard_normal((6, 1)), -2.0)
        states.append(s)
        eps.append(-2.0 / n if n > 1 else e)
    return states, np.array(eps)


@pytest.mark.parametrize("method", [1, METHOD_UNIVERSAL])
def test_ensemble_equals_single_system_steps(cuda, method):
    states, eps = _systems()
    whole = cuda.tensor(np.concatenate(states, axis=1), device="cuda")
    with BIASolver() as solver:
        ens = solver.ensemble(SIZES, eps)
        cfg = default_config(dt=1e-3, method=method)
        st = ens.run(whole, cfg, 3, graph=True)
        solver.stream.synchronize()
        got = whole.cpu().numpy()
        total = sum(n * (n - 1) // 2 for n in SIZES)
        assert sum(st[k] for k in ("hyperbola", "ellipse", "parabola", "universal", "degenerate")) == 3 * total
        off = 0
        for s, e, n in zip(states, eps, SIZES):
            t = cuda.tensor(s, device="cuda")
            for _ in range(3):
                solver.step(t, default_config(eps_th=e, dt=1e-3, method=method), stats=False)
            solver.stream.synchronize()
            assert np.array_equal(got[:, off:off + n], t.cpu().numpy()), n
            off += n
        ens.close()


def test_ensemble_matches_oracle_and_energy(cuda):
    states, eps = _systems(1)
    whole = cuda.tensor(np.concatenate(states, axis=1), device="cuda")
    with BIASolver() as solver:
        ens = solver.ensemble(SIZES, eps)
        ke, pe = ens.energy(whole)
        for k, (s, e) in enumerate(zip(states, eps)):
            ref = oracle.invariance(s, e, quad=True)
            assert abs(ke[k] - ref["KE"]) <= 1e-13 * max(1.0, abs(ref["KE"]))
            assert abs(pe[k] - ref["PE"]) <= 1e-13 * max(1e-300, abs(ref["PE"]))
        ens.run(whole, default_config(dt=1e-3), 2, graph=False)
        solver.stream.synchronize()
        got = whole.cpu().numpy()
        ens.close()
    off = 0
    for s, e, n in zip(states, eps, SIZES):
        r = s
        for _ in range(2):
            r, _, _ = oracle.bia_step(r, e, 1e-3)
        g = got[:, off:off + n]
        scale = max(np.abs(r[:3]).max(), 1e-300)
        assert np.abs(g[:3] - r[:3]).max() <= 1e-12 * scale, n
        off += n


def test_large_ensemble_phase_locked_equals_single_steps(cuda):
    """Enough warp-blocks (about 20000) for the phase-locked ALG ensemble kernel: every
    system still equals its own single-system step bitwise."""
    rng = np.random.default_rng(5)
    sizes = [int(x) for x in rng.integers(32, 320, 700)]
    states, eps = [], []
    for k, n in enumerate(sizes):
        s, e, q = initial.coulomb_cube(n, seed=1000 + k, dmin=1e-2)
        s[:3] *= 0.3
        states.append(s)
        eps.append(-2.0 / n)
    eps = np.array(eps)
    items = sum((n + 31) // 32 * ((n + 31) // 32 + 1) // 2 for n in sizes)
    assert items > 2 * 148 * 32
    whole = cuda.tensor(np.concatenate(states, axis=1), device="cuda")
    with BIASolver() as solver:
        ens = solver.ensemble(sizes, eps)
        ens.run(whole, default_config(dt=1e-4), 1, graph=False)
        solver.stream.synchronize()
        got = whole.cpu().numpy()
        off = 0
        for s, e, n in zip(states, eps, sizes):
            t = cuda.tensor(s, device="cuda")
            solver.step(t, default_config(eps_th=e, dt=1e-4), stats=False)
            solver.stream.synchronize()
            assert np.array_equal(got[:, off:off + n], t.cpu().numpy()), n
            off += n
        ens.close()


def test_ensemble_learned_equals_single_system_steps(cuda):
    """The learned form over the item table: each system equals its own learned step
    (same per-block code and order, bitwise) and the oracle's plain step to 1e-12."""
    from bia_3d_gpu_b200 import METHOD_LEARNED
    states, eps = _systems(2)
    whole = cuda.tensor(np.concatenate(states, axis=1), device="cuda")
    with BIASolver() as solver:
        solver.load_heads()
        ens = solver.ensemble(SIZES, eps)
        st = ens.run(whole, default_config(dt=1e-3, method=METHOD_LEARNED), 1, graph=True)
        solver.stream.synchronize()
        got = whole.cpu().numpy()
        assert st["learned"] > 0 and st["nonfinite"] == 0 and st["timeouts"] == 0
        off = 0
        for s, e, n in zip(states, eps, SIZES):
            t = cuda.tensor(s, device="cuda")
            solver.step(t, default_config(eps_th=e, dt=1e-3, method=METHOD_LEARNED), stats=False)
            solver.stream.synchronize()
            assert np.array_equal(got[:, off:off + n], t.cpu().numpy()), n
            r, _, _ = oracle.bia_step(s, e, 1e-3)
            scale = max(np.abs(r[:3]).max(), 1e-300)
            assert np.abs(got[:3, off:off + n] - r[:3]).max() <= 1e-12 * scale, n
            off += n
        ens.close()


@pytest.mark.parametrize("method", [1, METHOD_UNIVERSAL, 3])
def test_ensemble_autotune_keeps_results_bitwise(cuda, method):
    """The ensemble autotuner times each launch shape of the method's pair kernels on the
    caller's systems without changing the state, keeps the fastest, and a run with the tuned
    shape is bitwise equal to the untuned run (every shape runs the same per-item
    arithmetic)."""
    from bia_3d_gpu_b200 import initial as ini
    sizes = np.random.default_rng(70).integers(32, 400, 40)
    states = [ini.plummer(int(n), seed=700 + k)[0] for k, n in enumerate(sizes)]
    eps = -2.0 / sizes.astype(np.float64)
    host = np.concatenate(states, axis=1)
    cfg = default_config(dt=1e-3, method=method)
    outs = []
    with BIASolver() as solver:
        solver.load_heads()
        for tuned in (False, True):
            ens = solver.ensemble(sizes, eps)
            whole = cuda.tensor(host, device="cuda")
            if tuned:
                shape, ms = ens.autotune(whole, cfg)
                assert shape in ens.SHAPES[method] and set(ms) == set(ens.SHAPES[method])
                assert np.array_equal(whole.cpu().numpy(), host)
            ens.run(whole, cfg, 3, graph=True, stats=False)
            solver.stream.synchronize()
            outs.append(whole.cpu().numpy())
            ens.close()
    assert np.array_equal(outs[0], outs[1])
