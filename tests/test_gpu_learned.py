"""The learned mixed-precision form (BIA_METHOD_LEARNED) on the GPU.

* The heads evaluated on the tensor cores (tcgen05, BF16 operands, FP32 accumulators in
  tensor memory) agree with the numpy evaluation of the same BF16 network.
* Learned steps match the FP64 oracle's ALG step to the plain form's bar (<= 1e-12
  relative, positions and velocities) on mixed-class systems.  A pair goes to a head when
  its fifth-order universal-variable start is not exact and it lies inside a head's
  domain; at the benchmark steps (dt = 1e-5 on the Coulomb cube) that is under 0.1 % of
  the pairs, so these tests take steps of dt = 1e-3, where ~45 % of the Coulomb pairs and
  a few percent of the gravitational ones start from a head's guess; few of them fall back
  to the plain solver.
* Deterministic mode is bitwise reproducible; the method is refused without heads.
"""
import numpy as np
import pytest

import oracle
from bia_3d_gpu_b200 import BIASolver, BiaError, METHOD_LEARNED, default_config, initial
from bia_3d_gpu_b200 import train_heads as th
from conftest import max_rel_err, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("head", [0, 1])
def test_tensor_core_heads_match_numpy(cuda, head):
    rng = np.random.default_rng(30 + head)
    n = 5000  # not a multiple of the 256-row tile
    x = rng.uniform(-1, 1, (n, 2)).astype(np.float32)
    ref = th.head_forward(th.read_heads()[head], x)
    xin = cuda.tensor(x, device="cuda")
    out = cuda.empty(n, dtype=cuda.float32, device="cuda")
    with BIASolver() as solver:
        solver.load_heads()
        solver.head_eval(head, xin, out)
        solver.stream.synchronize()
    got = out.cpu().numpy()
    diff = np.abs(got - ref)
    assert np.all(np.isfinite(got))
    assert np.median(diff) <= 1e-5 and diff.max() <= 2e-3, (np.median(diff), diff.max())


def _learned_vs_oracle(cuda, s, eps, dt, q=None, steps=1, method=1):
    t = cuda.tensor(s, device="cuda")
    qt = cuda.tensor(q, device="cuda") if q is not None else None
    with BIASolver() as solver:
        solver.load_heads()
        st = None
        for _ in range(steps):
            st = solver.step(t, default_config(eps_th=eps, dt=dt, method=METHOD_LEARNED), q=qt)
    g = t.cpu().numpy()
    r = s
    for _ in range(steps):
        r, _, _ = oracle.bia_step(r, eps, dt, q=q, method=method)
    return g, r, st


def test_learned_coulomb_matches_oracle(cuda):
    """Coulomb cube n = 1500 at dt = 1e-3: one learned step against the oracle's step of the
    reference's ALG path; two steps against the oracle's FP64 universal-variable path.  (Two
    steps of the FP64 ALG path are already ~3e-13 off the exact, quad-precision steps in
    velocity at this step length, from its close pairs; the universal-variable path stays
    within 3e-16 of them.)"""
    s, eps, q = initial.coulomb_cube(1500, seed=31, dmin=1e-2)
    g, r, st = _learned_vs_oracle(cuda, s, eps, 1e-3, q=q, steps=1)
    assert rel_err(g[:3], r[:3]) <= 1e-12 and rel_err(g[3:], r[3:]) <= 1e-12
    assert max_rel_err(g[:3], r[:3]) <= 1e-12 and max_rel_err(g[3:], r[3:]) <= 1e-12
    g, r, st = _learned_vs_oracle(cuda, s, eps, 1e-3, q=q, steps=2, method=2)
    assert rel_err(g[:3], r[:3]) <= 1e-12 and rel_err(g[3:], r[3:]) <= 1e-12
    assert max_rel_err(g[:3], r[:3]) <= 1e-12 and max_rel_err(g[3:], r[3:]) <= 1e-12
    assert st["learned"] > 0.3 * 1500 * 1499 // 2
    assert st["learned_fallbacks"] <= 0.01 * st["learned"]
    assert st["nonfinite"] == 0 and st["timeouts"] == 0
    # one to four FP32 Newton steps per learned pair before its FP64 step
    assert st["learned"] <= st["learned_fp32_steps"] <= 4 * st["learned"]


def test_learned_gravity_ball_matches_oracle(cuda):
    s, eps = initial.gravity_ball(400, seed=32)
    g, r, st = _learned_vs_oracle(cuda, s, eps, 1e-3, steps=3)
    assert rel_err(g[:3], r[:3]) <= 1e-12 and rel_err(g[3:], r[3:]) <= 1e-12
    assert max_rel_err(g[:3], r[:3]) <= 1e-12 and max_rel_err(g[3:], r[3:]) <= 1e-12
    assert st["learned"] > 0 and st["nonfinite"] == 0 and st["timeouts"] == 0


def test_learned_against_quad(cuda):
    s, eps, q = initial.coulomb_cube(600, seed=33, dmin=1e-2)
    t = cuda.tensor(s, device="cuda")
    qt = cuda.tensor(q, device="cuda")
    with BIASolver() as solver:
        solver.load_heads()
        st = solver.step(t, default_config(eps_th=eps, dt=1e-3, method=METHOD_LEARNED), q=qt)
    g = t.cpu().numpy()
    assert st["learned"] > 0.3 * 600 * 599 // 2
    rq, _, _ = oracle.bia_step(s, eps, 1e-3, q=q, quad=True)
    assert max_rel_err(g[:3], rq[:3]) <= 1e-13 and max_rel_err(g[3:], rq[3:]) <= 1e-13


def test_learned_deterministic_and_atomic(cuda):
    s, eps, q = initial.coulomb_cube(5000, seed=34)
    outs = []
    for det in (1, 1, 0):
        t = cuda.tensor(s, device="cuda")
        qt = cuda.tensor(q, device="cuda")
        with BIASolver() as solver:
            solver.load_heads()
            solver.step(t, default_config(eps_th=eps, dt=1e-3, method=METHOD_LEARNED, deterministic=det), q=qt)
        outs.append(t.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    assert rel_err(outs[2], outs[0]) <= 1e-15


def test_learned_needs_heads(cuda):
    s, eps = initial.gravity_ball(64, seed=35)
    t = cuda.tensor(s, device="cuda")
    with BIASolver() as solver:
        with pytest.raises(BiaError):
            solver.step(t, default_config(eps_th=eps, dt=1e-4, method=METHOD_LEARNED))


@pytest.mark.parametrize("dt", [1e-5, 1e-3])
def test_learned_split_step_matches_oracle(cuda, dt):
    """The split learned step at n = 6000 (the plain pairs in the rest kernel, which lists
    the warp-blocks holding learned pairs; the head kernel's guesses; the finish kernel, which
    adds the learned pairs onto the same partials): sampled particles against the oracle's
    full pair sums, and momentum from the antisymmetry.  At dt = 1e-5 almost every series is
    exact and the listed blocks hold one or two pairs each (the batched finish); at dt = 1e-3
    ~45 % of the pairs are listed (the per-block finish)."""
    s, eps, q = initial.coulomb_cube(6000, seed=36)
    t = cuda.tensor(s, device="cuda")
    qt = cuda.tensor(q, device="cuda")
    d = cuda.zeros_like(t)
    with BIASolver() as solver:
        solver.load_heads()
        st = solver.step(t, default_config(eps_th=eps, dt=dt, method=METHOD_LEARNED), q=qt, disp=d)
    disp = d.cpu().numpy()
    n = 6000
    assert st["learned"] > (0.3 if dt > 1e-4 else 1e-4) * n * (n - 1) // 2
    assert sum(st[k] for k in ("hyperbola", "ellipse", "universal", "degenerate", "parabola")) == n * (n - 1) // 2
    sel = np.random.default_rng(37).choice(n, 24, replace=False)
    ref = oracle.particle_disp(s, eps, dt, sel, q=q)
    got = disp[:, sel].T
    assert np.abs(got[:, :3] - ref[:, :3]).max() <= 1e-12 * np.abs(s[:3]).max()
    assert np.abs(got[:, 3:] - ref[:, 3:]).max() <= 1e-12 * np.abs(s[3:]).max()
    kick = disp[3:].sum(axis=1)
    assert np.abs(kick).max() <= 1e-12 * np.abs(disp[3:]).sum(axis=1).max()


def test_learned_autotune_layout(cuda):
    """The autotuner times the learned step as one kernel and split, keeps the faster for
    this size without changing the state, and the step then still matches the oracle."""
    s, eps, q = initial.coulomb_cube(6000, seed=38)
    t = cuda.tensor(s, device="cuda")
    qt = cuda.tensor(q, device="cuda")
    cfg = default_config(eps_th=eps, dt=1e-5, method=METHOD_LEARNED)
    with BIASolver() as solver:
        solver.load_heads()
        var, ms = solver.autotune(t, cfg, q=qt)
        assert var in (0, 1) and set(ms) == {"one_kernel", "split"}
        assert cuda.equal(t, cuda.tensor(s, device="cuda"))
        d = cuda.zeros_like(t)
        solver.step(t, cfg, q=qt, disp=d)
    sel = np.random.default_rng(39).choice(6000, 16, replace=False)
    ref = oracle.particle_disp(s, eps, 1e-5, sel, q=q)
    got = d.cpu().numpy()[:, sel].T
    assert np.abs(got[:, :3] - ref[:, :3]).max() <= 1e-12 * np.abs(s[:3]).max()
    assert np.abs(got[:, 3:] - ref[:, 3:]).max() <= 1e-12 * np.abs(s[3:]).max()


@pytest.mark.parametrize("n", [2, 31, 33, 97, 1025])
def test_learned_split_step_ragged_sizes(cuda, n):
    """The split learned step (the untuned layout at every size) at particle counts that
    leave partial warp-blocks, down to one pair: against the oracle's ALG step (dt = 1e-3,
    so that heads are used)."""
    s, eps, q = initial.coulomb_cube(n, seed=40 + n, dmin=1e-2)
    g, r, st = _learned_vs_oracle(cuda, s, eps, 1e-3, q=q, steps=1)
    assert rel_err(g[:3], r[:3]) <= 1e-12 and rel_err(g[3:], r[3:]) <= 1e-12
    assert sum(st[k] for k in ("hyperbola", "ellipse", "universal", "degenerate", "parabola")) == n * (n - 1) // 2
    assert st["nonfinite"] == 0 and st["timeouts"] == 0
