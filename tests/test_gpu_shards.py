"""The shard kernels of the multi-GPU step on one GPU: the shards' sums of one step,
computed one after the other and added, applied with bia_apply_update, give the whole
step (deterministic and atomic reductions, the ALG, universal-variable and learned forms),
and the oracle's step."""
import numpy as np
import pytest

import oracle
from bia_3d_gpu_b200 import METHOD_ALG, METHOD_LEARNED, METHOD_UNIVERSAL, BIASolver, default_config, initial
from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", [METHOD_ALG, METHOD_UNIVERSAL, METHOD_LEARNED])
@pytest.mark.parametrize("nshards", [1, 2, 3, 7])
@pytest.mark.parametrize("det", [1, 0])
def test_shards_add_up_to_the_step(cuda, method, nshards, det):
    s, eps, q = initial.coulomb_cube(2000, seed=92, dmin=1e-2)
    dt = 1e-3 if method == METHOD_LEARNED else 1e-5
    cfg = default_config(eps_th=eps, dt=dt, method=method, deterministic=det)
    qt = cuda.tensor(q, device="cuda")
    whole = cuda.tensor(s, device="cuda")
    parts = cuda.tensor(s, device="cuda")
    with BIASolver() as solver:
        solver.load_heads()
        solver.step(whole, cfg, q=qt, stats=False)
        total = cuda.zeros_like(parts)
        sums = cuda.empty_like(parts)
        for r in range(nshards):
            solver.step_shard(parts, cfg, r, nshards, sums, q=qt)
            total += sums
        solver.apply_update(parts, dt, total)
        solver.stream.synchronize()
    a, b = whole.cpu().numpy(), parts.cpu().numpy()
    assert rel_err(b[:3], a[:3]) <= 1e-14 and rel_err(b[3:], a[3:]) <= 1e-14
    if nshards == 1 and det:
        assert np.array_equal(a, b)
    ref, _, _ = oracle.bia_step(s, eps, dt, q=q, method=1 if method != METHOD_UNIVERSAL else 2)
    assert rel_err(b[:3], ref[:3]) <= 1e-12 and rel_err(b[3:], ref[3:]) <= 1e-12


@pytest.mark.parametrize("n", [2, 33, 97])
def test_shards_of_ragged_sizes(cuda, n):
    """More shards than 32-particle columns (empty shards) and partial blocks: the shards'
    sums still add up to the step."""
    s, eps, q = initial.coulomb_cube(n, seed=93 + n, dmin=1e-2)
    cfg = default_config(eps_th=eps, dt=1e-5, method=METHOD_ALG)
    qt = cuda.tensor(q, device="cuda")
    whole = cuda.tensor(s, device="cuda")
    parts = cuda.tensor(s, device="cuda")
    with BIASolver() as solver:
        solver.step(whole, cfg, q=qt, stats=False)
        total = cuda.zeros_like(parts)
        sums = cuda.empty_like(parts)
        for r in range(5):
            solver.step_shard(parts, cfg, r, 5, sums, q=qt)
            total += sums
        solver.apply_update(parts, 1e-5, total)
        solver.stream.synchronize()
    a, b = whole.cpu().numpy(), parts.cpu().numpy()
    assert rel_err(b[:3], a[:3]) <= 1e-14 and rel_err(b[3:], a[3:]) <= 1e-14
