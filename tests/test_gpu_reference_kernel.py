"""The reference's own GPU pair kernel (bia/find_dXYUV_kernel.cu, compiled unmodified for
sm_100a by oracle/build_ref.sh) run on the B200 next to ours.

* It reproduces its own committed .BIA record (made on an older GPU) -- a pin of the
  record itself.
* On a gravitational ball with bound pairs, ours and the reference's GPU kernel agree with
  the quad-precision evaluation of the algorithm; ours is at least as close.
Only the reference's ALG method is run (its RKF mode has a __syncthreads() inside
divergent code, bia/bia-rkf.cu:102).
"""
import numpy as np
import pytest

import oracle
from bia_3d_gpu_b200 import BIASolver, default_config, initial
from conftest import max_rel_err, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_gpu_available(),
                                 reason="oracle/_ref/libref_bia.so not built (no reference sources)")]


def _ref_step(s, eps, dt):
    n = s.shape[1]
    d = oracle.ref_gpu_rows(s, eps, dt, range(1, n + 1))
    d[0] += s[3] * dt
    d[1] += s[4] * dt
    d[2] += s[5] * dt
    return s + d


def test_reference_kernel_reproduces_its_record(cuda, golden, golden_ic):
    got = _ref_step(golden_ic, -6e-7, 1.0)
    ref = golden_ic + golden["bia_disp_aos"].reshape(-1, 6).T
    assert rel_err(got[:3], ref[:3]) <= 1e-12 and max_rel_err(got[:3], ref[:3]) <= 1e-11
    assert rel_err(got[3:], ref[3:]) <= 1e-12


def test_ours_vs_reference_kernel_against_quad(cuda):
    s, eps = initial.gravity_ball(200, seed=71)
    dt = 1e-3
    ref_gpu = _ref_step(s, eps, dt)
    t = cuda.tensor(s, device="cuda")
    with BIASolver() as solver:
        st = solver.step(t, default_config(eps_th=eps, dt=dt))
    ours = t.cpu().numpy()
    quad, _, _ = oracle.bia_step(s, eps, dt, quad=True)
    assert st["ellipse"] > 0
    err_ours = max_rel_err(ours, quad)
    err_ref = max_rel_err(ref_gpu, quad)
    print(f"max relative error vs quad: ours {err_ours:.3e}, reference kernel {err_ref:.3e}")
    assert err_ours <= 1e-12
    assert err_ours <= max(err_ref, 1e-14)
