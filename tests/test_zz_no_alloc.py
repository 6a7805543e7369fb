"""The allocation-free step entry point, bia_step_noalloc, through the C-ABI.

It exists for callers that cannot allocate GPU memory while they run (their memory
pool belongs to another framework, or a real-time loop must not call into the CUDA
allocator): its scratch is a fixed array inside libbia_b200.so, for n <= 2048.  The
test compares two consecutive steps with the context-based bia_step on the same input
(same tolerance as the parity tests; the kernels and the reduction order are the same,
so the results are in fact identical), for the ALG and universal-variable methods and at
the size limit itself (n = 2048 fills the whole partial array); the first step is also
checked against the CPU oracle directly.  n above the limit is refused.
This file is collected last so that a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

import oracle
from bia_3d_gpu_b200 import METHOD_ALG, METHOD_UNIVERSAL, BIASolver, capi, default_config, initial
from conftest import max_rel_err, rel_err

pytestmark = pytest.mark.gpu


def _ptrs(t):
    n = t.shape[1]
    return [ctypes.c_void_p(t.data_ptr() + k * n * 8) for k in range(6)]


@pytest.mark.parametrize("method", [METHOD_ALG, METHOD_UNIVERSAL])
@pytest.mark.parametrize("n", [1500, 2048])
def test_noalloc_step_matches_context_step(cuda, n, method):
    s, eps, q = initial.coulomb_cube(n, seed=61)
    cfg = default_config(eps_th=eps, dt=1e-5, method=method)
    a = cuda.tensor(s, device="cuda")
    b = cuda.tensor(s, device="cuda")
    qt = cuda.tensor(q, device="cuda")
    da = cuda.zeros_like(a)
    db = cuda.zeros_like(b)
    stream = cuda.cuda.Stream()
    stream.wait_stream(cuda.cuda.current_stream())
    with BIASolver(stream=stream) as solver:
        for call in range(2):
            solver.step(a, cfg, q=qt, disp=da, stats=False)
            st = capi.lib().bia_step_noalloc(ctypes.byref(cfg), s.shape[1], *_ptrs(b),
                                             ctypes.c_void_p(qt.data_ptr()),
                                             ctypes.c_void_p(db.data_ptr()),
                                             ctypes.c_void_p(stream.cuda_stream))
            assert st == capi.BIA_OK
            stream.synchronize()
            ga, gb = a.cpu().numpy(), b.cpu().numpy()
            assert rel_err(gb[:3], ga[:3]) <= 1e-12 and max_rel_err(gb[:3], ga[:3]) <= 1e-12
            assert rel_err(gb[3:], ga[3:]) <= 1e-12 and max_rel_err(gb[3:], ga[3:]) <= 1e-12
            assert np.array_equal(db.cpu().numpy(), da.cpu().numpy())
            if call == 0:
                ref, _, _ = oracle.bia_step(s, eps, 1e-5, method=method, q=q)
                assert rel_err(gb[:3], ref[:3]) <= 1e-12 and max_rel_err(gb[:3], ref[:3]) <= 1e-12
                assert rel_err(gb[3:], ref[3:]) <= 1e-12 and max_rel_err(gb[3:], ref[3:]) <= 1e-12


def test_noalloc_step_rejects_n_above_limit(cuda):
    n = 2049
    s, eps = initial.gravity_ball(n, seed=62)
    t = cuda.tensor(s, device="cuda")
    before = t.clone()
    st = capi.lib().bia_step_noalloc(ctypes.byref(default_config(eps_th=eps, dt=1e-4)), n, *_ptrs(t),
                                     None, None, None)
    assert st == capi.BIA_ERR_INVALID_ARGUMENT
    cuda.cuda.synchronize()
    assert cuda.equal(t, before)
