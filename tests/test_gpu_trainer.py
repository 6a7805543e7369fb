"""Training of the learned heads on the GPU (bia_trainer_*).

* The samples: the targets solve Kepler's equation for the (e, M) the inputs encode.
* The gradient of one batch from the tensor-core forward and backward passes matches
  (a) a numpy evaluation that rounds the same operands to BF16 (the exact arithmetic of the
  kernels up to FP32 summation order) and (b) torch FP32 autograd of the same network (the
  unrounded gradient) to BF16 tolerance.
* Both heads trained from a fixed seed on 2^22 device samples reach the guess error of the
  heads the library ships (elliptic median <= 1.4e-3 rad, hyperbolic <= 2.2e-3 rad on new
  samples), and a learned step with the trained heads matches the oracle.
"""
import time

import numpy as np
import pytest

import oracle
from bia_3d_gpu_b200 import METHOD_LEARNED, BIASolver, default_config, initial
from bia_3d_gpu_b200 import train_heads as th

pytestmark = pytest.mark.gpu

H = 64


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((H, 2), (H,), (H, H), (H,), (H, H), (H,), (H,), (1,)):
        cnt = int(np.prod(shape))
        out.append(p[o:o + cnt].reshape(shape))
        o += cnt
    assert o == p.size
    return out


def bf16(a):
    return th.bf16_to_f32(th.bf16_round(np.asarray(a, np.float32))).astype(np.float64)


def grad_reference(p, x, y, rounded):
    """Gradient of mean((net(x) - y)^2); rounded: the kernels' BF16 operands."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p)
    R = bf16 if rounded else (lambda a: np.asarray(a, np.float64))
    rows = x.shape[0]
    xb, W1b, W2b, W3b = R(x), R(W1), R(W2), R(W3)
    z1 = xb @ W1b.T + b1
    h1 = R(np.maximum(z1, 0))
    z2 = h1 @ W2b.T + b2
    h2 = R(np.maximum(z2, 0))
    z3 = h2 @ W3b.T + b3
    h3 = np.maximum(z3, 0)
    yv = h3 @ w4 + b4[0]
    err = yv - y
    dy = err * (2.0 / rows)
    dyb = R(dy)
    dw4 = R(h3).T @ dyb
    db4 = np.array([dyb.sum()])
    dz3 = R(dy[:, None] * w4[None, :] * (z3 > 0))
    dW3, db3 = dz3.T @ h2, dz3.sum(0)
    dz2 = R((dz3 @ W3b) * (z2 > 0))
    dW2, db2 = dz2.T @ h1, dz2.sum(0)
    dz1 = R((dz2 @ W2b) * (z1 > 0))
    dW1, db1 = dz1.T @ xb, dz1.sum(0)
    g = np.concatenate([a.ravel() for a in (dW1, db1, dW2, db2, dW3, db3, dw4, db4)])
    return g, float(np.mean(err ** 2))


def grad_torch(p, x, y):
    import torch
    W1, b1, W2, b2, W3, b3, w4, b4 = [torch.tensor(a, dtype=torch.float32, requires_grad=True) for a in unpack(p)]
    X = torch.tensor(x, dtype=torch.float32)
    Y = torch.tensor(y, dtype=torch.float32)
    h = torch.relu(X @ W1.T + b1)
    h = torch.relu(h @ W2.T + b2)
    h = torch.relu(h @ W3.T + b3)
    loss = torch.mean((h @ w4 + b4 - Y) ** 2)
    loss.backward()
    return np.concatenate([a.grad.numpy().ravel() for a in (W1, b1, W2, b2, W3, b3, w4, b4)]).astype(np.float64)


LAYERS = {"W1": (0, 128), "b1": (128, 192), "W2": (192, 4288), "b2": (4288, 4352), "W3": (4352, 8448),
          "b3": (8448, 8512), "w4": (8512, 8576), "b4": (8576, 8577)}


@pytest.mark.parametrize("head", [0, 1])
def test_samples_solve_keplers_equation(cuda, head):
    with BIASolver() as solver:
        tr = solver.trainer(head, 1 << 14, seed=5)
        x, y = tr.copy_samples(0, 4096)
        tr.close()
    x, y = x.astype(np.float64), y.astype(np.float64)
    if head == 0:
        e = (x[:, 0] + 1.0) * 0.99 / 2.0
        M = (x[:, 1] + 1.0) * np.pi / 2.0
        E = y * np.pi
        res = E - e * np.sin(E) - M
        assert e.min() >= 0.0 and e.max() <= 0.99 * (1 + 1e-6) and M.min() >= 0.0 and M.max() <= np.pi * (1 + 1e-6)
    else:
        e = np.exp((x[:, 0] + 1.0) * np.log(50.0) / 2.0)
        M = np.expm1((x[:, 1] + 1.0) * np.log1p(100.0) / 2.0)
        Hy = y * 6.0
        res = (e * np.sinh(Hy) - Hy - M) / (e * np.cosh(Hy))
        assert e.min() >= 1.0 and e.max() <= 50.01 and M.max() <= 100.01
    # the inputs and targets are FP32 roundings of the FP64 solution
    assert np.abs(res).max() <= 1e-4, np.abs(res).max()


@pytest.mark.parametrize("head", [0, 1])
def test_trainer_gradient_matches_references(cuda, head):
    rows = 512
    rng = np.random.default_rng(50 + head)
    with BIASolver() as solver:
        tr = solver.trainer(head, 1 << 14, seed=6 + head)
        # parameters after a short training, so that every ReLU and gradient is in play
        tr.train(1, batch=1024, lr=2e-3)
        p = tr.params()
        x, y = tr.copy_samples(int(rng.integers(0, (1 << 14) - rows)), rows)
        xt = cuda.tensor(x, device="cuda")
        yt = cuda.tensor(y, device="cuda")
        g, loss = tr.gradient(xt.data_ptr(), yt.data_ptr(), rows)
        tr.close()
    ref_b, loss_b = grad_reference(p, x, y, rounded=True)
    ref_f = grad_torch(p, x, y)
    assert abs(loss - loss_b) <= 1e-3 * loss_b
    for name, (a, b) in LAYERS.items():
        gb, rb, rf = g[a:b].astype(np.float64), ref_b[a:b], ref_f[a:b]
        e_b = np.linalg.norm(gb - rb) / np.linalg.norm(rb)
        e_f = np.linalg.norm(gb - rf) / np.linalg.norm(rf)
        print(f"head {head} {name}: rel err vs BF16-operand reference {e_b:.2e}, vs torch FP32 {e_f:.2e}")
        assert e_b <= 5e-3, (name, e_b)
        assert e_f <= 5e-2, (name, e_f)


def test_trained_heads_reach_shipped_guess_error(cuda, tmp_path):
    """Both heads from seed 0: 2^22 samples each, 24 epochs of Adam (batch 4096, lr 2e-3,
    cosine annealing), all on the GPU.  Guess error of the exported BF16 heads on new samples
    (numpy solver) at the level of the shipped heads, and a learned step with them matches the
    oracle."""
    t0 = time.perf_counter()
    records, info = th.train_device(samples=1 << 22, epochs=24, seed=0)
    elapsed = time.perf_counter() - t0
    path = tmp_path / "heads.bin"
    th.write_records(str(path), records)
    heads = th.read_heads(str(path))
    ell, hyp = th.make_samples(200000, np.random.default_rng(123))
    e_ell = th.guess_error(heads[0], ell[0], ell[1], np.pi)
    e_hyp = th.guess_error(heads[1], hyp[0], hyp[1], th.HYP_OUT)
    print(f"device training: {elapsed:.1f} s for both heads ({[round(i['train_s'], 2) for i in info]} s of "
          f"epochs); guess error median elliptic {np.median(e_ell):.2e} rad, hyperbolic {np.median(e_hyp):.2e}")
    assert np.median(e_ell) <= 1.4e-3 and np.median(e_hyp) <= 2.2e-3
    s, eps, q = initial.coulomb_cube(1000, seed=52, dmin=1e-2)
    t = cuda.tensor(s, device="cuda")
    qt = cuda.tensor(q, device="cuda")
    with BIASolver() as solver:
        solver.load_heads(str(path))
        st = solver.step(t, default_config(eps_th=eps, dt=1e-3, method=METHOD_LEARNED), q=qt)
    g = t.cpu().numpy()
    r, _, _ = oracle.bia_step(s, eps, 1e-3, q=q)
    assert st["learned"] > 0 and st["learned_fallbacks"] <= 0.01 * st["learned"]
    assert np.linalg.norm(g - r) / np.linalg.norm(r) <= 1e-12
