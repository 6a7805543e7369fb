"""The learned Kepler heads (CPU): the committed learned_heads.bin parses, and its BF16
network, evaluated in numpy exactly as the tensor-core kernels compute it (BF16 weights and
activations, FP32 accumulation), gives starting guesses close to the FP64 solution on fresh
samples of both domains."""
import numpy as np

from bia_3d_gpu_b200 import HEADS_PATH
from bia_3d_gpu_b200 import train_heads as th


def test_heads_file_layout():
    heads = th.read_heads(HEADS_PATH)
    assert len(heads) == 2
    for h in heads:
        w1, w2, w3, b1, b2, b3, w4, b4 = h
        assert w1.shape == (64, 16) and w2.shape == (64, 64) and w3.shape == (64, 64)
        assert np.all(th.bf16_to_f32(w1)[:, 2:] == 0)   # padded inputs carry no weight
        assert b1.shape == b2.shape == b3.shape == w4.shape == (64,) and b4.shape == (1,)


def test_elliptic_head_guess_error():
    rng = np.random.default_rng(11)
    e = rng.uniform(0, 0.99, 20000)
    M = rng.uniform(0, np.pi, 20000)
    E = th.solve_elliptic(e, M)
    assert np.abs(E - e * np.sin(E) - M).max() < 1e-14
    guess = th.head_forward(th.read_heads(HEADS_PATH)[0], th.ell_features(e, M).astype(np.float32)) * np.pi
    err = np.abs(guess - E)
    assert np.median(err) < 5e-3 and np.quantile(err, 0.99) < 3e-2 and err.max() < 0.3


def test_hyperbolic_head_guess_error():
    rng = np.random.default_rng(12)
    e = rng.uniform(1.001, 50, 20000)
    M = rng.uniform(0, 100, 20000)
    H = th.solve_hyperbolic(e, M)
    assert np.abs((e * np.sinh(H) - H - M) / np.maximum(M, 1)).max() < 1e-13
    guess = th.head_forward(th.read_heads(HEADS_PATH)[1], th.hyp_features(e, M).astype(np.float32)) * th.HYP_OUT
    err = np.abs(guess - H)
    assert np.median(err) < 5e-3 and np.quantile(err, 0.99) < 3e-2 and err.max() < 0.3


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.0e-3], np.float32)
    r = th.bf16_to_f32(th.bf16_round(x))
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625 and r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2 ** -8
