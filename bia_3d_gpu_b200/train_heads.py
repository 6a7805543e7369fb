"""Train the two learned Kepler heads and write bia_3d_gpu_b200/learned_heads.bin.

    python -m bia_3d_gpu_b200.train_heads [--samples 4194304] [--epochs 24] [--seed 0] [--torch]

By default the heads are trained on the GPU by libbia_b200.so (bia_trainer_*): the samples
come from the FP64 Kepler solver on the device, the forward and backward passes run on the
tensor cores (BF16 operands, FP32 accumulation in tensor memory) and Adam updates FP32
master parameters on the device.  --torch trains the same network in FP32 with torch on
the CPU instead (the numpy solver below makes its samples); the tests use it as the
reference of the device gradients.

Each head is an MLP 2 -> 64 -> 64 -> 64 -> 1 (ReLU) that maps an orbit's eccentricity and
mean anomaly to a starting guess of its anomaly:

* elliptic head: e in [0, 0.99], M in [0, pi]  ->  eccentric anomaly E,
  M = E - e sin E (the symmetric half of the period; the kernel folds M into it);
* hyperbolic head: e in [1.001, 50], M in [0, 100] (input log-scaled)  ->  hyperbolic
  anomaly H, M = e sinh H - H (odd in M; the kernel folds the sign).

Targets come from a plain FP64 solver (bracketed Newton to machine precision, vectorised
numpy) on 2^22 samples per head drawn uniformly over the domain.  Training runs in FP32
(torch, Adam); the exported weights are rounded to BF16 (the kernels accumulate in FP32),
biases stay FP32.  Layer 1 is stored padded from 2 to 16 inputs, the K of one BF16
tensor-core step.

File layout (little endian), per head, elliptic first:
    W1 bf16 [64][16], W2 bf16 [64][64], W3 bf16 [64][64]   (output-major: W[n][k])
    b1 f32 [64], b2 f32 [64], b3 f32 [64], W4 f32 [64], b4 f32 [1], pad f32 [3]
preceded by the header: magic b"BIAHEAD1", u32 version 1, u32 heads 2.
"""
import argparse
import os
import struct
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "learned_heads.bin")

HIDDEN = 64
K1 = 16                       # layer-1 inputs padded to one BF16 MMA K step
ELL_E = (0.0, 0.99)
ELL_M = (0.0, np.pi)
HYP_E = (1.001, 50.0)
HYP_M = (0.0, 100.0)
HYP_LOGM = np.log1p(HYP_M[1])
HYP_OUT = 6.0                 # H / 6 is the network output (H < 5.3 on the domain)


def ell_features(e, M):
    """Network inputs of the elliptic head (same arithmetic as the CUDA kernels)."""
    return np.stack([2.0 * e / ELL_E[1] - 1.0, 2.0 * M / np.pi - 1.0], axis=-1)


def hyp_features(e, M):
    return np.stack([2.0 * np.log(e) / np.log(HYP_E[1]) - 1.0,
                     2.0 * np.log1p(M) / HYP_LOGM - 1.0], axis=-1)


def solve_elliptic(e, M):
    """E - e sin E = M, E in [M, M + e] for M in [0, pi]: bracketed Newton in FP64."""
    lo, hi = M.copy(), np.minimum(M + e, np.pi)
    x = np.clip(M + e * np.sin(M), lo, hi)
    for _ in range(80):
        f = x - e * np.sin(x) - M
        lo = np.where(f < 0, x, lo)
        hi = np.where(f >= 0, x, hi)
        xn = x - f / (1.0 - e * np.cos(x))
        bad = ~((xn > lo) & (xn < hi))
        xn = np.where(bad, 0.5 * (lo + hi), xn)
        x = xn
    return x


def solve_hyperbolic(e, M):
    """e sinh H - H = M, H in [0, asinh((M + H_hi)/e)] for M >= 0: bracketed Newton."""
    lo = np.zeros_like(M)
    hi = np.arcsinh((M + 10.0) / e) + 1.0
    hi = np.maximum(hi, np.cbrt(6.0 * M) + 1.0)
    x = np.clip(np.arcsinh(M / e), lo, hi)
    for _ in range(120):
        f = e * np.sinh(x) - x - M
        lo = np.where(f < 0, x, lo)
        hi = np.where(f >= 0, x, hi)
        xn = x - f / (e * np.cosh(x) - 1.0)
        bad = ~((xn > lo) & (xn < hi))
        xn = np.where(bad, 0.5 * (lo + hi), xn)
        x = xn
    return x


def make_samples(n, rng):
    e = rng.uniform(*ELL_E, n)
    M = rng.uniform(*ELL_M, n)
    ell = (ell_features(e, M), solve_elliptic(e, M) / np.pi, e, M)
    e = rng.uniform(*HYP_E, n)
    M = rng.uniform(*HYP_M, n)
    hyp = (hyp_features(e, M), solve_hyperbolic(e, M) / HYP_OUT, e, M)
    return ell, hyp


def train_head(x, y, epochs, seed, log):
    import torch
    torch.manual_seed(seed)
    net = torch.nn.Sequential(torch.nn.Linear(2, HIDDEN), torch.nn.ReLU(),
                              torch.nn.Linear(HIDDEN, HIDDEN), torch.nn.ReLU(),
                              torch.nn.Linear(HIDDEN, HIDDEN), torch.nn.ReLU(),
                              torch.nn.Linear(HIDDEN, 1))
    X = torch.tensor(x, dtype=torch.float32)
    Y = torch.tensor(y, dtype=torch.float32)[:, None]
    opt = torch.optim.Adam(net.parameters(), lr=2e-3)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=epochs)
    bs = 4096
    n = X.shape[0]
    for ep in range(epochs):
        perm = torch.randperm(n)
        tot = 0.0
        for k in range(0, n, bs):
            idx = perm[k:k + bs]
            opt.zero_grad()
            loss = torch.mean((net(X[idx]) - Y[idx]) ** 2)
            loss.backward()
            opt.step()
            tot += loss.item() * len(idx)
        sched.step()
        log(f"  epoch {ep + 1}/{epochs}: mse {tot / n:.3e}")
    return net


def bf16_round(a):
    """Round FP32 to BF16 (nearest even) and return the uint16 bit patterns."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def bf16_to_f32(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


def export_head(net):
    """(bf16 W1 [64][16], W2, W3 [64][64]; f32 b1, b2, b3, W4, b4) as numpy arrays."""
    L = [m for m in net if hasattr(m, "weight")]
    w1 = np.zeros((HIDDEN, K1), np.float32)
    w1[:, :2] = L[0].weight.detach().numpy()
    return (bf16_round(w1), bf16_round(L[1].weight.detach().numpy()),
            bf16_round(L[2].weight.detach().numpy()),
            L[0].bias.detach().numpy().astype(np.float32),
            L[1].bias.detach().numpy().astype(np.float32),
            L[2].bias.detach().numpy().astype(np.float32),
            L[3].weight.detach().numpy().reshape(-1).astype(np.float32),
            L[3].bias.detach().numpy().astype(np.float32))


def head_forward(head, x):
    """The exported head in numpy: BF16 weights, BF16-rounded activations between layers
    (the tensor-core operands), FP32 accumulation, as the CUDA kernels compute it."""
    w1, w2, w3, b1, b2, b3, w4, b4 = head
    a = np.zeros((x.shape[0], K1), np.float32)
    a[:, :2] = x
    a = bf16_to_f32(bf16_round(a))
    h = np.maximum(a @ bf16_to_f32(w1).reshape(HIDDEN, K1).T + b1, 0)
    h = np.maximum(bf16_to_f32(bf16_round(h)) @ bf16_to_f32(w2).reshape(HIDDEN, HIDDEN).T + b2, 0)
    h = np.maximum(bf16_to_f32(bf16_round(h)) @ bf16_to_f32(w3).reshape(HIDDEN, HIDDEN).T + b3, 0)
    return h @ w4 + b4[0]


def write_heads(path, heads):
    with open(path, "wb") as f:
        f.write(b"BIAHEAD1")
        f.write(struct.pack("<II", 1, len(heads)))
        for w1, w2, w3, b1, b2, b3, w4, b4 in heads:
            for w in (w1, w2, w3):
                f.write(np.ascontiguousarray(w, "<u2").tobytes())
            for b in (b1, b2, b3, w4, b4, np.zeros(3, np.float32)):
                f.write(np.ascontiguousarray(b, "<f4").tobytes())


def read_heads(path=OUT):
    """The heads in the file as tuples of numpy arrays (see export_head)."""
    raw = open(path, "rb").read()
    assert raw[:8] == b"BIAHEAD1"
    version, nheads = struct.unpack("<II", raw[8:16])
    off = 16
    heads = []
    for _ in range(nheads):
        ws = []
        for shape in ((HIDDEN, K1), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN)):
            cnt = shape[0] * shape[1]
            ws.append(np.frombuffer(raw, "<u2", cnt, off).reshape(shape))
            off += 2 * cnt
        fs = []
        for cnt in (HIDDEN, HIDDEN, HIDDEN, HIDDEN, 1, 3):
            fs.append(np.frombuffer(raw, "<f4", cnt, off))
            off += 4 * cnt
        heads.append(tuple(ws) + tuple(fs[:5]))
    return heads


def write_records(path, records):
    """learned_heads.bin from head records (bytes of 19472 each, as bia_trainer_export
    returns them)."""
    with open(path, "wb") as f:
        f.write(b"BIAHEAD1")
        f.write(struct.pack("<II", 1, len(records)))
        for r in records:
            f.write(r)


def guess_error(head, x, y, scale):
    """|head guess - solved anomaly| (radians) on samples (x, y) of one head."""
    guess = head_forward(head, x.astype(np.float32)) * scale
    return np.abs(guess - y * scale)


def train_device(samples=1 << 22, epochs=24, seed=0, batch=4096, lr=2e-3, device=0, log=print):
    """Both heads trained on the GPU (bia_trainer_*).  Returns (records, info): the head
    records in file order and per head the epoch losses and the training time."""
    import time as _time

    from . import BIASolver
    records, info = [], []
    with BIASolver(device=device) as solver:
        for head in (0, 1):
            t0 = _time.perf_counter()
            tr = solver.trainer(head, samples, seed + head)
            t1 = _time.perf_counter()
            losses = tr.train(epochs, batch, lr)
            t2 = _time.perf_counter()
            records.append(tr.export())
            tr.close()
            info.append({"samples_s": t1 - t0, "train_s": t2 - t1, "losses": losses.tolist()})
            log(f"  head {head}: samples {t1 - t0:.2f} s, {epochs} epochs {t2 - t1:.2f} s, "
                f"final mse {losses[-1]:.3e}")
    return records, info


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=1 << 22)
    ap.add_argument("--epochs", type=int, default=24)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=OUT)
    ap.add_argument("--torch", action="store_true", help="train with torch on the CPU instead of the GPU")
    args = ap.parse_args()
    log = lambda s: print(s, flush=True)
    if not args.torch:
        t0 = time.time()
        records, _ = train_device(args.samples, args.epochs, args.seed, log=log)
        write_records(args.out, records)
        rng = np.random.default_rng(args.seed + 100)
        ell, hyp = make_samples(200000, rng)
        for (name, (x, y, e, M), scale), head in zip((("elliptic", ell, np.pi), ("hyperbolic", hyp, HYP_OUT)),
                                                     read_heads(args.out)):
            err = guess_error(head, x, y, scale)
            log(f"  {name} head (BF16) guess error on new samples: median {np.median(err):.2e}, "
                f"p99 {np.quantile(err, 0.99):.2e}, max {err.max():.2e}")
        log(f"wrote {args.out} ({os.path.getsize(args.out)} bytes, {time.time() - t0:.0f} s)")
        return
    rng = np.random.default_rng(args.seed)
    t0 = time.time()
    ell, hyp = make_samples(args.samples, rng)
    log(f"samples: {args.samples} per head ({time.time() - t0:.1f} s)")
    heads = []
    for name, (x, y, e, M), scale in (("elliptic", ell, np.pi), ("hyperbolic", hyp, HYP_OUT)):
        log(f"training the {name} head")
        net = train_head(x, y, args.epochs, args.seed, log)
        head = export_head(net)
        guess = head_forward(head, x[:200000].astype(np.float32)) * scale
        err = np.abs(guess - y[:200000] * scale)
        log(f"  exported (BF16) guess error: median {np.median(err):.2e}, "
            f"p99 {np.quantile(err, 0.99):.2e}, max {err.max():.2e}")
        heads.append(head)
    write_heads(args.out, heads)
    log(f"wrote {args.out} ({os.path.getsize(args.out)} bytes, {time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
