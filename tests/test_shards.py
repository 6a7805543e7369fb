"""The multi-GPU split of one BIA step into shards (bia_shard_columns, bia_step_shard,
bia_apply_update), checked on the host: the column partition covers every pair once with
balanced pair counts, and two gloo ranks that each sum their shard's pairs (here with the
oracle), all-reduce the sums and apply drift and update reproduce the oracle's whole step.
On a GPU box each rank runs bia_step_shard and the sums cross NVLink in one NCCL
all-reduce of 6n doubles (BIASolver.step_distributed); tests/test_gpu_shards.py checks the
shard kernels on one GPU."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from bia_3d_gpu_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def shard_pair_sums(state, eps, dt, c0, c1, q=None):
    """The pair sums of shard columns [c0, c1): pairs (i, j), i < j, j in [32 c0, 32 c1).
    With the particle order reversed those pairs are the oracle's rows (all partners after
    them) of the shard's particles; the pair update is antisymmetric, so the reversed rows'
    sums are the shard's."""
    import oracle
    n = state.shape[1]
    rev = np.ascontiguousarray(state[:, ::-1])
    qrev = np.ascontiguousarray(q[::-1]) if q is not None else None
    js = np.arange(32 * c0, min(32 * c1, n))
    rows = n - 1 - js
    rows = rows[rows < n - 1]
    d, _, _ = oracle.bia_rows(rev, eps, dt, rows, q=qrev)
    return np.ascontiguousarray(d[:, ::-1])


@pytest.mark.parametrize("n", [1, 31, 33, 1000, 32768, 131072])
@pytest.mark.parametrize("nshards", [1, 2, 3, 8])
def test_shard_columns_partition_the_pairs(n, nshards):
    nb = (n + 31) // 32
    bounds = [capi.shard_columns(n, s, nshards) for s in range(nshards)]
    assert bounds[0][0] == 0 and bounds[-1][1] == nb
    for (a0, a1), (b0, b1) in zip(bounds, bounds[1:]):
        assert a1 == b0 and a0 <= a1
    blocks = [c1 * (c1 + 1) // 2 - c0 * (c0 + 1) // 2 for c0, c1 in bounds]
    assert sum(blocks) == nb * (nb + 1) // 2
    if nb >= 8 * nshards:  # whole columns: within one column of the even split
        assert max(blocks) - min(blocks) <= 2 * nb


def test_shard_sums_add_up_to_the_oracle_step():
    import oracle
    from bia_3d_gpu_b200 import initial
    s, eps = initial.gravity_ball(300, seed=90)
    dt = 1e-3
    total = sum(shard_pair_sums(s, eps, dt, *capi.shard_columns(300, r, 3)) for r in range(3))
    ref, disp, _ = oracle.bia_step(s, eps, dt)
    got = s.copy()
    got[:3] += total[:3] + s[3:] * dt
    got[3:] += total[3:]
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-13


RANK_PROGRAM = r"""
import os, sys, json
sys.path.insert(0, os.environ["BIA_ROOT"])
sys.path.insert(0, os.path.join(os.environ["BIA_ROOT"], "tests"))
import numpy as np
import torch
import torch.distributed as dist
import oracle
from bia_3d_gpu_b200 import capi, initial
from test_shards import shard_pair_sums
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo")
s, eps, q = initial.coulomb_cube(400, seed=91, dmin=1e-2)
dt = 1e-5
c0, c1 = capi.shard_columns(s.shape[1], rank, world)
sums = torch.tensor(shard_pair_sums(s, eps, dt, c0, c1, q=q))
dist.all_reduce(sums)
new = s.copy()
new[:3] += sums[:3].numpy() + s[3:] * dt
new[3:] += sums[3:].numpy()
ref, _, _ = oracle.bia_step(s, eps, dt, q=q)
err = float(np.linalg.norm(new - ref) / np.linalg.norm(ref))
print(json.dumps({"rank": rank, "columns": [c0, c1], "err": err}), flush=True)
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def test_two_gloo_ranks_all_reduce_shard_sums():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), BIA_ROOT=ROOT, CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_PROGRAM], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=300) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e
    res = [json.loads(o.strip().splitlines()[-1]) for o, _ in outs]
    assert res[0]["columns"][1] == res[1]["columns"][0]
    for r in res:
        assert r["err"] <= 1e-13, r
