"""The multi-GPU path of bench.py on the host: replicas only (one independent system per
rank, no data-path collective), timed as the maximum over ranks.  Two gloo ranks run the
bench's own process-group set-up and max-over-ranks reduction; the reference arm under
torchrun runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_PROGRAM = r"""
import os, sys, json
sys.path.insert(0, os.environ["BIA_ROOT"])
import torch
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist = bench._init_dist(world)
dist.barrier()
t = bench._max_over_ranks(dist, 1.5 + 2.0 * rank, torch.device("cpu"))
print(json.dumps({"rank": rank, "backend": dist.get_backend(), "max": t}), flush=True)
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), BIA_ROOT=ROOT, CUDA_VISIBLE_DEVICES="")
    return env


def test_two_gloo_ranks_take_the_max_over_ranks():
    port = _free_port()
    procs = [subprocess.Popen([sys.executable, "-c", RANK_PROGRAM], env=_env(r, 2, port), cwd=ROOT,
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True) for r in range(2)]
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    assert all(o["backend"] == "gloo" and o["max"] == 3.5 for o in outs)


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun every rank but 0 exits 0 without work or output."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], env=_env(1, 2, _free_port()), cwd=ROOT,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
