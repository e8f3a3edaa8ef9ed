"""The N > 1 path of bench.py on the CPU with gloo ranks (no GPU): ranks score
disjoint seeded batches, the step time is the maximum over ranks, and the
reference arm runs on rank 0 alone."""

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import bench
rank, world, local = bench.dist_setup()
got = bench.all_max(10.0 + rank, world)
bench.barrier(world)
seed = 0x5EED_0000 + 1000003 * rank
print(json.dumps({"rank": rank, "world": world, "max": got, "seed": seed}), flush=True)
import torch.distributed as dist
dist.destroy_process_group()
"""


def test_max_over_ranks_and_disjoint_seeds():
    port = _port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, str(ROOT)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert {o["rank"] for o in outs} == {0, 1} and all(o["world"] == 2 for o in outs)
    assert all(o["max"] == 11.0 for o in outs)
    assert outs[0]["seed"] != outs[1]["seed"]


def test_reference_arm_under_torchrun_prints_one_line():
    port = _port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--seconds", "1"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [line for line in r.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
