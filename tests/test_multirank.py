"""The multi-rank path of bench.py (replicas: per-rank query streams, barrier
and max-over-ranks timing) as world_size-2 gloo ranks on CPU."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r'''
import os, sys
sys.path.insert(0, {root!r})
import bench
world, rank, local = bench.dist_setup("gloo")
assert world == 2 and rank in (0, 1)
# each rank draws its own query stream; rank 0 keeps the configuration's seed
assert bench.shard_seed(0) == bench.SEED and bench.shard_seed(1) != bench.SEED
bench.barrier(world)
t = bench.max_over_ranks(10.0 + rank, world)
assert t == 11.0, t
if rank == 0:
    print("OK", t)
import torch.distributed as dist
dist.destroy_process_group()
'''


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks():
    code = WORKER.format(root=ROOT)
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    assert "OK 11.0" in outs[0][0]


def test_reference_arm_two_gloo_ranks():
    """bench.py --impl reference under two ranks: rank 0 times the reference's
    own matcher and prints one JSON line; rank 1 exits 0 without work."""
    import json
    sys.path.insert(0, ROOT)
    from oracle import oracle
    if not os.path.exists(oracle.REF_MATCHER):
        pytest.skip("reference matcher not built (oracle/_ref)")
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r), LOCAL_WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                                       "--steps", "1", "--warmup", "1", "--filters", "20000", "--queries", "4096"],
                                      env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, cwd=ROOT))
    outs = [p.communicate(timeout=600) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    lines = [l for l in outs[0][0].splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert not [l for l in outs[1][0].splitlines() if l.startswith("{")]
