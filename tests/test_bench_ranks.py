"""bench.py's multi-process contract on CPU (world size 2, gloo).

A multi-GPU run launches `bench.py --gpus N` under torchrun, one rank per GPU:
rank 0 alone prints the JSON line, the others exit 0, and device times are
the maximum over ranks. These tests run the parts of that path that need no
GPU: the reference arm under a two-rank torchrun, and the max-over-ranks
reduction over gloo.
"""

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_under_two_ranks_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), str(REPO / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["n_gpus"] == 2 and d["warmup"] == 3 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def _max_worker(rank: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE="2", LOCAL_RANK=str(rank))
    sys.path.insert(0, str(REPO))
    import bench

    ws, r, local = bench.dist_env()
    dist = bench.init_dist(ws, local)
    try:
        out.put((r, bench.allreduce_max(dist, 1.5 + r)))
    finally:
        dist.destroy_process_group()


@pytest.mark.skipif(sys.platform != "linux", reason="spawned gloo ranks")
def test_allreduce_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_max_worker, args=(r, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 2.5, 1: 2.5}
