"""The multi-rank host logic of bench.py on CPU (gloo, world size 2, no GPU):
the max-over-ranks step time every rank receives, and a two-process torchrun
launch of the reference arm, where rank 0 alone measures and prints."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(REPO))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        q.put((rank, got))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 15.0, 1: 15.0}


def test_reference_arm_under_torchrun_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(REPO / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--iters", "1", "--size", "32"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    # stdout carries exactly the one JSON line (the reference's own printf
    # diagnostics go to stderr)
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1 and lines[0].startswith("{"), r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert "unavailable" in d or (d["value"] > 0 and d["n_gpus"] == 2)
