"""The multi-GPU plumbing of ``bench.py``: independent replicas, one per rank, a barrier around
the timed region and the job time taken as the maximum over ranks. Run here as two ``gloo``
ranks on the CPU (the same calls ``bench.py`` makes over NCCL)."""

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    try:
        bench.barrier(world)
        # each replica timed its own K steps; the job's time is the slowest replica's
        ms = [12.5, 17.25][rank]
        out[rank] = bench.reduce_max(ms, world, device="cpu")
        bench.barrier(world)
    finally:
        bench.dist_done(world)


def test_two_replicas_report_the_slowest_rank():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert dict(out) == {0: 17.25, 1: 17.25}


def test_reference_arm_runs_one_oracle_process_per_core():
    """``bench.py --impl reference``: the oracle's step in spawned single-threaded processes,
    one per requested core, timed together; the line reports their number and sums their
    throughput (CPU only, a 24^3 proxy here)."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                        "--steps", "3", "--warmup", "3", "--ref-size", "24", "--ref-procs", "2"],
                       capture_output=True, text=True, timeout=300, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["cpu_baseline"]["cores"] == 2
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert "replicas x2" in line["config"]["parallelism"]
