"""The multi-process side of bench.py on the host: two gloo ranks.

The bench runs N independent replicas, one per GPU, with a barrier on both
sides of the timed region and the time taken as the maximum over ranks; the
reference arm runs on rank 0 alone and the other ranks exit without work.
Both are checked here with two CPU processes (no GPU involved).
"""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys
from argparse import Namespace
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup(Namespace(impl="reference"))   # gloo
    bench.barrier(w)
    m = bench.allreduce_max(0.25 + r, w)   # each rank's "time": the job's is the slowest
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, w, m))


def test_replica_timing_helpers_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 1.25), (1, 2, 1.25)]


def test_reference_arm_prints_one_line_from_rank_zero(oracle_mod):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--workload", "single", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
