"""The benchmark's multi-rank plumbing on CPU: two gloo ranks (no GPU).

bench.py runs one replica per rank and reports the maximum time over ranks;
this checks its max-reduction and barrier helpers, and the reference arm's
JSON line on a small case."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      WCNS_DIST_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    r, w = bench.dist_init(world)
    assert (r, w) == (rank, world)
    bench.dist_barrier(w)
    m = bench.dist_max(1.5 + rank, w)
    out.put((rank, m))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_gloo_two_ranks_max_over_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 2.5, 1: 2.5}


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--case", "small_plate",
                        "--steps", "2", "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "Mcell-steps/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
