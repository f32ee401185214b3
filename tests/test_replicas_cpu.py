"""The N > 1 path of bench.py on the host: ranks as gloo processes
(world size 2, 127.0.0.1).  The step of one domain has no data-path
collective (replicas only), so what N > 1 adds is the rank plumbing:
dist_setup, the barriers, the max over ranks of the per-rank times, and
rank 0 alone printing the line (the other ranks exit 0 without output).
"""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "aeolus.jl_b200")]
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup()
    bench.barrier(w)
    m = bench.max_over_ranks(10.0 * (r + 1), w)
    out.put((r, w, m, dist.get_backend()))
    bench.barrier(w)
    dist.destroy_process_group()


def test_rank_plumbing_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == 2 and g[2] == 20.0 and g[3] == "gloo" for g in got)


def test_reference_arm_prints_one_line_from_rank_zero():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--workload", "tracer", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
