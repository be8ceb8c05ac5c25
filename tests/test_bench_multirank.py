"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2).

The timed value of an N-rank run is the maximum over ranks of each rank's
device time, taken after a barrier; the CPU reference arm runs on rank 0 only
while the other ranks exit without work.  Both are exercised here with real
gloo process groups on 127.0.0.1.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    r, local, n = bench.dist_setup("gloo")
    bench.barrier(n)
    # rank-dependent "device times": the reported one is the slowest rank's
    t = 0.25 + 0.5 * r
    m = bench.max_over_ranks(t, n)
    bench.barrier(n)
    q.put((r, local, n, m))
    dist.destroy_process_group()


def test_max_over_ranks_and_barrier_gloo_world_size_2():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(ws))
    assert [g[0] for g in got] == [0, 1]
    assert all(g[2] == ws for g in got)
    assert all(g[3] == pytest.approx(0.75) for g in got)


def test_max_over_ranks_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(1.25, 1) == 1.25
    bench.barrier(1)


def test_reference_arm_under_torchrun_prints_one_line_from_rank_0():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1",
           "--lattice", "4,4,4,8"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference"
    assert rec["n_gpus"] == 2
    assert rec["higher_is_better"] is False
    assert rec["cpu_baseline"]["kind"] == "port"
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
    assert rec["value"] > 0
