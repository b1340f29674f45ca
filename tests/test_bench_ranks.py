"""The benchmark's multi-rank path on the CPU (gloo, world size 2): replicas
report all ranks' units over the slowest rank's time, and the reference arm
prints one line from rank 0 while the other rank exits without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), GPV_BENCH_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    w, r, _ = bench.dist_setup(None)
    t_ms = 100.0 + 50.0 * r  # rank 1 is the slower one
    value, t_max = bench.replica_rate(1000, 4, t_ms, w)
    bench.barrier(w)
    q.put((r, value, t_max))
    dist.destroy_process_group()


def test_replica_rate_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for r, value, t_max in got:
        assert t_max == 150.0
        assert value == pytest.approx(2 * 1000 * 4 / 0.150)


def test_reference_arm_under_torchrun_prints_one_line():
    env = dict(os.environ, GPV_BENCH_BACKEND="gloo", CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--config", "1", "--scale-down", "8",
           "--cpu-seconds", "0.3"]
    out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
