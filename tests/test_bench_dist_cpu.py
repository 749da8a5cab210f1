"""The multi-GPU plumbing of bench.py on CPU: two `gloo` ranks (the GPU runs
use one process per GPU over NCCL with the same code path): rank setup from
the torchrun environment, the max-over-ranks timing, the barrier, the
whole-job throughput of weak-scaled replicas, and the reference arm under
torchrun (rank 0 alone prints one JSON line, the other rank exits 0)."""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, REPO)
    import bench
    r, w, dist = bench.dist_setup(world, backend="gloo")
    bench.barrier(dist)
    m = bench.max_over_ranks(10.0 + 5.0 * r, dist)  # rank 1 is the slow one
    v = bench.job_throughput(1e12, 4, w, m)
    bench.barrier(dist)
    dist.destroy_process_group()
    out.put((r, w, m, v))


def test_two_gloo_ranks_share_the_max_time():
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, *_ in res] == [0, 1]
    for _, w, m, v in res:
        assert w == 2 and m == 15.0
        # 2 replicas x 4 steps x 1 TFLOP in 15 ms
        assert v == pytest.approx(2 * 4 * 1e12 / 15e-3 / 1e12)


def test_single_process_needs_no_process_group():
    sys.path.insert(0, REPO)
    import bench
    env = dict(os.environ)
    os.environ.pop("RANK", None)
    try:
        assert bench.dist_setup(2) == (0, 1, None)
        assert bench.max_over_ranks(3.5, None) == 3.5
    finally:
        os.environ.clear()
        os.environ.update(env)


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--nd", "4096", "--nb", "64"]
    r = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["config"]["Nd"] == 4096 and d["config"]["nb"] == 64
