"""bench.py's multi-process plumbing on CPU: world size 2 over gloo (no GPU).

The path has no data-path collective: `bench.py --gpus N` runs N replicas, one process per
GPU, each reconstructing its own scan; only the step time is reduced (the slowest rank's) and
the whole-job GUPS is N x updates / that time. The reference arm runs on rank 0 alone.
"""
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


def _worker(rank, ws, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(ws),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    w, r, _ = bench.dist_setup(ws, backend="gloo")
    bench.barrier(w)
    # rank r's step takes 10 (r + 1) ms: every rank must report the slowest
    slowest = bench.max_over_ranks(10.0 * (r + 1), w)
    gups = bench.replica_gups(1_000_000_000, slowest, w)
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, w, slowest, gups))


def test_replica_timing_over_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    for _, w, slowest, gups in out:
        assert w == 2
        assert slowest == 20.0                      # the slower rank's time, on every rank
        assert gups == pytest.approx(2 * 1e9 / 0.020 / 1e9)  # two replicas' updates


def test_reference_arm_runs_on_rank_0_only():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "1"], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""  # rank 1 exits without work and prints nothing
