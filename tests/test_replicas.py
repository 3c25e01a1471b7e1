"""The multi-GPU form is replicas only: every rank searches its own copy of
the index with no data-path collective; the benchmark reports the total
queries of all ranks over the slowest rank's time. These tests run that host
logic as world_size-2 gloo process groups on the CPU."""
import os
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = 0.5 + rank  # rank 1 is the slow one
        slowest = bench.max_over_ranks(local, torch.device("cpu"))
        qps = bench.replica_qps(10000, 4, world, slowest)
        dist.barrier()
        q.put((rank, slowest, qps))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_throughput():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29511
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, qps in out:
        assert slowest == 1.5
        assert abs(qps - 2 * 10000 * 4 / 1.5) < 1e-6


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
