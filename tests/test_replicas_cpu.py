"""CPU: the multi-rank host logic of bench.py (replicas, one system per rank) on gloo with
two ranks: barriers, the max over ranks of the per-rank time, and the reference arm
printing only on rank 0."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.rank_barrier(world)
        local = 1.5 + 2.0 * rank  # rank 1 is the slow replica
        got = bench.rank_max(local, world, torch.device("cpu"))
        bench.rank_barrier(world)
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_rank_max_takes_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29400 + os.getpid() % 500
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 3.5, 1: 3.5}


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.rank_max(2.25, 1, None) == 2.25
    bench.rank_barrier(1)


@pytest.mark.parametrize("rank", ["0", "1"])
def test_reference_arm_prints_only_on_rank0(rank):
    # tiny system so the host-side reference run finishes in seconds
    env = dict(os.environ, RANK=rank, WORLD_SIZE="2", LOCAL_RANK=rank)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--n", "256", "--nrhs", "4", "--steps", "1", "--warmup", "0",
                        "--gpus", "2"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if rank == "1":
        assert lines == []
    else:
        line = json.loads(lines[-1])
        assert line["impl"] == "reference" and line["unit"] == "s"
        assert line["higher_is_better"] is False and line["value"] > 0
        assert line["cpu_baseline"]["kind"] in ("reference", "port")
