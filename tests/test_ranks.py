"""The multi-rank bench path on CPU (gloo, world size 2): ranks pack disjoint universe
sets (seeds offset per rank), the job time is the slowest rank's and the candidates
add up; the reference arm runs on rank 0 only."""

import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "universe-generator_b200"))
    import bench
    import ugb200

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        us, _ = bench.workloads("c3", ugb200, 1000 * rank)
        t_ms, cands = bench.combine_ranks(100.0 + 50.0 * rank, 1000 + rank, dist, "cpu")
        out.put((rank, t_ms, cands, [u.seed for u in us]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_and_shard():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t_ms, cands, _ in res:
        assert t_ms == 150.0 and cands == 2001
    assert not set(res[0][3]) & set(res[1][3])  # each rank its own universes


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import argparse

    import bench

    args = argparse.Namespace(workload="c3", steps=1, warmup=1)
    assert bench.reference_arm(args, 1, 2) == 0
    assert capsys.readouterr().out == ""
