"""The N > 1 plumbing of bench.py on CPU ranks (gloo, world size 2): the
replicas' step time is the slowest rank's and the job's rate counts every
rank's interactions; the reference arm runs on rank 0 only."""
import os

import pytest


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms, value = bench.job_rate(10.0 * (rank + 1), 1.0e9, world)
    q.put((rank, ms, value))
    dist.barrier()
    dist.destroy_process_group()


def test_job_rate_is_max_over_ranks():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value in got:
        assert ms == 20.0                      # the slower rank's time on every rank
        assert value == pytest.approx(2 * 1.0e9 / 0.020)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import argparse
    import bench
    args = argparse.Namespace(steps=1, warmup=0, tol=0.0)
    assert bench.run_reference(args, bench.WORKLOADS["box32"], 1, 2) == 0
    assert capsys.readouterr().out == ""
