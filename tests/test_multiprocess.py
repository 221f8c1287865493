"""World-size-2 checks of bench.py's replica path on CPU (gloo): the step time
is the max over ranks and the job value counts every rank's solves."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    local_ms = 100.0 + 50.0 * rank
    mx = bench.reduce_max(local_ms, world, "cpu")
    out[rank] = (mx, bench.replica_value(mx, world))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_max_over_ranks_gloo():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == (150.0, world * 1000.0 / 150.0)


def test_reference_arm_other_ranks_exit_quietly(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps, warmup, subdiv = 1, 0, 1
    assert bench.run_reference(A(), rank=1, world=2) == 0
    assert capsys.readouterr().out == ""
