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


class _FakeSweepSolver:
    """Stands in for a GPU context: the cross sections of a wavelength are a
    fixed function of omega and the refractive indices."""

    def sweep(self, omegas, ri, srcs, precision, tol, maxit):
        import numpy as np
        ns = len(srcs)
        csca = np.outer(omegas, np.arange(1, ns + 1)) + np.abs(ri[:, :1])
        cabs = np.outer(omegas ** 2, np.ones(ns))
        return csca, cabs, np.zeros(len(omegas), dtype=np.int32)


def _shard_worker(rank, world, port, out):
    sys.path.insert(0, os.path.join(ROOT, "for90-mom2_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import numpy as np
    import torch.distributed as dist
    from datetime import timedelta
    from mom_b200 import shard
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    n = 7
    om = np.linspace(1.0, 2.0, n)
    ri = np.stack([np.ones(n), 1.5 + 0.1j * np.arange(n)], axis=1)
    srcs = [dict(type="pw", theta=0.0, phi=0.0, psi=0.0)] * 3
    csca, cabs = shard.sweep(_FakeSweepSolver(), om, ri, srcs, 1, rank, world)
    mine = shard.sources(list(range(5)), rank, world)
    out[rank] = (csca.tolist(), cabs.tolist(), mine)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_sweep_gathers_every_wavelength_gloo():
    """Wavelengths split round-robin over 2 ranks (no data-path collective); the
    all-gathered cross sections equal the unsharded sweep on every rank, and the
    right-hand-side columns split into disjoint shares."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "for90-mom2_b200"))
    from mom_b200 import shard
    world = 2
    port = 29500 + (os.getpid() + 17) % 1000
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_shard_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    n = 7
    om = np.linspace(1.0, 2.0, n)
    ri = np.stack([np.ones(n), 1.5 + 0.1j * np.arange(n)], axis=1)
    ref_csca, ref_cabs, _ = _FakeSweepSolver().sweep(om, ri, [None] * 3, 1, 0, 0)
    for r in range(world):
        assert np.allclose(res[r][0], ref_csca) and np.allclose(res[r][1], ref_cabs)
    assert sorted(res[0][2] + res[1][2]) == list(range(5)) and not set(res[0][2]) & set(res[1][2])
    for nn in (0, 1, 5, 8):
        for w in (1, 2, 3):
            idx = np.concatenate([shard.shard(nn, r, w) for r in range(w)])
            assert sorted(idx.tolist()) == list(range(nn))
    with pytest.raises(ValueError):
        shard.shard(4, 2, 2)
