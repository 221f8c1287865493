"""Data-parallel sharding over ranks (one process per GPU, torch.distributed).

The solve has no data exchange at one wavelength; its natural shards are
independent units (the wavelength loop of solve_batch, solver.f90:76-142,
and the right-hand-side columns of one factorisation, solver.f90:116-127).
Each rank takes a round-robin share, solves it on its own GPU, and the
per-unit results (cross sections) are gathered into the original order:
no collective on the data path, one all-gather of the small results.
"""
import numpy as np


def shard(n, rank, world):
    """Indices of the units of rank `rank` among n units: rank, rank + world, ..."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    return np.arange(rank, n, world)


def gather(local, n, rank, world):
    """Gathers every rank's rows (local[i] belongs to unit shard(n, rank, world)[i])
    into an array of n rows in unit order, on every rank (all_gather over the
    default process group; the identity for world == 1)."""
    local = np.asarray(local)
    idx = shard(n, rank, world)
    if len(local) != len(idx):
        raise ValueError("%d rows for %d units of rank %d" % (len(local), len(idx), rank))
    if world == 1:
        return local.copy()
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, (rank, local))
    out = np.zeros((n,) + local.shape[1:], dtype=local.dtype)
    for r, rows in parts:
        out[shard(n, r, world)] = rows
    return out


def sweep(solver, omegas, ri_table, srcs, precision, rank=0, world=1, tol=1e-12, maxit=30):
    """Cross sections of a wavelength sweep sharded over ranks: rank r solves
    wavelengths r, r + world, ... (mom_gpu_sweep on its GPU) and every rank
    returns (csca, cabs) of all wavelengths, [nwl][nsrc] each.  ri_table:
    [nwl][ndom] complex refractive indices."""
    omegas = np.asarray(omegas, dtype=np.float64)
    ri_table = np.asarray(ri_table, dtype=np.complex128)
    mine = shard(len(omegas), rank, world)
    if len(mine):
        csca, cabs, _ = solver.sweep(omegas[mine], ri_table[mine], srcs, precision, tol, maxit)
    else:
        ns = len(srcs) if not isinstance(srcs, dict) else 1
        csca = cabs = np.zeros((0, ns))
    both = gather(np.stack([np.asarray(csca), np.asarray(cabs)], axis=1), len(omegas), rank, world)
    return both[:, 0], both[:, 1]


def sources(srcs, rank, world):
    """The right-hand-side columns (sources) of rank `rank`: one factorisation per
    rank (replicated), a share of the columns each."""
    return [srcs[i] for i in shard(len(srcs), rank, world)]
