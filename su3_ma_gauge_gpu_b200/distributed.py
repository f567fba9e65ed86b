"""Multi-GPU host logic: one process per GPU, gauge copies sharded across ranks.

Gauge copies (and the lattices of a batch) are independent, so the path shards
by instance with no data-path collective.  The reference's only parallelism
is an MPI t-slab decomposition of ONE lattice
(apps/MultiGPU_MPI/MultiGPU_MPI_Communicator.hxx:351-430); for batches of
copies that exchange is unnecessary.  The collectives used here are for
bookkeeping only: the max-over-ranks time, the sum of site updates, and the
best copy (argmax of the functional) across ranks.
"""
from __future__ import annotations

from dataclasses import dataclass


def shard(n_items: int, rank: int, world: int) -> list[int]:
    """Item indices rank `rank` owns: contiguous blocks, sizes differing by at most one."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def shard_weighted(weights: list[float], rank: int, world: int) -> list[int]:
    """Greedy longest-processing-time assignment of weighted items (e.g. V x expected sweeps)."""
    loads = [0.0] * world
    owner = [0] * len(weights)
    for i in sorted(range(len(weights)), key=lambda k: -weights[k]):
        r = min(range(world), key=lambda q: loads[q])
        owner[i] = r
        loads[r] += weights[i]
    return [i for i in range(len(weights)) if owner[i] == rank]


@dataclass
class JobTiming:
    ms: float            # max over ranks
    site_updates: float  # sum over ranks
    gsite_per_s: float


def reduce_timing(ms: float, site_updates: float, group=None, device=None) -> JobTiming:
    """Whole-job throughput: site updates of all ranks / slowest rank's time."""
    import torch
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        u = torch.tensor([site_updates], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        dist.all_reduce(u, op=dist.ReduceOp.SUM, group=group)
        ms, site_updates = float(t.item()), float(u.item())
    return JobTiming(ms, site_updates, site_updates / (ms * 1e-3) / 1e9)


def best_copy(gff: float, copy_id: int, group=None, device=None) -> tuple[float, int]:
    """(best functional, its copy id) over all ranks (the reference keeps the copy with the
    largest functional, apps/LandauGaugeFixingSU3_4D.cu:274-281)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return gff, copy_id
    world = dist.get_world_size(group)
    t = torch.tensor([gff, float(copy_id)], dtype=torch.float64, device=device)
    out = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    vals = [(float(o[0]), int(o[1])) for o in out]
    return max(vals, key=lambda v: (v[0], -v[1]))
