"""Replica shards across GPUs (one process per GPU, no data-path collective).

Temperature exchange only mixes replicas of one (protein conformer, ligand conformer) group
(reference src/kernel_cuda_l1_exchangereplicas.cu:29-77), so a batch splits across ranks by whole
complexes, or a single complex by whole protein conformers, and the ranks never talk during Monte
Carlo. Each complex keeps the RNG stream id it has in the full batch (its batch index), so a shard
reproduces its part of the single-GPU batch bit for bit. Timing is reduced as the max over ranks.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def complex_cost(n_rep: int, lna: int, pnp: int) -> int:
    """Pair work per step of one complex (replicas x ligand atoms x protein points)."""
    return int(n_rep) * int(lna) * int(pnp)


def assign_complexes(costs: Sequence[int], world: int) -> List[List[int]]:
    """Longest-processing-time assignment of complexes to ranks: every complex on exactly one
    rank, ranks' totals balanced greedily; deterministic (ties to the lower rank / index)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += int(costs[i])
    for lst in out:
        lst.sort()
    return out


def split_protein_conformers(n_prt: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous, group-aligned split of one complex by protein conformer: [p0, p1)."""
    if not 0 <= rank < world:
        raise ValueError("rank outside [0, world)")
    base, extra = divmod(n_prt, world)
    p0 = rank * base + min(rank, extra)
    return p0, p0 + base + (1 if rank < extra else 0)


def shard_batch(complexes, world: int, rank: int):
    """(complexes of this rank, their RNG stream ids = batch indices)."""
    costs = [complex_cost(c.n_rep, c.lna, c.pnp) for c in complexes]
    mine = assign_complexes(costs, world)[rank]
    return [complexes[i] for i in mine], list(mine)


def max_over_ranks(value: float, dist=None) -> float:
    """Max of a per-rank time over the process group (identity without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    backend = dist.get_backend()
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
