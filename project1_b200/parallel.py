"""Multi-GPU decomposition of the polarisation: one process per GPU.

Two decompositions from the reference:
  * pair sharding: the band pairs (k, occ, unocc) of one q point are split into
    contiguous blocks over ranks, as `Mblocks` splits them over MPI ranks
    (src/susceptibility.f:632-642). Every rank accumulates a full partial chi
    and one reduction sums them (`Mreduce`, :2264-2293).
  * q sharding: independent q points go to different ranks, as the MPIKPT
    virtual nodes do (src/correlation.f:293-339). No collective is needed.

The reduction runs on torch.distributed (NCCL on GPUs, gloo on CPU). No kernel
reads another GPU's memory.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple


def pair_shard(npair: int, world: int, rank: int, block: int = 1) -> Tuple[int, int]:
    """[lo, hi) of the pairs owned by `rank`: contiguous, sizes differing by at most
    one `block` (e.g. nocc*nunocc to keep whole k points together)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    nblk = (npair + block - 1) // block
    lo_b = rank * nblk // world
    hi_b = (rank + 1) * nblk // world
    return min(npair, lo_b * block), min(npair, hi_b * block)


def q_shard(costs: Sequence[float], world: int) -> List[List[int]]:
    """Assigns q points to ranks, longest first to the least loaded rank (LPT),
    which keeps the largest rank load within 4/3 of the optimum."""
    loads = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for q in sorted(range(len(costs)), key=lambda i: -costs[i]):
        r = min(range(world), key=lambda i: loads[i])
        out[r].append(q)
        loads[r] += costs[q]
    for lst in out:
        lst.sort()
    return out


def reduce_partial(chi, dst: int = 0, group=None, all_ranks: bool = False) -> None:
    """Sums the partial packed chi of every rank into rank `dst` (or all ranks)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return
    if all_ranks:
        dist.all_reduce(chi, group=group)
    else:
        dist.reduce(chi, dst, group=group)


def chi0_pair_sharded(ctx, cprod_shard, ediff_shard, omega, susceph, scale_all: float = 1.0,
                      precision: str = "split", stream=None, dst: int = 0,
                      group=None) -> Optional[dict]:
    """One rank's share of a pair-sharded chi0: local accumulation on its GPU, then
    the reduction to `dst`. `susceph` must be zeroed by the caller on every rank."""
    st = ctx.chi0_accumulate_dev(cprod_shard, ediff_shard, omega, susceph, scale_all=scale_all,
                                 precision=precision, stream=stream, stats=True)
    reduce_partial(susceph, dst=dst, group=group)
    return st
