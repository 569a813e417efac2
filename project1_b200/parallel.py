"""Multi-GPU decomposition of the polarisation: one process per GPU.

Two decompositions from the reference:
  * pair sharding: the band pairs (k, occ, unocc) of one q point are split into
    contiguous blocks over ranks, as `Mblocks` splits them over MPI ranks
    (src/susceptibility.f:632-642). Every rank accumulates a full partial chi
    and one reduction sums them (`Mreduce`, :2264-2293).
  * q sharding: independent q points go to different ranks, as the MPIKPT
    virtual nodes do (src/correlation.f:293-339). No collective is needed.

The pair-sharded partial chi is reduced to one rank, all-reduced, or
reduce-scattered over frequencies (each rank keeps the frequencies it goes on to
build and invert the dielectric matrix for). The collectives run on
torch.distributed (NCCL on GPUs, gloo on CPU). No kernel reads another GPU's memory.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


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


def freq_shard(nw: int, world: int, rank: int) -> Tuple[int, int]:
    """[lo, hi) of the frequencies a rank keeps after a reduce-scatter."""
    return pair_shard(nw, world, rank)


def reduce_scatter_partial(chi, group=None):
    """Sums the partial chi (nw, ...) of every rank and leaves each rank the rows of its
    own frequencies (`freq_shard`): downstream, the dielectric matrix and its inverse
    are per frequency (src/correlation.f:614-647), so no rank needs the others' rows.
    NCCL reduce-scatters (rows padded to a multiple of the world size); other backends
    all-reduce and slice. Returns the rank's rows (a new tensor)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return chi.clone()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    nw = chi.shape[0]
    lo, hi = freq_shard(nw, world, rank)
    if dist.get_backend(group) == "nccl":
        per = (nw + world - 1) // world
        src = chi
        if per * world != nw:
            src = torch.zeros((per * world,) + tuple(chi.shape[1:]), dtype=chi.dtype, device=chi.device)
            # rank r's rows [lo_r, hi_r) go to block r
            for r in range(world):
                a, b = freq_shard(nw, world, r)
                src[r * per:r * per + (b - a)] = chi[a:b]
        out = torch.empty((per,) + tuple(chi.shape[1:]), dtype=chi.dtype, device=chi.device)
        dist.reduce_scatter_tensor(out, src.contiguous(), group=group)
        return out[:hi - lo].clone()
    dist.all_reduce(chi, group=group)
    return chi[lo:hi].clone()


def chi0_pair_sharded(ctx, cprod_shard, ediff_shard, omega, susceph, scale_all: float = 1.0,
                      precision: str = "split", stream=None, dst: int = 0,
                      group=None, scatter: bool = False):
    """One rank's share of a pair-sharded chi0: local accumulation on its GPU, then
    the reduction to `dst` (stats returned), or with `scatter` the reduce-scatter over
    frequencies (this rank's rows returned with the stats). `susceph` must be zeroed
    by the caller on every rank."""
    st = ctx.chi0_accumulate_dev(cprod_shard, ediff_shard, omega, susceph, scale_all=scale_all,
                                 precision=precision, stream=stream, stats=True)
    if scatter:
        return reduce_scatter_partial(susceph, group=group), st
    reduce_partial(susceph, dst=dst, group=group)
    return st


def q_cost(q: dict) -> float:
    """Work of one q point of a batch: N_MB^2 x pairs."""
    return float(q["nbas"]) ** 2 * float(q["npair"])


def chi0_batched_q_sharded(ctx, qs: Sequence[dict], omega, world: int, rank: int, **kw) -> List[int]:
    """The q points of a batch spread over ranks with no collective, as the reference's
    MPIKPT virtual nodes take whole q points (src/correlation.f:293-339): rank `rank`
    runs the batch of its own q (longest-first assignment, `q_shard`) through
    `ctx.chi0_batched` and returns their indices; the other q's outputs are left
    untouched on this rank."""
    mine = q_shard([q_cost(q) for q in qs], world)[rank]
    if mine:
        ctx.chi0_batched([qs[i] for i in mine], omega, **kw)
    return mine
