"""Multi-rank decomposition on CPU: gloo, world size 2 (no GPU).

Each rank accumulates its contiguous share of the band pairs with the CPU oracle,
the partial packed chi are summed with the same reduction the GPU ranks use, and
rank 0 checks the sum against the single-process result.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from project1_b200.parallel import pair_shard, q_shard, reduce_partial


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    rng = np.random.default_rng(3)
    nbas, nk, no, nu, nw = 20, 3, 4, 5, 3
    npair = nk * no * nu
    m = np.asfortranarray((rng.standard_normal((npair, nbas)) + 1j * rng.standard_normal((npair, nbas))) / 5)
    d = rng.uniform(0.5, 30, npair)
    om = np.linspace(0.5, 40, nw)
    return m, d, om, no * nu


def _worker(rank, world, port, q):
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, d, om, block = _case()
        lo, hi = pair_shard(m.shape[0], world, rank, block=block)
        part = oracle.chi0(m[lo:hi], oracle.weights(d[lo:hi], om, None, 0.5))
        t = torch.from_numpy(np.ascontiguousarray(part.T))  # (nw, npack) complex
        t = torch.view_as_real(t).contiguous()
        reduce_partial(t, dst=0)
        if rank == 0:
            full = oracle.chi0(m, oracle.weights(d, om, None, 0.5))
            got = torch.view_as_complex(t).numpy().T
            q.put(float(np.max(np.abs(got - full)) / np.max(np.abs(full))))
    finally:
        dist.destroy_process_group()


def test_pair_sharded_reduction_matches_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert q.get(timeout=10) < 1e-13


def test_pair_shard_covers_all_pairs_in_k_blocks():
    for world in (1, 2, 3, 8):
        spans = [pair_shard(64 * 16000, world, r, block=16000) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == 64 * 16000
        for (a, b), (c, _) in zip(spans, spans[1:]):
            assert b == c and (b % 16000) == 0


def test_q_shard_balances_uneven_q_points():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1, 10, 32) ** 2
    for world in (2, 4, 8):
        parts = q_shard(costs, world)
        assert sorted(q for p in parts for q in p) == list(range(32))
        loads = [sum(costs[q] for q in p) for p in parts]
        assert max(loads) <= 4 / 3 * max(sum(costs) / world, max(costs)) + 1e-9
