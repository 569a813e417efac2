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

from project1_b200.parallel import (chi0_batched_q_sharded, freq_shard, pair_shard, q_cost, q_shard,
                                    reduce_partial, reduce_scatter_partial)


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


def _worker_scatter(rank, world, port, q):
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, d, om, block = _case()
        om = np.linspace(0.5, 40, 5)          # 5 frequencies: uneven over 2 or 3 ranks
        lo, hi = pair_shard(m.shape[0], world, rank, block=block)
        part = oracle.chi0(m[lo:hi], oracle.weights(d[lo:hi], om, None, 0.5))
        t = torch.view_as_real(torch.from_numpy(np.ascontiguousarray(part.T))).contiguous()
        mine = torch.view_as_complex(reduce_scatter_partial(t)).numpy()
        full = oracle.chi0(m, oracle.weights(d, om, None, 0.5)).T
        f0, f1 = freq_shard(5, world, rank)
        q.put((rank, mine.shape[0] == f1 - f0, float(np.max(np.abs(mine - full[f0:f1])) / np.max(np.abs(full)))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_reduce_scatter_leaves_each_rank_its_frequencies(world):
    """The partial chi of the pair shards, reduce-scattered over frequencies: every
    rank holds the full sum for its own frequencies (uneven split: 5 over 2 or 3)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_scatter, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert [g[0] for g in got] == list(range(world))
    assert all(g[1] for g in got)
    assert max(g[2] for g in got) < 1e-13


class _FakeBatchCtx:
    def __init__(self):
        self.calls = []

    def chi0_batched(self, qs, omega, **kw):
        self.calls.append(([q["nbas"] for q in qs], kw))


def test_q_sharded_batch_runs_each_q_on_one_rank():
    """Every q point runs on exactly one rank, in one batched call per rank, with the
    longest-first balance of q_shard."""
    rng = np.random.default_rng(5)
    qs = [dict(nbas=int(n), npair=int(p)) for n, p in zip(rng.integers(600, 1800, 32),
                                                        rng.integers(10000, 2000000, 32))]
    for world in (1, 2, 4, 8):
        seen = []
        loads = []
        for rank in range(world):
            c = _FakeBatchCtx()
            mine = chi0_batched_q_sharded(c, qs, None, world, rank, precision="split")
            assert len(c.calls) == (1 if mine else 0)
            if mine:
                assert c.calls[0][0] == [qs[i]["nbas"] for i in mine]
                assert c.calls[0][1] == {"precision": "split"}
            seen += mine
            loads.append(sum(q_cost(qs[i]) for i in mine))
        assert sorted(seen) == list(range(32))
        costs = [q_cost(q) for q in qs]
        assert max(loads) <= 4 / 3 * max(sum(costs) / world, max(costs)) + 1e-6 * sum(costs)
