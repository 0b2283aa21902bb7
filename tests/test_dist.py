"""Multi-rank batch extraction, host side (CPU, gloo, world size 2).

The batch path shards geometries over ranks by cost and all-gathers the C
matrices (no data-path collective).  Here two gloo ranks run the sharding and
the gather with the oracle standing in for the per-GPU extraction; every rank
must end with the whole batch, in input order, equal to a one-rank run.
"""

import os
import socket

import numpy as np
import pytest

from fieldspice_b200.batch import capacitance_matrices, problem_cost, shard_by_cost


def test_shard_by_cost_is_balanced_and_deterministic():
    rng = np.random.default_rng(0)
    costs = np.exp(rng.uniform(np.log(32 ** 3), np.log(160 * 160 * 96), 64)) * rng.integers(2, 17, 64)
    for world in (1, 2, 4, 8):
        sh = shard_by_cost(costs, world)
        assert sorted(i for s in sh for i in s) == list(range(64))
        loads = [costs[s].sum() for s in sh]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= np.mean(loads) + costs.max() + 1e-6
        assert sh == shard_by_cost(list(costs), world)
    assert shard_by_cost([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard_by_cost([1.0], 0)


def _problems():
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.solvers.base import Terminal
    out = []
    for s, shape in enumerate([(10, 9, 8), (12, 10, 8), (9, 9, 9), (14, 8, 7), (8, 8, 10)]):
        w = W.layered_boxes(shape, nbox=2 + s % 3, seed=s, ext_xy=(16, 48), ext_z=(16, 30))
        terms = [Terminal(n, t) for n, t in zip(w.names, w.terminals)]
        out.append((w.grid(), w.eps_cell, terms))
    return out


def _oracle_local(problems, cfg, gcfg, streams, reports):
    from oracle import fs_oracle as O
    res = []
    for grid, eps, terms in problems:
        g = O.Grid(grid.xn, grid.yn, grid.zn)
        C, _ = O.capacitance_matrix(g, eps, [t.nodes for t in terms], method="direct")
        res.append(C)
    return res


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = capacitance_matrices(_problems(), local=_oracle_local)
        q.put((rank, [np.asarray(c) for c in out]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gather_the_whole_batch_in_order():
    import torch.multiprocessing as mp
    probs = _problems()
    want = _oracle_local(probs, None, None, 1, None)
    assert len(shard_by_cost([problem_cost(p) for p in probs], 2)[0]) > 0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, mats = q.get(timeout=120)
        got[r] = mats
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert len(got[r]) == len(want)
        for a, b in zip(got[r], want):
            assert np.array_equal(a, b)


def _failing_worker(rank, world, port, q):
    """Rank 1 fails before the gather; rank 0 must learn of it through the
    process group's timeout, not hang."""
    import datetime
    import time

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        q.put((rank, "raised"))
        raise SystemExit(3)   # leaves without joining the collective
    t0 = time.perf_counter()
    try:
        capacitance_matrices(_problems(), local=_oracle_local)
        q.put((rank, "no error"))
    except Exception as e:  # the gather times out / the peer is gone
        q.put((rank, f"error after {time.perf_counter() - t0:.1f} s: {type(e).__name__}"))


def test_a_failing_rank_is_detected_by_the_others():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert got[1] == "raised"
    assert got[0].startswith("error after"), got[0]


def test_data_parallel_schedule_covers_each_epoch_once():
    """Every step the ranks' batches are disjoint parts of one slice of that
    epoch's permutation (the same on every rank), and every rank has the same
    number of steps; one rank reproduces the plain shuffled schedule."""
    from fieldspice_b200.learned import dp_batches
    S, batch, epochs = 103, 4, 2
    for world in (1, 2, 3):
        per_rank = [list(dp_batches(S, batch, epochs, 5, r, world)) for r in range(world)]
        assert len({len(p) for p in per_rank}) == 1
        assert len(per_rank[0]) == epochs * (S // (batch * world))
        for ep in range(epochs):
            seen = []
            for p in per_rank:
                for e, _, idx in p:
                    if e == ep:
                        assert len(idx) == batch
                        seen.extend(int(i) for i in idx)
            assert len(seen) == len(set(seen)) == (S // (batch * world)) * batch * world
    rng = np.random.default_rng(5)
    perm = rng.permutation(S)
    one = list(dp_batches(S, batch, 1, 5))
    assert all(np.array_equal(idx, perm[b * batch:(b + 1) * batch]) for _, b, idx in one)


def _dp_worker(rank, world, port, q):
    """A toy data-parallel fit through the same helpers: per step, the mean
    gradient of this rank's batch, all-reduced, then one SGD step."""
    import torch
    import torch.distributed as dist
    from fieldspice_b200.learned import allreduce_mean, dp_batches, dp_world
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w = dp_world()
        data = torch.as_tensor(np.random.default_rng(1).standard_normal((64, 3)))
        theta = torch.zeros(3, dtype=torch.float64)
        for _, _, idx in dp_batches(64, 4, 2, 9, r, w):
            g = (theta - data[torch.as_tensor(idx)]).mean(0)
            allreduce_mean(g, None, w)
            theta -= 0.1 * g
        q.put((rank, theta.numpy().tolist()))
    finally:
        dist.destroy_process_group()


def test_data_parallel_fit_keeps_ranks_identical():
    """Two gloo ranks: the averaged-gradient steps leave theta identical on
    both, equal to one rank running the combined batches of each step."""
    import multiprocessing as mp

    import torch
    from fieldspice_b200.learned import dp_batches
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1]
    # the same steps on one process: the mean over both ranks' batches
    data = torch.as_tensor(np.random.default_rng(1).standard_normal((64, 3)))
    theta = torch.zeros(3, dtype=torch.float64)
    for (_, _, i0), (_, _, i1) in zip(dp_batches(64, 4, 2, 9, 0, 2), dp_batches(64, 4, 2, 9, 1, 2)):
        g0 = (theta - data[torch.as_tensor(i0)]).mean(0)
        g1 = (theta - data[torch.as_tensor(i1)]).mean(0)
        theta -= 0.1 * (g0 + g1) / 2
    assert np.allclose(res[0], theta.numpy(), rtol=0, atol=1e-15)
