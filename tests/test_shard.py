"""Cost-balanced reactor sharding over ranks (zerork_b200/shard.py), the host
logic of the multi-GPU plugin solve, on CPU with the gloo backend.

The stub solver stands in for the per-GPU plugin solve: it transforms each
reactor deterministically from its own state, records which rank solved it
and fails the reactors whose state says so, so the test can check that the
balanced exchange returns every reactor's own result to its owner and that
the work was split by cost (zerork_reactor_manager.cpp:659-832 LoadBalance).
"""
import os
import socket

import numpy as np
import pytest

from zerork_b200.shard import balanced_solve, partition_by_cost


def test_partition_balances_cumulative_cost():
    rng = np.random.default_rng(0)
    cost = rng.exponential(100.0, size=1000)
    b = partition_by_cost(cost, 4)
    assert b[0] == 0 and b[-1] == 1000 and np.all(np.diff(b) >= 0)
    sums = [cost[b[i]:b[i + 1]].sum() for i in range(4)]
    assert max(sums) - min(sums) <= 2 * cost.max()
    # failed reactors carry negative cost: the magnitude counts
    assert np.array_equal(partition_by_cost(-cost, 4), b)


def test_partition_edge_cases():
    assert list(partition_by_cost([], 3)) == [0, 0, 0, 0]
    assert list(partition_by_cost(np.zeros(6), 3)) == [0, 2, 4, 6]  # first call: equal counts
    b = partition_by_cost([1.0, 1.0], 4)  # more ranks than reactors
    assert b[0] == 0 and b[-1] == 2 and np.all(np.diff(b) >= 0)
    b = partition_by_cost([1000.0, 1, 1, 1], 2)  # one dominant reactor
    assert list(b) == [0, 1, 4]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _local(rank):
    rng = np.random.default_rng(10 + rank)
    n = 5 if rank == 0 else 13
    T = rng.uniform(800, 1600, n)
    P = rng.uniform(1e5, 5e6, n)
    Y = rng.dirichlet(np.ones(4), n)
    cost = rng.exponential(50.0, n) * (20.0 if rank == 0 else 1.0)  # rank 0 owns the costly ones
    return T, P, Y, cost


def _stub_solve(rank_box):
    def solve(dt, T, P, Y, cost):
        T[:] = T * (1.0 + dt) + 1.0
        P[:] = P * 2.0
        Y[:] = Y[:, ::-1]
        fail = T > 1600.0 * (1.0 + dt)
        cost[:] = np.where(fail, -(rank_box[0] + 1.0), rank_box[0] + 1.0)
        return int(fail.sum())
    return solve


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        T, P, Y, cost = _local(rank)
        box = [rank]
        nfail = balanced_solve(dist, _stub_solve(box), 0.5, T, P, Y, cost)
        np.savez(os.path.join(out, f"r{rank}.npz"), T=T, P=P, Y=Y, cost=cost, nfail=nfail)
    finally:
        dist.destroy_process_group()


def test_balanced_solve_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    solved_by = []
    total_fail = 0
    for rank in range(2):
        T0, P0, Y0, c0 = _local(rank)
        r = np.load(tmp_path / f"r{rank}.npz")
        # every reactor comes back to its owner, transformed from its own state
        assert np.allclose(r["T"], T0 * 1.5 + 1.0)
        assert np.allclose(r["P"], P0 * 2.0)
        assert np.allclose(r["Y"], Y0[:, ::-1])
        solved_by.append(np.abs(r["cost"]) - 1.0)
        total_fail += int(np.sum(r["cost"] < 0))
        nfail = int(r["nfail"])
    assert nfail == total_fail  # the failure count is global and the same on every rank
    # the work was split by cost: rank 1 solved some of rank 0's costly reactors
    # or rank 0 solved fewer than it owns
    allc = np.concatenate([_local(0)[3], _local(1)[3]])
    b = partition_by_cost(allc, 2)
    who = np.concatenate(solved_by)
    assert np.array_equal(who[: b[1]], np.zeros(b[1])) and np.all(who[b[1]:] == 1.0)
    assert b[1] != 5  # not the ownership split


def test_exchange_plan_moves_only_reassigned_reactors():
    """The forward exchange sends each rank only the reactors the partition
    gives it from other ranks; the block a rank keeps stays local."""
    from zerork_b200.shard import exchange_plan
    counts = [5, 13, 7]
    rng = np.random.default_rng(3)
    cost = rng.exponential(10.0, sum(counts))
    cost[:5] *= 30.0
    send, recv, b = exchange_plan(counts, cost, 3)
    offs = np.concatenate([[0], np.cumsum(counts)])
    for r in range(3):
        assert sum(send[r]) == counts[r] and sum(recv[r]) == b[r + 1] - b[r]
        keep = max(0, min(offs[r + 1], b[r + 1]) - max(offs[r], b[r]))
        assert send[r][r] == keep
    moved = sum(send[r][d] for r in range(3) for d in range(3) if d != r)
    assert moved < sum(counts)  # not everything travels


def _plugin_worker(rank, world, port, out, mech, therm):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch
    import torch.distributed as dist
    from zerork_b200.plugin import Plugin
    from zerork_b200.shard import plugin_solver
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        from zerork_b200 import mechgen
        g = mechgen.generate(mechgen.SPECS["c1_h2"])
        T, P, Y = mechgen.reactor_states(g, 24, "c1", seed=40 + rank)
        n = 8 if rank == 0 else 16
        T, P, Y = T[:n].copy(), P[:n].copy(), np.ascontiguousarray(Y[:n])
        cost = np.full(n, 100.0 if rank == 0 else 1.0)
        p = Plugin(mech, therm)
        nfail = balanced_solve(dist, plugin_solver(p), 1e-4, T, P, Y, cost)
        np.savez(os.path.join(out, f"p{rank}.npz"), T=T, P=P, Y=Y, cost=cost, nfail=nfail)
        p.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_balanced_plugin_solve_two_ranks_one_gpu(tmp_path):
    """The real plugin solve through the balanced exchange: two gloo ranks
    sharing cuda:0 (independent solves, no cross-rank waits inside a
    kernel); each rank's reactors come back solved, identical to solving
    them on one rank without sharding."""
    from conftest import have_gpu
    if not have_gpu():
        pytest.skip("no CUDA device")
    import torch.multiprocessing as mp
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    g = mechgen.generate(mechgen.SPECS["c1_h2"])
    mech, therm = g.write(str(tmp_path))
    mp.spawn(_plugin_worker, args=(2, _free_port(), str(tmp_path), mech, therm), nprocs=2, join=True)
    p = Plugin(mech, therm)
    for rank in range(2):
        T, P, Y = mechgen.reactor_states(g, 24, "c1", seed=40 + rank)
        n = 8 if rank == 0 else 16
        T, P, Y = T[:n].copy(), P[:n].copy(), np.ascontiguousarray(Y[:n])
        assert p.solve(1e-4, T, P, Y) == 0
        r = np.load(tmp_path / f"p{rank}.npz")
        assert int(r["nfail"]) == 0 and np.all(r["cost"] > 0)
        np.testing.assert_allclose(r["T"], T, rtol=0, atol=1e-9 * T.max())
        np.testing.assert_allclose(r["Y"], Y, rtol=0, atol=1e-12)
