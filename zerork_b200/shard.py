"""Cost-balanced reactor sharding across GPUs, one process per GPU.

The reference balances reactors over MPI ranks before its per-rank solve
(zerork_reactor_manager.cpp:659-832, LoadBalance): every rank owns the
reactors of its part of the CFD mesh, the previous call's per-reactor cost
(ZERORK_FIELD_COST) decides how many each rank solves, reactors travel to
the rank that solves them and the results travel back.  Here the same host
logic runs over torch.distributed (NCCL between GPUs, gloo on CPU for
tests): ranks all-gather their states and costs, every rank computes the
same contiguous partition of the global reactor list by cumulative cost,
solves its slice on its own GPU with no collective inside the solve, and the
solved slices are all-gathered back so each rank keeps its own reactors.
"""
import numpy as np


def partition_by_cost(cost, world):
    """Contiguous split of len(cost) reactors into `world` ranges of nearly
    equal total |cost| (zero costs count as 1, as for a first call).
    Returns world + 1 boundaries; deterministic."""
    w = np.abs(np.asarray(cost, dtype=np.float64))
    w = np.where(w > 0, w, 1.0)
    n = w.size
    if n == 0:
        return np.zeros(world + 1, dtype=np.int64)
    c = np.concatenate([[0.0], np.cumsum(w)])
    targets = c[-1] * np.arange(1, world) / world
    cuts = np.searchsorted(c, targets, side="left")
    bounds = np.concatenate([[0], cuts, [n]]).astype(np.int64)
    return np.maximum.accumulate(np.minimum(bounds, n))


def _all_gather_rows(dist, x, group=None):
    """All-gather a float64 [rows, cols] host array of per-rank row counts."""
    import torch
    world = dist.get_world_size(group)
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64))
    cnt = torch.tensor([t.shape[0]], dtype=torch.int64)
    cnts = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(cnts, cnt, group=group)
    cnts = [int(c.item()) for c in cnts]
    mx = max(cnts)
    pad = torch.zeros((mx,) + tuple(t.shape[1:]), dtype=torch.float64)
    pad[: t.shape[0]] = t
    out = [torch.zeros_like(pad) for _ in range(world)]
    dist.all_gather(out, pad, group=group)
    return [o[:c].numpy() for o, c in zip(out, cnts)], cnts


def balanced_solve(dist, solve, dt, T, P, Y, cost, group=None):
    """Solve this rank's reactors (T[n], P[n], Y[n, nsp], cost[n], updated in
    place) with the work spread over all ranks by cost.

    solve(dt, T, P, Y, cost) integrates the reactors it is given in place and
    returns the number that failed; every rank calls balanced_solve with the
    same dt.  Returns the global number of failed reactors."""
    import torch
    rank = dist.get_rank(group)
    nsp = Y.shape[1]
    packed = np.concatenate([T[:, None], P[:, None], cost[:, None], Y], axis=1)
    parts, cnts = _all_gather_rows(dist, packed, group)
    allp = np.concatenate(parts, axis=0)
    bounds = partition_by_cost(allp[:, 2], len(cnts))
    lo, hi = int(bounds[rank]), int(bounds[rank + 1])
    mine = allp[lo:hi].copy()
    Tm, Pm, cm = mine[:, 0].copy(), mine[:, 1].copy(), mine[:, 2].copy()
    Ym = np.ascontiguousarray(mine[:, 3:])
    nfail = solve(dt, Tm, Pm, Ym, cm) if hi > lo else 0
    mine[:, 0], mine[:, 1], mine[:, 2], mine[:, 3:] = Tm, Pm, cm, Ym
    solved, _ = _all_gather_rows(dist, mine, group)
    allp = np.concatenate(solved, axis=0)
    off = int(np.sum(cnts[:rank]))
    own = allp[off:off + cnts[rank]]
    T[:], P[:], cost[:] = own[:, 0], own[:, 1], own[:, 2]
    Y[:] = own[:, 3:3 + nsp]
    f = torch.tensor([nfail], dtype=torch.int64)
    dist.all_reduce(f, group=group)
    return int(f.item())


def plugin_solver(plugin):
    """solve() callable for balanced_solve backed by a Plugin handle on this
    rank's GPU: the COST field is written back per reactor."""
    def solve(dt, T, P, Y, cost):
        c = plugin.set_aux_field("COST", cost)
        rc = plugin.solve(dt, T, P, Y, raise_on_fail=False)
        cost[:] = c
        return int(np.sum(c < 0)) if rc != 0 else 0
    return solve
