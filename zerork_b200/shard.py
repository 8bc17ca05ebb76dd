"""Cost-balanced reactor sharding across GPUs, one process per GPU.

The reference balances reactors over MPI ranks before its per-rank solve
(zerork_reactor_manager.cpp:659-832, LoadBalance): every rank owns the
reactors of its part of the CFD mesh, the previous call's per-reactor cost
(ZERORK_FIELD_COST) decides how many each rank solves, reactors travel to
the rank that solves them and the results travel back.  Here the same host
logic runs over torch.distributed: ranks all-gather only their per-reactor
costs, every rank computes the same contiguous partition of the global
reactor list by cumulative cost, the reactors that change rank move in one
all-to-all exchange (a rank's own reactors form one contiguous run of the
global list, so each destination receives one contiguous block and the block
a rank keeps never leaves it), each rank solves its share on its own GPU with
no collective inside the solve, and a second all-to-all returns the results
to their owners.  The exchanges use CUDA tensors on the current device when
the process group's backend is NCCL and CPU tensors otherwise (gloo).
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


def _device(dist, group):
    import torch
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _split(lo_own, hi_own, bounds):
    """Rows [lo_own, hi_own) of the global list, cut at the partition
    bounds: how many of them go to each rank."""
    world = len(bounds) - 1
    return [int(max(0, min(hi_own, bounds[r + 1]) - max(lo_own, bounds[r]))) for r in range(world)]


def exchange_plan(counts, cost_all, world):
    """For every rank: (send sizes, receive sizes) of the forward exchange,
    and the partition bounds, from the per-rank reactor counts and the
    all-gathered costs (rank-major)."""
    bounds = partition_by_cost(cost_all, world)
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    send = [_split(offs[r], offs[r + 1], bounds) for r in range(world)]
    recv = [[send[src][r] for src in range(world)] for r in range(world)]
    return send, recv, bounds


def balanced_solve(dist, solve, dt, T, P, Y, cost, group=None):
    """Solve this rank's reactors (T[n], P[n], Y[n, nsp], cost[n], updated in
    place) with the work spread over all ranks by cost.

    solve(dt, T, P, Y, cost) integrates the reactors it is given in place and
    returns the number that failed; every rank calls balanced_solve with the
    same dt.  Returns the global number of failed reactors."""
    import torch
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    dev = _device(dist, group)
    n, nsp = T.shape[0], Y.shape[1]
    # per-rank counts and the global cost list (8 bytes per reactor)
    cnt = torch.tensor([n], dtype=torch.int64, device=dev)
    cnts = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(cnts, cnt, group=group)
    counts = [int(c.item()) for c in cnts]
    mx = max(counts)
    cpad = torch.zeros(mx, dtype=torch.float64, device=dev)
    cpad[:n] = torch.from_numpy(np.ascontiguousarray(cost, dtype=np.float64)).to(dev)
    call = [torch.zeros(mx, dtype=torch.float64, device=dev) for _ in range(world)]
    dist.all_gather(call, cpad, group=group)
    cost_all = np.concatenate([c[:k].cpu().numpy() for c, k in zip(call, counts)])
    send, recv, bounds = exchange_plan(counts, cost_all, world)
    # forward: my reactors to the ranks that solve them
    packed = np.concatenate([T[:, None], P[:, None], cost[:, None], Y], axis=1)
    cols = packed.shape[1]
    src = torch.from_numpy(np.ascontiguousarray(packed)).to(dev)
    m = int(bounds[rank + 1] - bounds[rank])
    dst = torch.zeros((m, cols), dtype=torch.float64, device=dev)
    dist.all_to_all_single(dst, src, output_split_sizes=recv[rank], input_split_sizes=send[rank],
                           group=group)
    mine = dst.cpu().numpy()
    Tm, Pm, cm = mine[:, 0].copy(), mine[:, 1].copy(), mine[:, 2].copy()
    Ym = np.ascontiguousarray(mine[:, 3:])
    nfail = solve(dt, Tm, Pm, Ym, cm) if m > 0 else 0
    mine = np.concatenate([Tm[:, None], Pm[:, None], cm[:, None], Ym], axis=1)
    # back: the results to their owners (the reverse split)
    back = torch.zeros((n, cols), dtype=torch.float64, device=dev)
    dist.all_to_all_single(back, torch.from_numpy(np.ascontiguousarray(mine)).to(dev),
                           output_split_sizes=send[rank], input_split_sizes=recv[rank], group=group)
    own = back.cpu().numpy()
    T[:], P[:], cost[:] = own[:, 0], own[:, 1], own[:, 2]
    Y[:] = own[:, 3:3 + nsp]
    f = torch.tensor([nfail], dtype=torch.int64, device=dev)
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
