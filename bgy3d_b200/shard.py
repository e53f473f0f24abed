"""Many independent solutes over the ranks of a process group (one process per
GPU): the solute-parallel form of the batch loops of guile/bgy3d.scm:819-880
and 943-975.  Solves never communicate; each rank solves its share with
rism3d_solve_batch on its own device and the results are gathered on the host
(the only collective), so any torch.distributed backend serves (NCCL between
GPUs, gloo for the host-side tests).
"""
import heapq


def solve_cost(settings):
    """Relative cost of one solve: N log N of its grid (the FFT passes; the
    Newton and Krylov iteration counts vary little between solutes)."""
    import math
    n = settings["N"]
    N = tuple(n) if isinstance(n, (tuple, list)) else (int(n),) * 3
    tot = N[0] * N[1] * N[2]
    return tot * math.log2(tot)


def shard(costs, world):
    """Longest-processing-time partition of job indices over `world` ranks:
    jobs by decreasing cost, each to the least loaded rank (ties to the
    lower rank).  Returns one ascending index list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def hnc3d_run_batch_sharded(solutes, solvent, settings, chi, group=None, workers=0, solve=None):
    """hnc3d_run_batch over the ranks of `group` (the default process group):
    every rank calls this with the same arguments, solves its shard and
    returns the full list of result dicts in job order.  settings / chi as
    hnc3d_run_batch (one for all, or one per solute).  `solve` replaces
    hnc3d_run_batch(solutes, solvent, settings, chi, workers=...) for the
    local shard (tests)."""
    import torch.distributed as dist
    from .solver import hnc3d_run_batch

    n = len(solutes)
    sets = settings if isinstance(settings, (list, tuple)) else [settings] * n
    chis = chi if isinstance(chi, (list, tuple)) else [chi] * n
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    mine = shard([solve_cost(s) for s in sets], world)[rank]
    run = solve or (lambda so, sv, st, ch: hnc3d_run_batch(so, sv, st, ch, workers=workers))
    local = run([solutes[i] for i in mine], solvent, [sets[i] for i in mine], [chis[i] for i in mine]) if mine else []
    if world == 1:
        return list(local)
    gathered = [None] * world
    dist.all_gather_object(gathered, list(zip(mine, local)), group=group)
    out = [None] * n
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
