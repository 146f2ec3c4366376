"""Many independent bodies over several GPUs: one process per GPU, bodies
partitioned by predicted cost, each rank solving its share as one forest
batch (BatchMobility) with no communication until a final gather of the
per-body results.

The cost of a body is dominated by the pair sums over its quadrature points
(P2P, P2L and S2M all scale with them), so the partition balances quadrature
counts with the longest-processing-time rule: bodies in decreasing cost,
each to the rank with the least load so far (ties to the lower rank), which
keeps every rank within one body's cost of the mean.  The only collective is
`all_gather_object` of (body ids, 6 x 6 matrices, GMRES info) at the end.
"""
import numpy as np

__all__ = ["body_costs", "partition", "solve_modes_sharded"]


def body_costs(bodies):
    """Predicted cost per body: its number of quadrature points."""
    return [int(len(fine)) for _, fine in bodies]


def partition(costs, world):
    """Longest-processing-time assignment: a list of `world` lists of body
    indices (ascending within each list)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def _solve_batch(bodies, kernelPar, tol, maxIter, **kw):
    from .batch import BatchMobility
    B = BatchMobility(bodies, kernelPar, **kw)
    return B.solve_modes(tol=tol, maxIter=maxIter)


def solve_modes_sharded(bodies, kernelPar, tol=1e-6, maxIter=200, group=None, solver=None, **batch_kw):
    """Per body its 6 x 6 mobility matrix (as BatchMobility.solve_modes), the
    bodies shared among the ranks of `group` (torch.distributed, initialised
    by the caller; each rank on its own GPU).  Returns (matrices, infos) in
    body order on every rank.  `solver(bodies, kernelPar, tol, maxIter,
    **batch_kw)` replaces the forest batch (for tests without a GPU)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    parts = partition(body_costs(bodies), world)
    mine = parts[rank]
    solve = solver or _solve_batch
    if mine:
        mats, infos = solve([bodies[i] for i in mine], kernelPar, tol, maxIter, **batch_kw)
        mats = [np.asarray(m) for m in mats]
    else:
        mats, infos = [], []
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, mats, infos), group=group)
    out_m, out_i = [None] * len(bodies), [None] * len(bodies)
    for ids, ms, inf in gathered:
        for k, b in enumerate(ids):
            out_m[b], out_i[b] = ms[k], inf[k]
    return out_m, out_i
