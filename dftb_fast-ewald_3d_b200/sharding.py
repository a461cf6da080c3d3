"""Sharding of the batched form (many independent cells) over ranks.

Independent cells are the only unit of this path that shards: a single cell is
evaluated whole on one GPU ("replicas only").  Cells are assigned to ranks by a
longest-processing-time greedy pass over a cost estimate, each rank evaluates
its cells on its own GPU with no collective in the data path, and the per-cell
results are gathered once at the end (torch.distributed.all_gather_object over
NCCL or gloo).  The reference evaluates cells one by one on one process; its
distributed grids are listed as future work (fft3d_readme.md:33).
"""

from __future__ import annotations

import math

import numpy as np


def cell_cost(n_atoms: int, n_modes, window_cutoff: int) -> float:
    """Work estimate of one shift+force evaluation: stencil points (spread and
    four gathers) plus FFT volume, in arbitrary but consistent units."""
    grid = 1.0
    for m in n_modes:
        grid *= 2 * m
    stencil = (2 * window_cutoff + 1) ** 3
    return 5.0 * n_atoms * stencil + 5.0 * grid * math.log2(max(grid, 2.0))


def partition(costs, world_size: int):
    """Greedy LPT: heaviest cell first onto the least loaded rank (ties to the
    lower rank, equal costs in index order).  Returns, per rank, its cell
    indices in ascending order."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world_size
    shards = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shards]


def cell_costs(cells, tol, parameters):
    """Costs from the reference parameter chain; `parameters(pos, q, lat, tol)`
    returns a dict with n_modes and window_cutoff."""
    out = []
    for pos, q, lat in cells:
        p = parameters(pos, q, lat, tol)
        out.append(cell_cost(len(q), p["n_modes"], p["window_cutoff"]))
    return out


def shard_of(cells, tol, parameters, rank: int, world_size: int):
    """This rank's cell indices (ascending) under the LPT partition.  Every
    rank computes the same partition from the same cells, so no message is
    needed to agree on it."""
    return partition(cell_costs(cells, tol, parameters), world_size)[rank]


def gather_results(mine, pots, forces, n_cells: int, world_size: int, group=None):
    """Every cell's (potential, force) on every rank, in cell order, from each
    rank's results for its own cells `mine`.  The one collective of the path."""
    local = {i: (np.asarray(p), np.asarray(f)) for i, p, f in zip(mine, pots, forces)}
    if world_size == 1:
        gathered = [local]
    else:
        import torch.distributed as dist

        gathered = [None] * world_size
        dist.all_gather_object(gathered, local, group=group)
    merged = {}
    for part in gathered:
        merged.update(part)
    return [merged[i][0] for i in range(n_cells)], [merged[i][1] for i in range(n_cells)]


def run_sharded(cells, tol, evaluate, parameters, rank: int, world_size: int, group=None):
    """Evaluate `cells` across `world_size` ranks and return every cell's
    (potential, force) on every rank, in cell order.

    evaluate(list_of_cells, tol) -> (list of potentials, list of forces) runs on
    this rank's device; parameters(...) is the host-side parameter chain."""
    mine = shard_of(cells, tol, parameters, rank, world_size)
    pots, forces = evaluate([cells[i] for i in mine], tol) if mine else ([], [])
    return gather_results(mine, pots, forces, len(cells), world_size, group)


def library_parameters(pos, q, lat, tol):
    """The CUDA library's host-side parameter chain (ewald_parameters), the
    cost model's input."""
    import ewald_b200

    return ewald_b200.ewald_parameters(pos, q, len(q), lat, tol)


def library_evaluator(ctx, **overrides):
    """evaluate() for run_sharded on the CUDA library: this rank's cells in one
    batched call (ewg_batch_potential_force) on `ctx`, an ewald_b200.Context
    of this rank's GPU."""

    def evaluate(cells, tol):
        return ctx.batch_potential_force(cells, tol, **overrides)

    return evaluate
