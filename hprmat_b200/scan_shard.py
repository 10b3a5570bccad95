"""Energy scans over several GPUs: one process per GPU, the scan's units sharded by cost.

Every (block, energy) solve of a scan is independent, so the scan shards without any
collective on the data path: each block's energies are cut into runs of consecutive energies
(a run is a sub-block with the block's potential), the runs are assigned to ranks by greedy
longest-processing-time on their cost, nenergies x (nch nr)^3 (the LU work), each rank solves
its runs with ``Context.rmatrix_scan`` on its own GPU, and one gather at the end gives every
rank all collision matrices (a few KB per solve).  The reference has no counterpart (its
drivers loop energies in one process, examples/Ex1/example1_hp.f90:102-110).
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np

__all__ = ["block_costs", "unit_cost", "lpt_shards", "scan_units", "shard_units", "run_sharded_scan"]


def unit_cost(nch: int, nr: int, nenergies: int, method: str = "lu") -> float:
    """Cost of solving nenergies energies of one block of nch channels: nenergies N^3 for the LU
    method (one factorisation each, N = nch nr); N^3 + nenergies N^2 nch for the shifted method
    (one Hessenberg reduction for the unit, then O(N^2 nch) per energy)."""
    n = float(nch * nr)
    if method == "shifted":
        return n ** 3 + nenergies * n * n * nch
    if method == "lu":
        return nenergies * n ** 3
    raise ValueError(f"unknown scan method {method!r}")


def block_costs(blocks: Sequence, nr: int) -> list[float]:
    """Cost of each block (lval, cpot, qk, eta): nenergies x N^3 with N = nch nr."""
    return [float(np.asarray(qk).shape[0]) * float(len(lval) * nr) ** 3 for lval, _c, qk, _e in blocks]


def lpt_shards(costs: Sequence[float], world: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment of items to ``world`` ranks: items in order
    of decreasing cost (ties by index) go to the least-loaded rank (ties by rank).  Every item
    is in exactly one shard; each shard lists its items in increasing index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shards]


def scan_units(blocks: Sequence, chunk: int | None) -> list[tuple[int, np.ndarray]]:
    """The scan's units: (block index, energy indices), runs of up to ``chunk`` energies of a
    block in the given energy order (``chunk`` None: whole blocks)."""
    units = []
    for b, (_lval, _cpot, qk, _eta) in enumerate(blocks):
        ne = int(np.asarray(qk).shape[0])
        step = ne if not chunk else int(chunk)
        for e0 in range(0, ne, max(step, 1)):
            units.append((b, np.arange(e0, min(ne, e0 + step))))
    return units


def shard_units(blocks: Sequence, nr: int, rank: int, world: int, chunk: int | None = 32, method: str = "lu"):
    """This rank's units and the sub-blocks (lval, cpot, qk[idx], eta[idx]) that solve them, with
    the units' costs by ``method`` (unit_cost).  The shifted method reduces every unit's block
    once, so it is sharded in whole blocks (``chunk`` ignored): a block split over ranks would
    repeat its reduction on each."""
    if method == "shifted":
        chunk = None
    units = scan_units(blocks, chunk)
    costs = [unit_cost(len(blocks[b][0]), nr, len(idx), method) for b, idx in units]
    mine = [units[i] for i in lpt_shards(costs, world)[rank]]
    subs = [(blocks[b][0], blocks[b][1], np.asarray(blocks[b][2])[idx], np.asarray(blocks[b][3])[idx])
            for b, idx in mine]
    return mine, subs


def run_sharded_scan(blocks: Sequence, nr: int, solve: Callable[[list], list], rank: int = 0, world: int = 1,
                     gather: bool = True, chunk: int | None = 32):
    """Solve this rank's units with ``solve`` (a list of blocks -> a list of per-block results,
    each a tuple of arrays with the energy as leading axis, e.g. ``ctx.rmatrix_scan(b, rmax,
    nr)``) and, with ``gather`` and world > 1, all-gather over the default process group.
    Returns (results, my_units): results[b] is the tuple for block b with every energy filled
    in (only this rank's energies without the gather; other entries stay zero)."""
    mine, subs = shard_units(blocks, nr, rank, world, chunk)
    local = solve(subs) if subs else []
    if len(local) != len(mine):
        raise RuntimeError("solve returned %d results for %d units" % (len(local), len(mine)))
    parts = [(mine, local)]
    if gather and world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, (mine, local))
    results: list = [None] * len(blocks)
    for units, res in parts:
        for (b, idx), r in zip(units, res):
            ne = int(np.asarray(blocks[b][2]).shape[0])
            if results[b] is None:
                results[b] = tuple(np.zeros((ne,) + np.asarray(a).shape[1:], dtype=np.asarray(a).dtype) for a in r)
            for dst, a in zip(results[b], r):
                dst[idx] = a
    return results, mine
