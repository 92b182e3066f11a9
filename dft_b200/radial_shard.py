"""Radial batch across ranks: one process per GPU, independent atoms sharded by rank.

The reference solves each atom on its own (`solveAtom`, AtomicDFT.cpp; the Z = 1..30 sweep of
main.cpp:36-48).  Runs share nothing, so ranks split them with no data-path collective: each
rank solves its share in one `dft_solve_atoms` launch and the small per-run records (energies,
iteration counts, eigenvalues) are gathered on the host with `all_gather_object`.

Partition: longest-processing-time first.  A run's cost grows with its orbital count, so runs
are taken in order of descending Z and each goes to the rank with the least estimated work;
ties go to the lowest rank.  The result list is returned in the caller's order on every rank.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence


def run_cost(Z: int) -> float:
    """Relative cost of one radial SCF: one warp per orbital per spin, so the slowest warp
    (the deepest shell) and the number of shells both grow with Z."""
    return 1.0 + Z


def partition(Zs: Sequence[int], world: int) -> List[List[int]]:
    """Indices of the runs each rank solves (LPT order, deterministic)."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    order = sorted(range(len(Zs)), key=lambda i: (-run_cost(Zs[i]), i))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += run_cost(Zs[i])
    return [sorted(p) for p in parts]


def solve_atoms_sharded(Zs: Sequence[int], kinds: Sequence, points: int = 2000, rmax: float = 30.0,
                        engine=None, group=None, solve: Optional[Callable] = None) -> list:
    """Solve every (Z, functional) run, each rank its own share, and return all results.

    `solve(Zs, kinds)` solves a list of runs and returns one record per run; it defaults to
    `engine.solve_atoms` (one persistent launch on this rank's GPU).  Without an initialised
    process group this is a plain single-rank call."""
    import torch.distributed as dist

    if len(Zs) != len(kinds):
        raise ValueError("Zs and kinds must have the same length")
    if solve is None:
        if engine is None:
            raise ValueError("either an engine or a solve function is required")

        def solve(z, k):
            return engine.solve_atoms(z, k, points, rmax)

    distributed = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if distributed else 1
    rank = dist.get_rank(group) if distributed else 0
    mine = partition(Zs, world)[rank]
    local = solve([Zs[i] for i in mine], [kinds[i] for i in mine]) if mine else []
    if len(local) != len(mine):
        raise RuntimeError("the solver returned a different number of runs than it was given")
    if not distributed:
        return list(local)
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, list(local)), group=group)
    out = [None] * len(Zs)
    for idx, recs in gathered:
        for i, r in zip(idx, recs):
            out[i] = r
    if any(r is None for r in out):
        raise RuntimeError("a run is missing from the gathered results")
    return out
