"""Process-parameter sweep: many independent melt-pool instances, sharded over ranks.

The reference solves one instance per process (main.cpp:25-233), so a laser
power/speed/radius sweep is a set of independent runs.  Here the unit of work
is a whole instance:

* ranks (one per GPU) take disjoint shards of the instance list, balanced by
  cost = interior cells x time steps with the longest-processing-time rule;
* on a GPU, a shard runs through ``amcfd_run_batch``: every instance is a
  context with its own stream and a pool of host threads keeps several of them
  in flight at once;
* no collective touches the solve; the per-instance results (iterations, peak
  temperature, melt-pool length/depth/width) are gathered on the host at the
  end with one ``all_gather_object``.
"""
from __future__ import annotations

import os
import time
from typing import Callable, Dict, List, Optional, Sequence

import amcfd

RESULT_KEYS = ("niter", "itertot", "tpeak", "alen", "depth", "width", "timet")


def instance_cost(dims: Sequence[int], steps: int) -> int:
    """Interior cells x steps: the work of one instance (the reference's loops
    run over the interior, CFDSolverManager.cpp:2459-2526)."""
    ni, nj, nk = dims
    return max(ni - 2, 0) * max(nj - 2, 0) * max(nk - 2, 0) * max(int(steps), 0)


def shard(costs: Sequence[int], world: int) -> List[List[int]]:
    """Longest-processing-time partition of instance indices over `world` ranks.

    Instances are taken in decreasing cost (ties by index) and each goes to the
    rank with the smallest load so far (ties by rank).  Every index appears in
    exactly one shard; each shard lists its instances largest first, the order
    ``amcfd_run_batch`` wants.  The largest load is at most 4/3 of the optimum."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda q: (-int(costs[q]), q))
    loads = [0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for q in order:
        r = min(range(world), key=lambda x: (loads[x], x))
        parts[r].append(q)
        loads[r] += int(costs[q])
    return parts


def gpu_runner(device: int = 0, precision: int = amcfd.PREC_FP32,
               order: int = amcfd.ORDER_REDBLACK, nthreads: int = 0) -> Callable:
    """Runner that solves a shard on one GPU through amcfd_run_batch."""

    def run(paths: Sequence[str], steps: int) -> List[Dict]:
        decks = [amcfd.Deck(p) for p in paths]
        solvers = [amcfd.Solver(d, order=order, precision=precision, device=device) for d in decks]
        try:
            reps, _ = amcfd.run_batch(solvers, steps, nthreads)
        finally:
            for s in solvers:
                s.close()
        return [{k: r[k] for k in RESULT_KEYS} for r in reps]

    return run


def run_sweep(paths: Sequence[str], steps: int, runner: Optional[Callable] = None,
              rank: Optional[int] = None, world: Optional[int] = None) -> Dict:
    """Solve every deck in `paths` for `steps` steps, this rank's shard locally.

    With torch.distributed initialised, rank and world come from the default
    process group and the results of all ranks are gathered on every rank.
    Returns {"results": [per-instance dict, in `paths` order], "shards": [...],
    "local_seconds": wall time of this rank's shard, "max_seconds": the maximum
    over ranks}."""
    dist = None
    try:
        import torch.distributed as _d
        if _d.is_available() and _d.is_initialized():
            dist = _d
    except ImportError:
        pass
    if rank is None:
        rank = dist.get_rank() if dist else int(os.environ.get("RANK", "0"))
    if world is None:
        world = dist.get_world_size() if dist else int(os.environ.get("WORLD_SIZE", "1"))
    costs = [instance_cost(amcfd.Deck(p).dims, steps) for p in paths]
    parts = shard(costs, world)
    mine = parts[rank]
    if runner is None:
        runner = gpu_runner(device=int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    local = runner([paths[q] for q in mine], steps) if mine else []
    secs = time.perf_counter() - t0
    if len(local) != len(mine):
        raise RuntimeError(f"runner returned {len(local)} results for {len(mine)} instances")
    payload = (rank, list(zip(mine, local)), secs)
    if dist is not None and world > 1:
        gathered: List = [None] * world
        dist.all_gather_object(gathered, payload)
    else:
        gathered = [payload]
    results: List[Optional[Dict]] = [None] * len(paths)
    for _, pairs, _ in gathered:
        for q, res in pairs:
            results[q] = dict(res, instance=q, cost=costs[q])
    missing = [q for q, r in enumerate(results) if r is None]
    if missing:
        raise RuntimeError(f"instances without a result: {missing}")
    return {"results": results, "shards": parts, "local_seconds": secs,
            "max_seconds": max(g[2] for g in gathered)}
