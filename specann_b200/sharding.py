"""Multi-GPU form of the batched workload: independent (instance, seed) problems sharded over ranks.

One process per GPU (torch.distributed). A single instance's sweep is a sequential warm-start chain
whose SpMV would need an all-gather of x every Lanczos step, so a single solve runs as replicas
only. Batches shard naturally: every rank takes a subset of the instances (greedy balance of the
estimated cost, all seeds of an instance on the same rank so the instance is uploaded once), runs
its shard as one batched launch on its own GPU, and the only exchange is the final gather of the
per-problem results (best energy, spins, counters) with all_gather_object. There is no
collective on the data path.
"""
from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np


def instance_cost(n: int, nnz: int) -> float:
    """Bytes moved by one Lanczos step of an instance (the SpMV stream plus the basis passes):
    the cost model of the batch planner."""
    return 8.0 * float(nnz) + 100.0 * float(n)


def shard_instances(sizes: Sequence[tuple], world: int) -> List[List[int]]:
    """Instances (n, nnz) -> `world` lists of instance indices: longest first onto the least-loaded
    rank (LPT). Every rank gets a list (possibly empty); each list is in increasing index order."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    costs = np.array([instance_cost(n, z) for n, z in sizes], dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world)
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        out[r].append(int(i))
        load[r] += costs[i]
    return [sorted(x) for x in out]


def merge_results(per_rank: Sequence[Dict[int, dict]]) -> List[dict]:
    """Results gathered from every rank ({instance index: [results per seed]}) in instance order."""
    merged: Dict[int, list] = {}
    for part in per_rank:
        for k, v in part.items():
            if k in merged:
                raise ValueError(f"instance {k} was solved on two ranks")
            merged[k] = v
    return [r for k in sorted(merged) for r in merged[k]]


def run_sharded(instances: Sequence, seeds: Sequence[int], rank: int, world: int, group=None, **solver_kwargs):
    """Solve this rank's shard of (instances x seeds) in one batched launch and gather every rank's
    results; returns the results of all problems (instance-major, seed-minor) on every rank."""
    import torch.distributed as dist
    from .batch import BatchedSpectralAnnealing
    sizes = [(J.shape[0], J.nnz) for J in instances]
    mine = shard_instances(sizes, world)[rank]
    local: Dict[int, list] = {}
    if mine:
        b = BatchedSpectralAnnealing(seeds=seeds, **solver_kwargs)
        b.load([instances[i] for i in mine])
        b.sweep()
        res = b.results()
        S = len(seeds)
        for j, i in enumerate(mine):
            rows = res[j * S:(j + 1) * S]
            for r in rows:
                r["instance"] = i
            local[i] = [{"instance": i, "seed": r["seed"], "energy": r["energy"], "spins": r["spins"],
                         "num_candidates": r["num_candidates"], "device_ms": r["device_ms"]} for r in rows]
        b.close()
    gathered = [None] * world
    if world > 1:
        dist.all_gather_object(gathered, local, group=group)
    else:
        gathered = [local]
    return merge_results(gathered)
