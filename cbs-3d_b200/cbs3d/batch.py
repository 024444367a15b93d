"""Batched cases across GPUs: independent instances bin-packed by tet count
onto ranks (longest processing time first), one cbs3d_batch per rank, and a
host gather of per-instance metrics -- the only collective.  One process per
GPU under torchrun; any torch.distributed backend serves the gather."""
from __future__ import annotations

import heapq


def lpt_shard(weights, nranks: int) -> list[list[int]]:
    """Longest-processing-time assignment: instances in decreasing weight
    (ties by index) each go to the least-loaded rank (ties to the lowest
    rank).  Deterministic, so every rank computes the same shards; the
    heaviest rank is within 4/3 of the optimum.  Returns the instance indices
    of each rank, in ascending order."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0, r) for r in range(nranks)]
    shards = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return [sorted(s) for s in shards]


def shard_loads(weights, shards) -> list:
    return [sum(weights[i] for i in s) for s in shards]


def run_sharded(cases, steps: int, rank: int, world: int, runner, dist=None) -> list | None:
    """Runs this rank's shard with runner(list_of_cases, steps) -> list of
    per-instance metric dicts (same order), tags each with its global
    instance index, and gathers every rank's list to rank 0, which gets all
    of them sorted by instance; other ranks get None."""
    shards = lpt_shard([c.mesh.nelem for c in cases], world)
    mine = shards[rank]
    local = runner([cases[i] for i in mine], steps) if mine else []
    for i, m in zip(mine, local):
        m["instance"] = i
    if dist is None or world == 1:
        gathered = [local]
    else:
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
    if rank != 0:
        return None
    return sorted((m for part in gathered for m in part), key=lambda m: m["instance"])


def gpu_runner(precision: int = 0, device: int = 0, autotune: bool = True):
    """runner for run_sharded: one cbs3d_batch on this rank's GPU; per
    instance its steps, PCG iterations of the last step and the batch's
    device time."""
    def run(cases, steps):
        from . import gpu
        b = gpu.Batch(cases, precision=precision, device=device, autotune=autotune)
        b.step(1)
        st, sec = b.step(steps)
        out = [{"nelem": c.mesh.nelem, "steps": s.steps_done, "cg_iterations": s.cg.iterations,
                "gpu_seconds": sec} for c, s in zip(cases, st)]
        b.close()
        return out
    return run
