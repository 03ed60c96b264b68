"""Many systems over several GPUs, one process per GPU: a host-side assignment of systems to ranks
and a gather of the results to rank 0.

One system does not shard (every sub-step needs a barrier between its check and its perform, and
a colour group spans the whole box), so several GPUs share a set of independent systems: each
rank advances its own subset on its own GPU with no collective on the hot path, and the results
(positions, move counters) travel to rank 0 once, after the runs, through the initialised
torch.distributed process group (NCCL or gloo; ``gather_object`` needs no device tensors).
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence


def shard_systems(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time assignment: systems in decreasing cost (monomers x MCS, the work of
    a run), each to the rank with the least assigned cost so far (ties: the lower rank; equal
    costs: the lower index first). Returns, per rank, its system indices in increasing order.
    Deterministic, so every rank computes the same assignment without communicating."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(ix) for ix in out]


def run_sharded(systems: Sequence, mcs: Sequence[int], run_local: Callable[[list, list], list],
                rank: int = 0, world: int = 1):
    """Runs this rank's shard with ``run_local(systems, mcs) -> results`` (one result per system,
    any picklable object) and gathers every rank's results to rank 0 in the original system order.
    Rank 0 returns the full list; the other ranks return None. With world == 1 no process group is
    needed."""
    if len(systems) != len(mcs):
        raise ValueError("one MCS count per system")
    shards = shard_systems([s.n * int(m) for s, m in zip(systems, mcs)], world)
    mine = shards[rank]
    local = run_local([systems[i] for i in mine], [int(mcs[i]) for i in mine]) if mine else []
    if len(local) != len(mine):
        raise RuntimeError("run_local returned the wrong number of results")
    if world == 1:
        return list(local)
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, local)), parts, dst=0)
    if rank != 0:
        return None
    out = [None] * len(systems)
    for part in parts:
        for i, res in part:
            out[i] = res
    return out


def batch_runner(gpu: int):
    """A ``run_local`` for run_sharded: the shard's systems advance together as one Batch on GPU
    ``gpu`` (each its own MCS count); returns per system its positions and move counters."""
    def run(systems, mcs):
        from .updater import Batch, UpdaterGPUScBFM_AB_Type
        members, b = [], None
        try:
            for s in systems:
                u = UpdaterGPUScBFM_AB_Type(gpu)
                members.append(u)           # closed below even if load_system raises
                u.load_system(s)
            b = Batch(members, gpu=gpu)
            b.run_each(list(mcs))
            return [(m.get_coords(), m.stats()) for m in members]
        finally:
            if b is not None:
                b.close()
            for m in members:
                m.close()
    return run
