"""Spreading independent patches over the GPUs of one node.

The reference runs one MPI child per GPU and a parent that hands each child
the next patch of a queue (forcepho/dispatcher.py:29-300).  Patches are
independent, so here every rank (one process per GPU, launched by torchrun)
computes the same assignment of jobs to ranks from their estimated costs --
longest job first, each to the rank with the least work so far -- evaluates
its own jobs on its own GPU, and the results come back to rank 0 with one
``gather_object`` at the end.  Nothing crosses GPUs while jobs run; the only
collective is that final gather of host objects (on a gloo group when the
default group is NCCL).
"""

import heapq

__all__ = ["assign", "dispatch"]


def assign(costs, n_ranks):
    """Jobs (indices into `costs`) of each rank: longest-processing-time
    first, each job to the least-loaded rank (ties to the lowest rank), so
    that every rank computes the same assignment."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    out = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return out


def dispatch(jobs, work_fn, cost_fn=None, group=None):
    """Run ``work_fn(job)`` for every job, spread over the ranks of `group`
    (the default process group if None; a single process runs everything).
    Returns, on rank 0, the list of results in job order (None elsewhere).
    `cost_fn(job)` estimates a job's cost (default 1 for every job)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    costs = [cost_fn(j) if cost_fn else 1.0 for j in jobs]
    mine = assign(costs, world)[rank]
    local = [(i, work_fn(jobs[i])) for i in mine]
    if world == 1:
        gathered = [local]
    else:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(local, gathered, dst=0, group=group)
    if rank != 0:
        return None
    results = [None] * len(jobs)
    for part in gathered:
        for i, r in part:
            results[i] = r
    return results
