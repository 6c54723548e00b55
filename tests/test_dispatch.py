"""CPU: the patch dispatcher's assignment and its gather over two gloo ranks."""
import os

import pytest
import torch.multiprocessing as mp


def test_assign_balances_and_covers():
    from forcepho_b200.dispatch import assign
    costs = [5, 1, 4, 2, 3, 3, 7, 1]
    parts = assign(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert parts == assign(costs, 3)          # deterministic


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from forcepho_b200.dispatch import dispatch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = list(range(10))
        res = dispatch(jobs, lambda j: (j * j, dist.get_rank()), cost_fn=lambda j: 1 + j % 3)
        if rank == 0:
            out.put(res)
    finally:
        dist.destroy_process_group()


def test_dispatch_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [j * j for j in range(10)]
    assert {r[1] for r in res} == {0, 1}


def test_dispatch_single_process():
    from forcepho_b200.dispatch import dispatch
    assert dispatch([1, 2, 3], lambda j: j + 1) == [2, 3, 4]
