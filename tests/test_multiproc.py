"""The multi-process plumbing on CPU ranks (gloo, world size 2): the cost split of a batch over ranks is a partition with
balanced loads, and the bench's reductions give the slowest rank's time and the sum of the ranks' work."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from fenice_b200 import initial
        from fenice_b200.runtime import batch_cost, split_batch

        params, _, _ = initial.shock_tubes(512, seed=0)
        mine = split_batch(params, world)[rank]
        lists = [None] * world
        dist.all_gather_object(lists, mine)
        load = sum(batch_cost(params[i]) for i in mine)
        slowest = bench.allmax(float(rank + 1), world)
        total = bench.allsum(load, world)
        q.put((rank, lists, load, slowest, total))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
def test_batch_split_and_reductions_on_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=200) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    lists = res[0][1]
    assert lists == res[1][1]
    flat = sorted(i for part in lists for i in part)
    assert flat == list(range(512))
    loads = [r[2] for r in res]
    assert max(loads) / (sum(loads) / 2) < 1.001
    assert all(r[3] == 2.0 for r in res)
    assert all(abs(r[4] - sum(loads)) <= 1e-6 * sum(loads) for r in res)
