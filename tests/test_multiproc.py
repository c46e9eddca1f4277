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


def _slab_worker(rank, world, port, periodic, q):
    """One part's exchange and all-reduce over gloo with CPU tensors: every buffer is tagged with its rank and side."""
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import torch

        from fenice_b200.slabs import DistExchange

        n = 7
        send_lo = torch.full((n,), 100.0 * rank + 1.0, dtype=torch.float64)
        send_hi = torch.full((n,), 100.0 * rank + 2.0, dtype=torch.float64)
        recv_lo = torch.full((n,), -1.0, dtype=torch.float64)
        recv_hi = torch.full((n,), -1.0, dtype=torch.float64)
        red = torch.tensor([float(rank), 10.0 - rank], dtype=torch.float64)
        peer_lo = periodic or rank > 0
        peer_hi = periodic or rank < world - 1
        ex = DistExchange([send_lo, send_hi, recv_lo, recv_hi, red], peer_lo, peer_hi)
        ex.exchange()
        ex.allreduce(2)
        q.put((rank, float(recv_lo[0]), float(recv_hi[0]), bool((recv_lo == recv_lo[0]).all() and (recv_hi == recv_hi[0]).all()), red.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
@pytest.mark.parametrize("world,periodic", [(2, False), (2, True), (3, False), (3, True)])
def test_slab_exchange_routes_planes_to_neighbours(world, periodic):
    """Each part's low ghost planes receive its low neighbour's high planes and vice versa (a periodic axis joins the last
    part to the first; with two parts both neighbours are one rank); the all-reduce gives every rank the maximum."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() + 7 * world + (1 if periodic else 0)) % 300
    procs = [ctx.Process(target=_slab_worker, args=(r, world, port, periodic, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=200) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, lo, hi, uniform, red in res:
        assert uniform
        lo_n, hi_n = (rank - 1) % world, (rank + 1) % world
        assert lo == (100.0 * lo_n + 2.0 if (periodic or rank > 0) else -1.0)          # the low neighbour's send_hi
        assert hi == (100.0 * hi_n + 1.0 if (periodic or rank < world - 1) else -1.0)  # the high neighbour's send_lo
        assert red == [float(world - 1), 10.0]
