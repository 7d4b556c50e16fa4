"""The bench's multi-rank host logic on CPU: two gloo ranks reduce the timed
region's max and the ensemble's total cells over ranks, and step disjoint
ensemble shards (no GPU needed)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mx = bench.reduce_over_ranks(dist, 1.5 + rank)
        sm = bench.reduce_over_ranks(dist, 10.0 * (rank + 1), op="sum")
        shard = bench.ensemble_shard(rank)
        out.put((rank, mx, sm, [kw["mesh"] for kw, _ in shard[:8]], len(shard)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, mx0, sm0, m0, n0), (r1, mx1, sm1, m1, n1) = res
    assert mx0 == mx1 == 2.5            # max over ranks of 1.5 and 2.5
    assert sm0 == sm1 == 30.0           # sum over ranks of 10 and 20
    assert n0 == n1 == 256
    assert m0 != m1                     # the shards are different simulations


def test_single_process_reduction_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(None, 3.25) == 3.25
    assert bench.reduce_over_ranks(None, 3.25, op="sum") == 3.25
