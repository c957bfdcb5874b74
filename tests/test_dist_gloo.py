"""The multi-GPU path on CPU: two gloo ranks shard an uneven ensemble between them and take the
max over ranks of their timings, as bench.py does under torchrun (one rank per GPU, independent
members, no data-path collective)."""

import datetime
import os
import socket
from types import SimpleNamespace

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _requests():
    out = []
    for i in range(13):
        L = (127, 255, 511)[i % 3]
        out.append(SimpleNamespace(rid=i, lmax=L, nsteps=50 + 97 * i, outer_passes=3 if i % 10 == 9 else 1))
    return out


def _worker(rank, world, port, results):
    import torch.distributed as dist

    from slevolve_b200.serving import max_over_ranks, request_cost, shard_requests

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        reqs = _requests()
        mine = shard_requests(reqs, rank, world)
        ids = [r.rid for r in mine]
        work = sum(request_cost(r) for r in mine)
        gathered = [None] * world
        dist.all_gather_object(gathered, (ids, work))
        t = max_over_ranks(0.5 + rank, dist, device="cpu")
        results[rank] = (gathered, t)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_sharding_and_max_timing():
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        results = mgr.dict()
        mp.spawn(_worker, args=(world, port, results), nprocs=world, join=True)
        res = dict(results)
    assert set(res) == {0, 1}
    gathered, t0 = res[0]
    assert res[1][0] == gathered and t0 == res[1][1] == 1.5
    ids = [i for ids, _ in gathered for i in ids]
    assert sorted(ids) == list(range(13)) and len(set(ids)) == 13   # disjoint, complete
    w0, w1 = gathered[0][1], gathered[1][1]
    assert max(w0, w1) / min(w0, w1) < 1.6                           # balanced work
