"""Host logic of the multi-GPU path: rate-set shards and max-over-ranks timing,
run as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from paraexastolog_b200.shards import max_over_ranks, shard_bounds


@pytest.mark.parametrize("total,world", [(0, 2), (1, 2), (512, 1), (512, 2), (513, 4), (7, 8)])
def test_shards_cover_exactly_once(total, world):
    seen = []
    sizes = []
    for r in range(world):
        b, e = shard_bounds(total, r, world)
        seen.extend(range(b, e))
        sizes.append(e - b)
    assert seen == list(range(total))
    assert max(sizes) - min(sizes) <= 1


def test_shard_bounds_rejects_bad_rank():
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)
    with pytest.raises(ValueError):
        shard_bounds(10, 0, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    b, e = shard_bounds(512, rank, world)
    t = max_over_ranks(10.0 + rank, world)
    q.put((rank, b, e, t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    assert [(b, e) for _, b, e, _ in res] == [(0, 256), (256, 512)]
    assert all(t == 11.0 for *_, t in res)
