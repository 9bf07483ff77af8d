"""Host logic of the multi-GPU path, the same functions bench.py calls: the weak-scaling
rate-set sweep split across ranks (bench.workload -> shards.rank_rate_sets) and the
max-over-ranks reduction (shards.max_over_ranks), run as gloo ranks on the CPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import bench
from paraexastolog_b200.shards import global_sweep, max_over_ranks, shard_bounds


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


def test_bench_single_rank_is_the_held_out_sweep():
    """At N=1 the bench solves exactly the 512 held-out rate sets of the learned workload."""
    from paraexastolog_b200 import synth

    _, rates, _, train, bounds = bench.workload(0, 1)
    w = synth.config_learned(n_rate_sets=4096)
    assert bounds == (0, bench.BATCH)
    assert np.array_equal(rates, w.rates[0][-bench.BATCH:])
    assert np.array_equal(train, w.rates[0][:bench.N_TRAIN])


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
    _, rates, _, _, bounds = bench.workload(rank, world)
    t = max_over_ranks([10.0 + rank, -float(rank)], world)
    q.put((rank, bounds, rates, t))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_cover_the_global_sweep_exactly_once(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=240) for _ in range(world)), key=lambda x: x[0])
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    # the ranks' slices tile [0, world * BATCH) in order, BATCH each
    assert [b for _, b, _, _ in res] == [(r * bench.BATCH, (r + 1) * bench.BATCH) for r in range(world)]
    got = np.concatenate([rates for _, _, rates, _ in res])
    _, held, _, _, _ = bench.workload(0, 1)
    from paraexastolog_b200 import synth
    n = held.shape[1] // 2
    want = global_sweep(held, world,
                        lambda seed, count: synth.log_uniform_rates(np.random.default_rng(10_000 + seed), n, count))
    assert np.array_equal(got, want)
    # every global rate set once: no two rows equal
    assert len(np.unique(got, axis=0)) == world * bench.BATCH
    assert np.array_equal(got[:bench.BATCH], held)
    # element-wise max over ranks
    assert all(t == [10.0 + world - 1, 0.0] for *_, t in res)
