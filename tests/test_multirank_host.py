"""The multi-GPU sweep's host logic on CPU ranks (gloo, world size 2): sample
sharding is disjoint and complete, and the one exchange -- gathering every
rank's sigma results in rank order -- reassembles the single-process sweep."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as tmp

from elasticscattering_b200 import workloads


def _rank_main(rank: int, world: int, port: int, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        per = 3
        wl = workloads.shard_samples(workloads.config2(n_samples=64, n_fields=4), rank, world, per)
        # a stand-in per-sample result: deterministic in the sample's seed
        mine = torch.tensor([[s.seed, s.dim, s.density] for s in wl.samples], dtype=torch.float64)
        got = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(got, mine)
        q.put((rank, torch.cat(got).numpy().tolist()))
    finally:
        dist.destroy_process_group()


def test_sample_sharding_over_two_ranks():
    world = 2
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = workloads.config2(n_samples=64, n_fields=4)
    expect = [[s.seed, s.dim, s.density] for s in full.samples[:world * 3]]
    assert np.allclose(out[0], expect) and np.allclose(out[1], expect)


def test_shard_bounds():
    wl = workloads.config2(n_samples=8)
    assert [s.index for s in workloads.shard_samples(wl, 1, 2, 4).samples] == [4, 5, 6, 7]
    with pytest.raises(ValueError):
        workloads.shard_samples(wl, 2, 2, 4)
    with pytest.raises(ValueError):
        workloads.shard_samples(wl, 1, 2, 5)
