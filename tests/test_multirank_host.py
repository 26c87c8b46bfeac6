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


# ---- LPT partitioning, slices, row splits ----------------------------------

def test_lpt_partition_is_deterministic_disjoint_and_balanced():
    wl = workloads.config2()
    costs = [workloads.sample_cost(wl, s) for s in wl.samples]
    for world in (1, 2, 3, 4, 8):
        parts = workloads.lpt_partition(costs, world)
        assert parts == workloads.lpt_partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        mean = sum(costs) / world
        # LPT's bound: the largest load is below mean + the largest item
        assert max(loads) <= mean + max(costs)
        if world > 1:
            per = len(costs) // world
            contiguous = [sum(costs[r * per:(r + 1) * per]) for r in range(world)]
            assert max(loads) <= max(contiguous)
    # 8 GPUs over the 64-sample draw: within 1% of a perfect split
    loads = [sum(costs[i] for i in p) for p in workloads.lpt_partition(costs, 8)]
    assert max(loads) <= 1.01 * sum(costs) / 8
    shards = [workloads.lpt_shard(wl, r, 4) for r in range(4)]
    assert sorted(s.index for sh in shards for s in sh.samples) == list(range(64))


def test_sample_cost_grows_with_orbits_and_density():
    wl = workloads.config2()
    a, b, c = (workloads.SweepSample(0, 100, d, dens) for d, dens in ((129, 5e15), (257, 5e15), (257, 1e15)))
    assert workloads.sample_cost(wl, b) > 3.9 * workloads.sample_cost(wl, a)
    # a thinner field has longer walks
    assert workloads.sample_cost(wl, c) > workloads.sample_cost(wl, b)


def test_representative_slices_are_disjoint_with_one_sample_per_start_grid():
    wl = workloads.config2()
    per_pass = 4 * wl.phi_steps * 2 * len(wl.fields)

    def cost_per_orbit(samples):
        return sum(workloads.sample_cost(wl, s) for s in samples) / (sum(s.dim ** 2 for s in samples) * per_pass)

    target = cost_per_orbit(wl.samples)
    seen = set()
    for k in range(8):
        sl = workloads.representative_slice(wl, k)
        assert sorted(s.dim for s in sl.samples) == [129, 257, 513]
        # each slice's estimated cost per orbit stands for the whole draw's
        assert abs(cost_per_orbit(sl.samples) - target) <= 0.07 * target, k
        idx = {s.index for s in sl.samples}
        assert not (idx & seen)
        seen |= idx
        assert sl.fields == wl.fields and sl.temperatures == wl.temperatures
    with pytest.raises(ValueError):
        workloads.representative_slice(wl, 40)


def test_row_split_covers_every_row_once():
    for dim, world in ((1025, 8), (257, 3), (5, 5)):
        spans = [workloads.row_split(dim, r, world) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == dim
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1
    with pytest.raises(ValueError):
        workloads.row_split(3, 0, 4)


# ---- FinishResults after the gather ----------------------------------------

def test_finish_results_follows_the_reference_arithmetic():
    from elasticscattering_b200.batch import finish_results
    rng = np.random.default_rng(3)
    coh = rng.uniform(0.1, 1.0, size=(5, 2, 3, 2))
    inc = rng.uniform(0.1, 1.0, size=(5, 2, 3, 2))
    r = finish_results(coh, inc)
    for f in range(2):
        for t in range(3):
            cs = [0.0, 0.0]
            isum = [0.0, 0.0]
            dsq = 0.0
            for s in range(5):  # src/SimulationRunner.cpp:166-173, in sample order
                cs = [cs[0] + coh[s, f, t, 0], cs[1] + coh[s, f, t, 1]]
                isum = [isum[0] + inc[s, f, t, 0], isum[1] + inc[s, f, t, 1]]
                dsq += (coh[s, f, t, 0] + inc[s, f, t, 0]) ** 2
            c = [cs[0] / 5.0, cs[1] / 5.0]
            i = [isum[0] / 5.0, isum[1] / 5.0]
            e = c[0] + i[0]
            assert r["coherent"][f, t].tolist() == c and r["incoherent"][f, t].tolist() == i
            assert r["delta_xx"][f, t] == np.sqrt((dsq / 5.0 - e * e) / 4.0) / e
    one = finish_results(coh[:1], inc[:1])
    assert (one["delta_xx"] == 0).all()


TINY = {"dim": 9, "ppq": 5, "fields": [10.0, 40.0], "temps": [1e-3, 10.0], "samples": 4}


def _tiny_sweep():
    wl = workloads.config2(n_samples=TINY["samples"], n_fields=2)
    wl.fields = list(TINY["fields"])
    wl.temperatures = list(TINY["temps"])
    wl.phi_steps = TINY["ppq"]
    for s in wl.samples:
        s.dim = TINY["dim"]
    return wl


def _sample_sigmas_ref(wl, s):
    """One sample's sweep on the reference's own CPU build (oracle/_ref):
    coherent and incoherent sigma per (field, temperature)."""
    import oracle_lib as O
    lib = O.ref()
    g = lib.ref_grid_new_seed(s.seed, wl.region_size, wl.region_extends, s.density, wl.impurity_radius,
                              wl.target_cell_population)
    out = []
    for coh in (1, 0):
        sim = lib.ref_sim_new(g, s.dim, wl.phi_steps, wl.tau, wl.alpha, int(wl.clockwise), wl.particle_speed,
                              wl.region_size, wl.region_extends)
        lib.ref_sim_init_sample(sim, coh)
        temps = np.asarray(wl.temperatures, dtype=np.float64)
        arr = np.zeros((len(wl.fields), len(temps), 2))
        for f, B in enumerate(wl.fields):
            o = np.zeros(2 * len(temps))
            lib.ref_sim_sigmas(sim, float(B), temps.ctypes.data, len(temps), o.ctypes.data, None)
            arr[f] = o.reshape(len(temps), 2)
        lib.ref_sim_free(sim)
        out.append(arr)
    lib.ref_grid_free(g)
    return out[0], out[1]


def _rank_sigma_main(rank: int, world: int, port: int, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    from elasticscattering_b200.batch import finish_results, gather_sweep
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        wl = _tiny_sweep()
        mine = workloads.lpt_partition([workloads.sample_cost(wl, s) for s in wl.samples], world)[rank]
        local = {i: _sample_sigmas_ref(wl, wl.samples[i]) for i in mine}
        coh, inc = gather_sweep(local, len(wl.samples), dist)
        r = finish_results(coh, inc)
        q.put((rank, sorted(mine), {k: v.tolist() for k, v in r.items()}))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_real_sigmas_and_finish_like_one_process():
    """World size 2 over gloo: each rank computes real per-sample sigmas (the
    reference's CPU build) for its LPT share of a tiny 4-sample sweep, the
    sigmas are gathered, and FinishResults' sample averages and delta_xx equal
    those of the same sweep run in one process, bit for bit."""
    import oracle_lib as O
    if not O.ref_available():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    from elasticscattering_b200.batch import finish_results, gather_sweep
    world = 2
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank_sigma_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, mine, res = q.get(timeout=300)
        out[rank] = (mine, res)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(out[0][0] + out[1][0]) == list(range(TINY["samples"])) and out[0][0] and out[1][0]
    wl = _tiny_sweep()
    single = {s.index: _sample_sigmas_ref(wl, s) for s in wl.samples}
    ref = finish_results(*gather_sweep(single, len(wl.samples)))
    for rank in range(world):
        for k, v in ref.items():
            assert out[rank][1][k] == v.tolist(), (rank, k)
    assert np.all(ref["delta_xx"] > 0)
