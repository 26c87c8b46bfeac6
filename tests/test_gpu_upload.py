"""Grid uploads from pageable host memory and the batch's reuse of cleared grid
memory.

- es_upload_grid / es_batch_add_grid copy a pageable host Grid through a pinned
  staging ring in 16 MiB chunks (csrc/es_upload.cu). A config-1 grid (2.3 M
  indexed impurities, 37 MB: two full chunks and a partial one) uploaded that
  way, from a pinned copy of the same arrays, and built on the GPU
  (DeviceGrid, bit-identical to the host Grid) must give the same lifetimes
  and sigma bit for bit.
- es_batch_clear keeps the grids' device memory and es_batch_add_grid reuses
  the smallest cleared allocation that fits. Clearing and adding the same
  grids again, in another order, or a larger grid that fits no kept
  allocation, must give what a fresh batch gives, bit for bit.
The reference uploads with blocking clEnqueueWriteBuffer calls
(src/sim/SimulationCL.cpp:121-122) and has no batch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from elasticscattering_b200 import DeviceGrid, Grid, SimulationCUDA, make_settings, workloads
from elasticscattering_b200 import _native as N
from elasticscattering_b200.batch import BatchPass, BatchSweep

pytestmark = pytest.mark.gpu

W = workloads.config1()
TEMPS = [1.0, 10.0, 40.0]


def _settings(w=W):
    return make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                         w.impurity_radius, w.target_cell_population)


def _lifetimes_and_sigma(sim, field=20.0):
    lt, _ = sim.ComputeLifetimes(field)
    sig = sim.ComputeSigmas(field, TEMPS)
    return lt, [v for s in sig for v in (s.xx, s.xy)]


@pytest.mark.parametrize("precision", [N.ES_PRECISION_FP64, N.ES_PRECISION_SPLIT])
def test_staged_pinned_and_device_uploads_agree(cuda_device, precision):
    import torch

    seed = W.seed(0)
    grid = Grid.from_seed(seed, W.region_size, W.region_extends, W.density, W.impurity_radius,
                          W.target_cell_population)
    n = grid.GetTotalImpurityCount()
    assert n * 16 > 2 * (16 << 20), "the grid must span more than two staging chunks"
    st = _settings()
    dim, ppq = 33, 25
    out = {}
    with SimulationCUDA(dim, ppq, grid.info(), precision=precision) as sim:
        sim.InitSample(grid, st, False)  # pageable: the staging ring
        out["staged"] = _lifetimes_and_sigma(sim)
        pin_xy = torch.from_numpy(grid.GetImpurities().ravel()).pin_memory()
        pin_idx = torch.from_numpy(grid.GetIndex()).pin_memory()
        s = grid.GetSettings()
        # a new generation forces the upload, now from pinned memory (a direct copy)
        sim._check(N.cuda_lib().es_upload_grid(sim.ctx, C.c_void_p(pin_xy.data_ptr()), n,
                                               C.c_void_p(pin_idx.data_ptr()), C.byref(s), 12345))
        out["pinned"] = _lifetimes_and_sigma(sim)
    dg = DeviceGrid.from_seed(seed, W.region_size, W.region_extends, W.density, W.impurity_radius,
                              W.target_cell_population)
    with SimulationCUDA(dim, ppq, dg.info(), precision=precision) as sim:
        sim.InitSample(dg, st, False)
        out["device"] = _lifetimes_and_sigma(sim)
    dg.close()
    for k in ("pinned", "device"):
        assert np.array_equal(out[k][0], out["staged"][0]), k
        assert out[k][1] == out["staged"][1], k


def _grids():
    """Three host grids of different sizes (the last one the largest)."""
    ext = workloads.orbit_diameter(W.particle_speed, 5.0)
    specs = [(101, 2e15), (202, 6e15), (303, 1.2e16)]
    return ext, [(Grid.from_seed(seed, W.region_size, ext, dens, W.impurity_radius, 12), dens)
                 for seed, dens in specs]


def _passes(ext, grids, ids):
    ps = []
    for (g, dens), gid in zip(grids, ids):
        st = make_settings(W.tau, W.alpha, True, W.particle_speed, W.region_size, ext, dens, W.impurity_radius, 12)
        for b in (5.0, 30.0):
            for coh in (True, False):
                ps.append(BatchPass(gid, 33, 9, coh, W.region_size, g.info().cell_size, b, st, list(TEMPS)))
    return ps


def _run_fresh(ext, grids):
    with BatchSweep(precision=N.ES_PRECISION_SPLIT) as bs:
        ids = [bs.add_grid(g) for g, _ in grids]
        bs.set_passes(_passes(ext, grids, ids))
        out, mets = bs.run()
    return out, mets


def test_batch_reuses_cleared_grid_memory(cuda_device):
    ext, grids = _grids()
    assert grids[0][0].GetTotalImpurityCount() < grids[1][0].GetTotalImpurityCount() \
        < grids[2][0].GetTotalImpurityCount()
    ref, ref_m = _run_fresh(ext, grids)
    with BatchSweep(precision=N.ES_PRECISION_SPLIT) as bs:
        ids = [bs.add_grid(g) for g, _ in grids]
        bs.set_passes(_passes(ext, grids, ids))
        first, _ = bs.run()
        assert np.array_equal(first, ref)
        # same grids again: every one takes its own kept allocation
        bs.clear()
        ids = [bs.add_grid(g) for g, _ in grids]
        bs.set_passes(_passes(ext, grids, ids))
        again, again_m = bs.run()
        assert np.array_equal(again, ref) and again_m == ref_m
        # reverse order: the smallest kept allocation that fits each
        bs.clear()
        rev = list(reversed(grids))
        rid = [bs.add_grid(g) for g, _ in rev]
        bs.set_passes(_passes(ext, rev, rid))
        out_rev, _ = bs.run()
        n_per = 4  # passes per grid
        expect = np.concatenate([ref[n_per * k:n_per * (k + 1)] for k in (2, 1, 0)])
        assert np.array_equal(out_rev, expect)
        # only the two small grids, then a larger one than any kept allocation
        bs.clear()
        big = [(Grid.from_seed(404, W.region_size, ext, 3e16, W.impurity_radius, 12), 3e16)]
        bid = [bs.add_grid(g) for g, _ in big]
        bs.set_passes(_passes(ext, big, bid))
        out_big, _ = bs.run()
    fresh_big, _ = _run_fresh(ext, big)
    assert np.array_equal(out_big, fresh_big)
