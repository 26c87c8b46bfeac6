"""The seeded Grid built on the GPU (es_dgrid_*) against the host Grid
(reference Grid::Grid(seed, ...), src/sim/Grid.cpp:28-188), through the C ABI.

Integer and byte work: the impurity positions, the ordered (cell-major) array
and the cumulative cell index must be the host Grid's bit for bit, and a pass
computed on the device-built grid must give the host-built grid's lifetimes
and sigma exactly.
"""
from __future__ import annotations

import numpy as np
import pytest

from elasticscattering_b200 import DeviceGrid, EsError, Grid, SimulationCUDA, make_settings, workloads
from elasticscattering_b200 import _native as N
from elasticscattering_b200.batch import BatchPass, BatchSweep

pytestmark = pytest.mark.gpu


def _cases():
    c0, c1, c3 = workloads.config0(), workloads.config1(), workloads.config3()
    sweep = workloads.config2(n_samples=64, n_fields=2)
    out = [
        ("config0", c0.seed(0), c0.region_size, c0.region_extends, c0.density, c0.impurity_radius,
         c0.target_cell_population),
        ("config1", c1.seed(0), c1.region_size, c1.region_extends, c1.density, c1.impurity_radius,
         c1.target_cell_population),
        # the stress case's large disks (r_i 5e-9 m) and dense field: many corner filings
        ("config3", c3.seed(0), c3.region_size, c3.region_extends, c3.density, c3.impurity_radius,
         c3.target_cell_population),
    ]
    for k, tcp in ((0, 8), (1, 12), (6, 4)):
        s = sweep.samples[k]
        out.append((f"sweep-sample-{k}", s.seed, sweep.region_size, sweep.region_extends, s.density,
                    sweep.impurity_radius, tcp))
    out += [
        # seeds that pass through a negative int, and the zero state minstd_rand0 maps to 1
        ("seed-negative-int", 0xFFFFFFF0, 1e-6, 5e-7, 2e15, 2e-9, 3),
        ("seed-2^31", 0x80000000, 1e-6, 5e-7, 2e15, 2e-9, 3),
        ("seed-zero", 0, 1e-6, 5e-7, 2e15, 2e-9, 3),
        ("seed-m", 2147483647, 1e-6, 5e-7, 2e15, 2e-9, 3),
        # one cell per impurity; disks as large as the cells (every probe and corner rule)
        ("tcp-1", 12345, 1e-6, 2e-7, 5e15, 2e-9, 1),
        ("large-disks", 777, 1e-6, 2e-7, 1e15, 2.5e-8, 2),
        # two impurities in a single cell
        ("tiny", 5, 1e-7, 0.0, 1.5e14, 2e-9, 1),
    ]
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_device_grid_is_the_host_grid(cuda_device, case):
    name, seed, size, ext, dens, r, tcp = case
    h = Grid.from_seed(seed, size, ext, dens, r, tcp)
    d = DeviceGrid.from_seed(seed, size, ext, dens, r, tcp, device=cuda_device)
    try:
        hs, ds = h.GetSettings(), d.GetSettings()
        for f in ("spawn_region_start", "spawn_region_size", "cell_size", "cells_per_row", "impurity_radius"):
            assert getattr(hs, f) == getattr(ds, f), f
        assert h.GetUniqueImpurityCount() == d.GetUniqueImpurityCount()
        assert h.GetTotalImpurityCount() == d.GetTotalImpurityCount()
        assert np.array_equal(h.GetIndex(), d.GetIndex())
        a, b = h.GetImpurities(), d.GetImpurities()
        assert a.shape == b.shape
        assert np.array_equal(a.view(np.int64), b.view(np.int64))
    finally:
        d.close()


def test_device_grid_errors_match_the_host(cuda_device):
    with pytest.raises(EsError, match="Woah"):
        DeviceGrid.from_seed(1, 1e-6, 1e-4, 1e16, 2e-9, 12, device=cuda_device)
    with pytest.raises(EsError, match="No impurities"):
        DeviceGrid.from_seed(1, 1e-9, 0.0, 1e10, 2e-9, 12, device=cuda_device)
    with pytest.raises(EsError):
        DeviceGrid.from_seed(1, 1e-6, 1e-7, 1e15, 2e-9, 0, device=cuda_device)


def test_pass_on_device_grid_is_bit_identical(cuda_device):
    w = workloads.config0()
    h = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    d = DeviceGrid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                             w.target_cell_population, device=cuda_device)
    st = make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                       w.impurity_radius, w.target_cell_population)
    try:
        for prec in (N.ES_PRECISION_FP64, N.ES_PRECISION_SPLIT):
            res = []
            for g in (h, d):
                with SimulationCUDA(w.dim, w.phi_steps, g.info(), device=cuda_device, precision=prec) as sim:
                    sim.InitSample(g, st, False)
                    lt, m = sim.ComputeLifetimes(20.0)
                    sig = sim.DeriveTemperatures([1e-3, 10.0])
                    res.append((lt, m, [(s.xx, s.xy) for s in sig]))
            assert np.array_equal(res[0][0].view(np.int64), res[1][0].view(np.int64))
            assert res[0][1] == res[1][1]
            assert res[0][2] == res[1][2]
        # the batched path
        sig = []
        for g in (h, d):
            with BatchSweep(cuda_device) as b:
                gid = b.add_grid(g)
                b.set_passes([BatchPass(gid, w.dim, w.phi_steps, coh, w.region_size, g.info().cell_size, 20.0, st,
                                        [1e-3, 10.0]) for coh in (True, False)])
                out, _ = b.run()
                sig.append(out.copy())
        assert np.array_equal(sig[0], sig[1])
    finally:
        d.close()
