"""es_set_rows: a sector pass split by start rows (the multi-GPU split of one
pass too large for one GPU), checked on one GPU. Each row range is computed in
its own context, as each GPU would; the ranges' lifetimes are the whole pass's,
bit for bit, and their sigma shares, summed in range order, give the whole
pass's sigma (only the summation order differs)."""
from __future__ import annotations

import numpy as np
import pytest

from elasticscattering_b200 import EsError, Grid, SimulationCUDA, make_settings, workloads
from elasticscattering_b200 import _native as N

pytestmark = pytest.mark.gpu

TEMPS = [1e-3, 10.0, 40.0]


def _settings(w):
    return make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                         w.impurity_radius, w.target_cell_population)


@pytest.mark.parametrize("precision", [N.ES_PRECISION_FP64, N.ES_PRECISION_SPLIT])
@pytest.mark.parametrize("coherent", [True, False])
def test_row_ranges_add_up_to_the_whole_pass(cuda_device, precision, coherent):
    w = workloads.config0()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    s = _settings(w)
    per_row = w.dim * 4 * w.phi_steps
    with SimulationCUDA(w.dim, w.phi_steps, g.info(), device=cuda_device, precision=precision) as whole:
        whole.InitSample(g, s, coherent)
        lt, m = whole.ComputeLifetimes(20.0)
        full = whole.DeriveTemperatures(TEMPS)
    world = 3
    shares, cells = [], 0
    for r in range(world):
        j0, j1 = workloads.row_split(w.dim, r, world)
        with SimulationCUDA(w.dim, w.phi_steps, g.info(), device=cuda_device, precision=precision) as part:
            part.InitSample(g, s, coherent)
            part.SetRows(j0, j1)
            _, mr = part.ComputeLifetimes(20.0, copy=False)
            cells += mr["cells_passed"]
            mine = part.ReadLifetimes(j0 * per_row, (j1 - j0) * per_row)
            assert np.array_equal(mine.view(np.int64), lt[j0 * per_row:j1 * per_row].view(np.int64)), (r, j0, j1)
            shares.append(part.DeriveTemperatures(TEMPS))
            with pytest.raises(EsError):
                part.ComputeSigmasWithImages(20.0, TEMPS)
    assert cells == m["cells_passed"]
    for t in range(len(TEMPS)):
        xx = sum(sh[t].xx for sh in shares)
        xy = sum(sh[t].xy for sh in shares)
        assert abs(xx - full[t].xx) <= 1e-12 * abs(full[t].xx), (t, xx, full[t].xx)
        assert abs(xy - full[t].xy) <= 1e-12 * abs(full[t].xy), (t, xy, full[t].xy)


def test_row_split_of_a_full_size_1025_squared_pass(cuda_device):
    """1025^2 x 1028 orbits, B = 40 T, split precision: two row ranges against the
    whole pass."""
    w = workloads.config3()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    s = _settings(w)
    with SimulationCUDA(w.dim, w.phi_steps, g.info(), device=cuda_device, precision=N.ES_PRECISION_SPLIT) as sim:
        sim.InitSample(g, s, False)
        sim.ComputeLifetimes(40.0, copy=False)
        full = sim.DeriveTemperatures(TEMPS)
        parts = []
        for r in range(2):
            sim.SetRows(*workloads.row_split(w.dim, r, 2))
            sim.ComputeLifetimes(40.0, copy=False)
            parts.append(sim.DeriveTemperatures(TEMPS))
    for t in range(len(TEMPS)):
        assert abs(parts[0][t].xx + parts[1][t].xx - full[t].xx) <= 1e-12 * abs(full[t].xx)
        assert abs(parts[0][t].xy + parts[1][t].xy - full[t].xy) <= 1e-12 * abs(full[t].xy)


def test_set_rows_rejects_bad_ranges(cuda_device):
    w = workloads.config0()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    with SimulationCUDA(w.dim, w.phi_steps, g.info(), device=cuda_device) as sim:
        for j0, j1 in ((-1, 3), (3, 3), (5, 2), (0, w.dim + 1)):
            with pytest.raises(EsError):
                sim.SetRows(j0, j1)
