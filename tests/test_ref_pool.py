"""The multi-process runner of the reference's CPU build (tests/ref_pool.py),
which the full-size GPU parity tests use as their oracle, reproduces the
reference's own single-process SimulationCPU bit for bit: lifetimes, metric
counters and sigma, on config 0 and on a band of rows."""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as O
from elasticscattering_b200 import workloads
from ref_pool import RefPool, spec_of

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference tree absent)")


def test_pool_matches_serial_reference():
    w = workloads.config0()
    dim, temps = 33, [1e-3, 10.0]
    lib = O.ref()
    g = lib.ref_grid_new_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                              w.target_cell_population)
    with RefPool(procs=3) as pool:
        for coh in (True, False):
            spec = spec_of(w, w.seed(0), coh, 20.0, dim=dim)
            sim = lib.ref_sim_new(g, dim, w.phi_steps, w.tau, w.alpha, int(w.clockwise), w.particle_speed,
                                  w.region_size, w.region_extends)
            lib.ref_sim_init_sample(sim, int(coh))
            n = dim * dim * 4 * w.phi_steps
            serial = np.zeros(n)
            m = np.zeros(7, dtype=np.int32)
            lib.ref_sim_lifetimes(sim, 20.0, serial.ctypes.data, m.ctypes.data)
            sig = np.zeros(2 * len(temps))
            lib.ref_sim_sigmas(sim, 20.0, np.asarray(temps).ctypes.data, len(temps), sig.ctypes.data, None)
            lib.ref_sim_free(sim)
            (res,) = pool.run([spec], temperatures=temps, rows_per_task=5)
            assert np.array_equal(res.lifetimes().view(np.int64), serial.view(np.int64))
            assert [res.metrics[k] for k in ("cells_passed", "impurities_tested", "particles_inside_impurity",
                                             "particles_escaped", "particles_at_bound", "max_impurities_tested",
                                             "max_cells_passed")] == [int(v) for v in m]
            for t, T in enumerate(temps):
                assert res.sigmas[T] == (sig[2 * t], sig[2 * t + 1])
            # a band of rows only: the same orbits, no sigma
            (band,) = pool.run([spec], temperatures=temps, rows=(7, 12), rows_per_task=2)
            per_row = dim * 4 * w.phi_steps
            assert np.array_equal(band.lifetimes(), serial[7 * per_row:12 * per_row])
            assert band.sigmas == {}
            pool.discard([res, band])
    lib.ref_grid_free(g)
