"""The reference-side binding (elasticscattering_b200/refbind/SimulationCUDA.h),
compiled against the reference's own headers into oracle/_ref/libes_refbind.so.

On the CPU: the library loads, and its sweep loop through the reference's
SimulationCPU (backend 0) reproduces the reference's sigmas as the plain
reference build computes them. The CUDA backend is exercised by
tests/test_gpu_refbind.py."""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as O
import refbind_lib as RB
from elasticscattering_b200 import workloads

pytestmark = pytest.mark.skipif(not (RB.available() and O.ref_available()),
                                reason="oracle/_ref/libes_refbind.so not built (reference tree absent)")


def test_binding_library_exports_the_sweep_entry():
    assert hasattr(RB.lib(), "rb_sweep")


def test_cpu_backend_through_the_binding_harness_is_the_reference():
    w = workloads.config0()
    dim, ppq, fields, temps = 17, 7, [20.0, 5.0], [1e-3, 10.0]
    seeds = [w.seed(0), w.seed(1)]
    out, met, avg, _ = RB.sweep(0, w, seeds, dim, ppq, fields, temps)
    lib = O.ref()
    for s, seed in enumerate(seeds):
        g = lib.ref_grid_new_seed(seed, w.region_size, w.region_extends, w.density, w.impurity_radius,
                                  w.target_cell_population)
        for sector, coh in enumerate((1, 0)):
            sim = lib.ref_sim_new(g, dim, ppq, w.tau, w.alpha, int(w.clockwise), w.particle_speed, w.region_size,
                                  w.region_extends)
            lib.ref_sim_init_sample(sim, coh)
            for f, B in enumerate(fields):
                o = np.zeros(2 * len(temps))
                m = np.zeros(7, dtype=np.int32)
                lib.ref_sim_sigmas(sim, B, np.asarray(temps).ctypes.data, len(temps), o.ctypes.data, m.ctypes.data)
                assert out[s, sector, f].ravel().tolist() == o.tolist()
                assert met[s, sector, f].tolist() == m.tolist()
            lib.ref_sim_free(sim)
        lib.ref_grid_free(g)
    assert (avg > 0).all()
