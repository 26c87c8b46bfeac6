"""The drop-in, compiled: the reference's own sweep loop (RunSimulation /
RunSample, one Simulation object for every sample, InitSample per sector,
ComputeSigmas per field) driving the reference-side binding SimulationCUDA
through a `Simulation*`, against the same loop on the reference's SimulationCPU.

Bars: sigma within 1e-9 relative (the parity bar), the reference's metric
counters equal, the average lifetime within 1e-9, the images path's per-position
maps within 1e-9 of their largest value; and the binding's sigma equals
es_compute_sigmas called directly, bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as O
import refbind_lib as RB
from elasticscattering_b200 import Grid, SimulationCUDA, make_settings, workloads

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (RB.available() and O.ref_available()),
                                 reason="oracle/_ref/libes_refbind.so not built")]

RTOL = 1e-9


def test_binding_matches_the_reference_cpu_backend(cuda_device):
    w = workloads.config0()
    fields, temps = [20.0, 5.0], [1e-3, 10.0]
    seeds = [w.seed(0), w.seed(1), w.seed(2)]
    cpu = RB.sweep(0, w, seeds, w.dim, w.phi_steps, fields, temps)
    gpu = RB.sweep(1, w, seeds, w.dim, w.phi_steps, fields, temps)
    assert np.all(np.abs(gpu[0] - cpu[0]) <= RTOL * np.abs(cpu[0]))
    assert np.array_equal(gpu[1], cpu[1])
    assert np.all(np.abs(gpu[2] - cpu[2]) <= RTOL * np.abs(cpu[2]))
    # the binding forwards to the C ABI: the same sigma as calling it directly
    s = make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                      w.impurity_radius, w.target_cell_population)
    g = Grid.from_seed(seeds[1], w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    with SimulationCUDA(w.dim, w.phi_steps, g.info(), device=cuda_device) as sim:
        for sector, coh in enumerate((True, False)):
            sim.InitSample(g, s, coh)
            for f, B in enumerate(fields):
                direct = sim.ComputeSigmas(B, temps)
                assert [[x.xx, x.xy] for x in direct] == gpu[0][1, sector, f].tolist()


def test_binding_images_path_matches_the_reference(cuda_device):
    w = workloads.config0()
    dim, ppq, fields, temps = 33, 9, [20.0], [1e-3, 10.0]
    cpu = RB.sweep(0, w, [w.seed(0)], dim, ppq, fields, temps, images=True)
    gpu = RB.sweep(1, w, [w.seed(0)], dim, ppq, fields, temps, images=True)
    assert np.all(np.abs(gpu[0] - cpu[0]) <= RTOL * np.abs(cpu[0]))
    assert np.array_equal(gpu[1], cpu[1])
    scale = np.abs(cpu[3]).max(axis=-1, keepdims=True)
    assert np.all(np.abs(gpu[3] - cpu[3]) <= RTOL * scale)
