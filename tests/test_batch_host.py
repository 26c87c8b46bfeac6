"""Host-side logic of the batched sweep (no GPU): the config-2 draw, the pass list,
the pass records handed to the C ABI and the autotuner's bookkeeping."""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import asdict

import numpy as np
import pytest

from elasticscattering_b200 import _native as N
from elasticscattering_b200 import workloads
from elasticscattering_b200.autotune import TuneResult, signature
from elasticscattering_b200.batch import BatchPass, incoherent_temperature, sweep_passes
from elasticscattering_b200.simulation import make_settings


def test_config2_draw_is_reproducible_and_in_range():
    a, b = workloads.config2(), workloads.config2()
    assert [(s.seed, s.dim, s.density) for s in a.samples] == [(s.seed, s.dim, s.density) for s in b.samples]
    assert len(a.samples) == 64 and len(a.fields) == 32
    assert a.fields[0] == 1.0 and a.fields[-1] == 40.0
    assert np.allclose(np.diff(a.fields), 39.0 / 31.0)
    assert {s.dim for s in a.samples} <= {129, 257, 513}
    assert all(1e15 <= s.density <= 1e16 for s in a.samples)
    # Grid seed of sample k with start_seed 0 (src/SimulationConfiguration.h:209-210)
    assert [s.seed for s in a.samples[:3]] == [100, 200, 300]
    assert a.temperatures == [0.0, 10.0, 40.0]
    assert a.region_extends == pytest.approx(workloads.orbit_diameter(1.68e5, 1.0))
    assert a.sigma_points == 64 * 32 * 3
    c = workloads.config2(draw_seed=1)
    assert [s.dim for s in c.samples] != [s.dim for s in a.samples]


def test_sweep_passes_order_and_temperatures():
    wl = workloads.config2(n_samples=3, n_fields=4)
    ids = {s.index: 10 + s.index for s in wl.samples}
    cells = {s.index: 5e-8 for s in wl.samples}
    passes = sweep_passes(wl, ids, cells)
    assert len(passes) == 3 * 4 * 2
    # per sample, per field: coherent then incoherent (SimulationRunner.cpp:91-92)
    assert [p.coherent for p in passes[:4]] == [True, False, True, False]
    assert passes[0].magnetic_field == passes[1].magnetic_field == 1.0
    assert passes[0].grid == 10 and passes[-1].grid == 12
    assert passes[0].temperatures == [workloads.T_ZERO_STANDIN, 10.0, 40.0]
    assert incoherent_temperature(0.0) == workloads.T_ZERO_STANDIN
    assert passes[0].settings.impurity_density == wl.samples[0].density
    assert passes[-1].n_orbits == wl.samples[2].dim ** 2 * 4 * wl.phi_steps


def test_batch_pass_record_layout():
    st = make_settings(1e-12, 0.3, True, 1.68e5, 1e-6, 2e-6, 1e15, 2e-9, 12)
    p = BatchPass(3, 33, 9, False, 1e-6, 5e-8, 7.5, st, [1.0, 2.0])
    c = p.to_c()
    assert (c.grid, c.positions_per_row, c.particles_per_quadrant, c.coherent) == (3, 33, 9, 0)
    assert c.magnetic_field == 7.5 and c.n_t == 2
    assert list(c.temperatures)[:3] == [1.0, 2.0, 0.0]
    assert c.settings.particle_speed == 1.68e5
    # es_batch_instance: 4 int32, 3 doubles, es_settings, n_t (padded), 8 doubles
    assert C.sizeof(N.BatchInstance) == 16 + 24 + C.sizeof(N.Settings) + 8 + 64
    assert C.sizeof(N.BatchTuning) == 16
    with pytest.raises(ValueError):
        BatchPass(0, 33, 9, False, 1e-6, 5e-8, 7.5, st, list(range(1, 10))).to_c()


def test_tune_result_classes_and_cache_round_trip(tmp_path):
    r = TuneResult(key="k", density_edges=[1e15, 2e15, 5e15, 1e16], tcp=[4, 12, 20],
                   shape={"mode": 2, "blocks_per_sm": 4, "chunk_iters": 32})
    assert r.tcp_for(1e15) == 4
    assert r.tcp_for(3e15) == 12
    assert r.tcp_for(9.99e15) == 20
    assert r.tcp_for(1e16) == 20  # the top edge belongs to the last class
    p = tmp_path / "t.json"
    p.write_text(json.dumps({"k": asdict(r)}))
    assert TuneResult(**json.loads(p.read_text())["k"]) == r


def test_tuner_signature_tracks_the_workload():
    a = workloads.config2(n_samples=8)
    b = workloads.config2(n_samples=8, n_fields=16)
    assert signature(a, 3) == signature(workloads.config2(n_samples=8), 3)
    assert signature(a, 3) != signature(b, 3)
    assert signature(a, 3) != signature(a, 2)
