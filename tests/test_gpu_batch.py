"""Batched sweeps (es_batch_*) against the per-pass path, through the C ABI.

Each batched pass must reproduce what one Simulation::ComputeSigmas call
returns for it (src/sim/Simulation.h:128): the per-pass FP64 path
(SimulationCUDA, ES_PRECISION_FP64) is the reference. Bars:
- ES_PRECISION_FP64 batch: sigma within 1e-9 relative -- the plain path's parity
  bar; only the summation order and the fixed-point rounding of the work-item
  sums differ (observed ~1e-11 on sigma_xy, whose terms cancel) -- and identical
  metrics;
- ES_PRECISION_SPLIT batch: sigma within 1e-6 relative (FP32 Boltzmann kernel),
  identical metrics (every lifetime equals the FP64 one);
- runs are bit-reproducible, independent of the launch shape, and a replayed
  graph with a new instance table equals a fresh batch.
"""
from __future__ import annotations

import numpy as np
import pytest

from elasticscattering_b200 import Grid, SimulationCUDA, make_settings, workloads
from elasticscattering_b200 import _native as N
from elasticscattering_b200.simulation import SampleMetrics
from elasticscattering_b200.batch import BatchPass, BatchSweep, incoherent_temperature

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-9
SPLIT_RTOL = 1e-6
METRIC_KEYS = ("cells_passed", "impurities_tested", "crossings_tested", "particles_inside_impurity",
               "particles_escaped", "particles_at_bound", "max_cells_passed", "max_impurities_tested")

SPEED, ALPHA, TAU, L, R_IMP = 1.68e5, 0.3, 1e-12, 1e-6, 2e-9
FIELDS = (1.5, 7.0, 20.0, 40.0)
TEMPS = (0.0, 10.0, 40.0)
# (sample index, start positions per row, phases per quadrant, density)
SAMPLES = ((0, 17, 9, 1e15), (1, 33, 25, 4e15), (2, 65, 9, 1e16))


@pytest.fixture(scope="module")
def sweep_inputs(cuda_device):
    ext = workloads.orbit_diameter(SPEED, min(FIELDS))
    grids = {}
    for k, dim, ppq, dens in SAMPLES:
        grids[k] = Grid.from_seed((0 + 100) * (k + 1), L, ext, dens, R_IMP, 12)
    return ext, grids


def make_passes(ext, grids, grid_ids, fields=FIELDS):
    passes = []
    temps = [incoherent_temperature(t) for t in TEMPS]
    for k, dim, ppq, dens in SAMPLES:
        st = make_settings(TAU, ALPHA, True, SPEED, L, ext, dens, R_IMP, 12)
        for b in fields:
            for coherent in (True, False):
                passes.append(BatchPass(grid_ids[k], dim, ppq, coherent, L, grids[k].info().cell_size, b, st,
                                        list(temps)))
    return passes


def per_pass_reference(grids, passes, device):
    """sigma [n, T, 2] and metrics of every pass from the per-pass FP64 path
    (passes built with grid = sample index)."""
    out = np.zeros((len(passes), len(TEMPS), 2))
    mets = []
    sims = {}
    try:
        for n, p in enumerate(passes):
            key = (p.grid, p.coherent)
            if key not in sims:
                sims[key] = SimulationCUDA(p.positions_per_row, p.phi_steps, grids[p.grid].info(), device=device,
                                           precision=N.ES_PRECISION_FP64)
                sims[key].InitSample(grids[p.grid], p.settings, p.coherent)
            sm = SampleMetrics()
            sig = sims[key].ComputeSigmas(p.magnetic_field, p.temperatures, sample_metrics=sm)
            for t, s in enumerate(sig):
                out[n, t] = (s.xx, s.xy)
            mets.append(sm.iteration_metrics[-1])
    finally:
        for s in sims.values():
            s.close()
    return out, mets


def rel_err(a, b):
    return np.abs(a - b) / np.abs(b)


@pytest.fixture(scope="module")
def reference(sweep_inputs, cuda_device):
    ext, grids = sweep_inputs
    passes = make_passes(ext, grids, {k: k for k, *_rest in SAMPLES})
    return per_pass_reference(grids, passes, cuda_device)


def new_batch(grids, device, precision, chunk_iters=8, blocks_per_sm=4, mode=N.ES_BATCH_PERSISTENT):
    b = BatchSweep(device, chunk_iters=chunk_iters, blocks_per_sm=blocks_per_sm, precision=precision, mode=mode)
    ids = {k: b.add_grid(grids[k]) for k, *_rest in SAMPLES}
    return b, ids


@pytest.mark.parametrize("precision,rtol", [(N.ES_PRECISION_FP64, FP64_RTOL), (N.ES_PRECISION_SPLIT, SPLIT_RTOL)])
def test_batch_matches_per_pass(sweep_inputs, reference, cuda_device, precision, rtol):
    ext, grids = sweep_inputs
    ref_sigma, ref_mets = reference
    b, ids = new_batch(grids, cuda_device, precision)
    try:
        passes = make_passes(ext, grids, ids)
        b.set_passes(passes)
        out, mets = b.run()
        got = out[:, :len(TEMPS), :]
        err = rel_err(got, ref_sigma)
        assert float(err.max()) <= rtol, (precision, float(err.max()), np.unravel_index(err.argmax(), err.shape))
        for n, (m, r) in enumerate(zip(mets, ref_mets)):
            for k in METRIC_KEYS:
                assert m[k] == r[k], (precision, n, k, m[k], r[k])
        assert out[:, len(TEMPS):, :].max() == 0.0 and out[:, len(TEMPS):, :].min() == 0.0
    finally:
        b.close()


def test_batch_bit_reproducible_and_shape_independent(sweep_inputs, cuda_device):
    ext, grids = sweep_inputs
    b, ids = new_batch(grids, cuda_device, N.ES_PRECISION_SPLIT, chunk_iters=4, blocks_per_sm=4)
    try:
        b.set_passes(make_passes(ext, grids, ids))
        first, m1 = b.run()
        second, m2 = b.run()
        assert np.array_equal(first.view(np.int64), second.view(np.int64))
        assert m1 == m2
        b.set_tuning(blocks_per_sm=3)
        third, m3 = b.run()
        assert np.array_equal(first.view(np.int64), third.view(np.int64))
        assert m1 == m3
        # another work-item size regroups the FP64 partial sums: equal to rounding
        b.set_tuning(chunk_iters=32)
        fourth, m4 = b.run()
        assert float(rel_err(fourth[:, :3], first[:, :3]).max()) <= FP64_RTOL
        assert m1 == m4
    finally:
        b.close()


def test_batch_modes_agree(sweep_inputs, cuda_device):
    """The persistent fused kernel and the per-pass kernels (the default) sum in
    different orders: equal to rounding. Metrics are integers and equal. The
    removed mode numbers are rejected."""
    ext, grids = sweep_inputs
    outs = {}
    for mode in (N.ES_BATCH_PASS_KERNELS, N.ES_BATCH_PERSISTENT):
        b, ids = new_batch(grids, cuda_device, N.ES_PRECISION_SPLIT)
        try:
            b.set_tuning(mode=mode)
            b.set_passes(make_passes(ext, grids, ids))
            outs[mode] = b.run()
        finally:
            b.close()
    (k, mk), (p, mp) = outs[N.ES_BATCH_PASS_KERNELS], outs[N.ES_BATCH_PERSISTENT]
    assert float(rel_err(p[:, :3], k[:, :3]).max()) <= SPLIT_RTOL
    for a, c in zip(mk, mp):
        for key in ("cells_passed", "impurities_tested", "particles_inside_impurity", "particles_escaped",
                    "particles_at_bound"):
            assert a[key] == c[key], key
    b, _ = new_batch(grids, cuda_device, N.ES_PRECISION_SPLIT)
    try:
        for mode in (0, 1, 4):
            with pytest.raises(N.EsError):
                b.set_tuning(mode=mode)
    finally:
        b.close()


def test_batch_graph_replay_with_new_table(sweep_inputs, cuda_device):
    """The recorded graph is replayed with a rewritten instance table (same capacity
    and work-item count; the persistent kernel reads the table from device memory)."""
    ext, grids = sweep_inputs
    b, ids = new_batch(grids, cuda_device, N.ES_PRECISION_SPLIT)
    fresh, fids = new_batch(grids, cuda_device, N.ES_PRECISION_SPLIT)
    b.set_tuning(mode=N.ES_BATCH_PERSISTENT)
    fresh.set_tuning(mode=N.ES_BATCH_PERSISTENT)
    try:
        b.set_passes(make_passes(ext, grids, ids, fields=(1.5, 7.0)))
        b.run()
        launches = b.launch_count()
        b.set_passes(make_passes(ext, grids, ids, fields=(3.0, 33.0)))
        replayed, mr = b.run()
        assert b.launch_count() == launches + 1
        fresh.set_passes(make_passes(ext, grids, fids, fields=(3.0, 33.0)))
        direct, md = fresh.run()
        assert np.array_equal(replayed.view(np.int64), direct.view(np.int64))
        assert mr == md
    finally:
        b.close()
        fresh.close()


def test_batch_rejects_bad_instances(sweep_inputs, cuda_device):
    ext, grids = sweep_inputs
    b, ids = new_batch(grids, cuda_device, N.ES_PRECISION_SPLIT)
    try:
        good = make_passes(ext, grids, ids, fields=(7.0,))
        bad = [BatchPass(**{**good[1].__dict__, "grid": 99})]
        with pytest.raises(N.EsError, match="unknown grid"):
            b.set_passes(bad)
        many_t = [BatchPass(**{**good[1].__dict__, "temperatures": [1.0, 2.0, 3.0, 4.0, 5.0]})]
        with pytest.raises(N.EsError, match="distinct relaxation times"):
            b.set_passes(many_t)
        far = [BatchPass(**{**good[0].__dict__, "region_size": 1.0})]
        with pytest.raises(N.EsError, match="outside its grid"):
            b.set_passes(far)
        zero_t = [BatchPass(**{**good[1].__dict__, "temperatures": [0.0]})]
        with pytest.raises(N.EsError, match="needs T > 0"):
            b.set_passes(zero_t)
        # the batch is still usable
        b.set_passes(good)
        out, _ = b.run()
        assert np.isfinite(out).all()
    finally:
        b.close()


def test_autotuner_picks_from_measured_candidates_and_caches(tmp_path, cuda_device):
    """A small sweep: the tuner times every candidate on pilot passes, keeps a
    candidate per density class and one launch shape, and the second call
    answers from the cache without timing anything."""
    from elasticscattering_b200 import autotune
    wl = workloads.config2(n_samples=4, n_fields=4)
    wl.region_extends = workloads.orbit_diameter(SPEED, 8.0)
    wl.fields = [8.0, 16.0, 24.0, 40.0]
    for s in wl.samples:
        s.density = min(s.density, 3e15)
    cache = tmp_path / "tune.json"
    shapes = autotune.SHAPE_CANDIDATES[:2] + autotune.SHAPE_CANDIDATES[4:]
    r = autotune.tune_sweep(wl, device=cuda_device, n_classes=2, cache=cache, tcp_candidates=(6, 16),
                            shape_candidates=shapes)
    assert all(t in (6, 16) for t in r.tcp) and len(r.tcp) == 2
    assert r.shape in [dict(s) for s in shapes]
    cells = [t for t in r.trials if t["stage"] == "cell"]
    assert len(cells) == 2 * 2 and all(t["ms"] > 0 for t in r.trials)
    best = min((t for t in r.trials if t["stage"] == "shape"), key=lambda t: t["ms"])
    assert {k: best[k] for k in r.shape} == r.shape
    again = autotune.tune_sweep(wl, device=cuda_device, n_classes=2, cache=cache, tcp_candidates=(6, 16),
                                shape_candidates=shapes)
    assert again == r


@pytest.mark.parametrize("precision,rtol", [(N.ES_PRECISION_FP64, FP64_RTOL), (N.ES_PRECISION_SPLIT, SPLIT_RTOL)])
def test_batch_pass_kernels_mode(sweep_inputs, reference, cuda_device, precision, rtol):
    """ES_BATCH_PASS_KERNELS runs the single-pass path's kernels for each pass
    (lifetimes to device scratch, then the integration kernels): the same sigma
    as the per-pass FP64 path within the precision's bar, the same counters, and
    the same bits on a second replay."""
    ext, grids = sweep_inputs
    ref_sigma, ref_mets = reference
    b, ids = new_batch(grids, cuda_device, precision)
    try:
        b.set_tuning(mode=N.ES_BATCH_PASS_KERNELS)
        b.set_passes(make_passes(ext, grids, ids))
        out, mets = b.run()
        again, mets2 = b.run()
        got = out[:, :len(TEMPS), :]
        err = rel_err(got, ref_sigma)
        assert float(err.max()) <= rtol, (precision, float(err.max()), np.unravel_index(err.argmax(), err.shape))
        for n, (m, r) in enumerate(zip(mets, ref_mets)):
            for k in METRIC_KEYS:
                assert m[k] == r[k], (precision, n, k, m[k], r[k])
        assert np.array_equal(out.view(np.int64), again.view(np.int64)) and mets == mets2
        assert out[:, len(TEMPS):, :].max() == 0.0 and out[:, len(TEMPS):, :].min() == 0.0
    finally:
        b.close()


def test_split_exact_batch_equals_fp64_batch(sweep_inputs, cuda_device):
    """A batch in ES_PRECISION_SPLIT_EXACT (per-pass kernels: the split walk, FP64
    integration) returns the FP64 batch's sigma bit for bit and its counters;
    the persistent mode refuses the precision."""
    ext, grids = sweep_inputs
    outs, mets = {}, {}
    for prec in (N.ES_PRECISION_FP64, N.ES_PRECISION_SPLIT_EXACT):
        with BatchSweep(cuda_device, precision=prec, mode=N.ES_BATCH_PASS_KERNELS) as b:
            ids = {k: b.add_grid(g) for k, g in grids.items()}
            b.set_passes(make_passes(ext, grids, ids))
            outs[prec], mets[prec] = b.run()
    assert np.array_equal(outs[N.ES_PRECISION_FP64], outs[N.ES_PRECISION_SPLIT_EXACT])
    for x, y in zip(mets[N.ES_PRECISION_FP64], mets[N.ES_PRECISION_SPLIT_EXACT]):
        assert all(x[k] == y[k] for k in METRIC_KEYS)
    with BatchSweep(cuda_device, precision=N.ES_PRECISION_SPLIT, mode=N.ES_BATCH_PASS_KERNELS) as b:
        with pytest.raises(N.EsError):
            b.set_tuning(precision=N.ES_PRECISION_SPLIT_EXACT, mode=N.ES_BATCH_PERSISTENT)


def _long_walks(grid) -> bool:
    """The library's choice of the split-finish form for a pass on `grid`: the
    grid's straight-line mean free path through its disks, in cells, >= 0.5."""
    s = grid.GetSettings()
    per_cell = grid.GetTotalImpurityCount() / float(s.cells_per_row ** 2)
    return per_cell <= 0.0 or s.cell_size / (per_cell * 2.0 * s.impurity_radius) >= 0.5


def test_graph_kernel_count(sweep_inputs, cuda_device):
    """es_batch_graph_kernels counts the recorded graph's kernel nodes: per pass
    the orbit table, the split walk, the winners' FP64 finish on long-walk
    passes, the FP64 re-trace, integration and reduction (3 temperatures, one
    group); two for the persistent mode (its kernel and the re-trace)."""
    ext, grids = sweep_inputs
    b, ids = new_batch(grids, cuda_device, N.ES_PRECISION_SPLIT, mode=N.ES_BATCH_PASS_KERNELS)
    try:
        assert b.graph_kernels() == 0
        passes = make_passes(ext, grids, ids, fields=(1.5, 7.0))
        b.set_passes(passes)
        b.run()
        long_by_grid = {ids[k]: _long_walks(grids[k]) for k in grids}
        assert b.graph_kernels() == sum(6 if long_by_grid[p.grid] else 5 for p in passes)
        b.set_tuning(mode=N.ES_BATCH_PERSISTENT)
        b.run()
        assert b.graph_kernels() == 2
    finally:
        b.close()
