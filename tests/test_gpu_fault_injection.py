"""Host-side fault injection (es_fault_inject) through every error path of a
sector pass, the no-alloc entry point, a batched sweep and a GPU grid build.

For each kind of operation -- device or pinned allocation, copy, kernel launch --
a scenario runs once with injection disarmed, which counts its operations of
that kind, then once per operation with exactly that one failing. Each time
exactly one call must fail, with ES_ERR_OOM (allocation) or ES_ERR_LAUNCH (copy,
launch); repeating that call with injection disarmed must succeed on the same
objects; and everything the scenario returns (sigma, metrics, lifetimes, maps)
must equal the undisturbed run bit for bit.

The failures are made on the host: an injected allocation is never made, and an
injected copy or launch failure is reported after the real operation completed,
so no device fault is provoked. The reference has no counterpart: every error
there prints and exits (src/utils/ErrorMacros.h:22-38).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from elasticscattering_b200 import DeviceGrid, Grid, SimulationCUDA, make_settings, workloads
from elasticscattering_b200 import _native as N
from elasticscattering_b200.batch import BatchPass, BatchSweep
from elasticscattering_b200.simulation import SampleMetrics

pytestmark = pytest.mark.gpu

SPEED, ALPHA, TAU, L, R_IMP, DENSITY = 1.68e5, 0.3, 1e-12, 1e-6, 2e-9, 4e15
EXT = workloads.orbit_diameter(SPEED, 5.0)
DIM, PPQ = 17, 9
TEMPS = [1.0, 10.0, 40.0]
KINDS = {"alloc": N.ES_ERR_OOM, "copy": N.ES_ERR_LAUNCH, "launch": N.ES_ERR_LAUNCH}


def _settings():
    return make_settings(TAU, ALPHA, True, SPEED, L, EXT, DENSITY, R_IMP, 12)


def _grid(k=0):
    return Grid.from_seed(100 * (k + 1), L, EXT, DENSITY, R_IMP, 12)


def _metrics(sm):
    m = sm.iteration_metrics[-1]
    return [m[k] for k in sorted(m)]


def _sigmas(sig):
    return [v for s in sig for v in (s.xx, s.xy)]


def steps_pass():
    """A split-precision context: create, grid + sector, two fields,
    per-position maps, a lifetime read, the average lifetime."""
    grid, st = _grid(), _settings()

    def create(s):
        s["sim"] = SimulationCUDA(DIM, PPQ, grid.info(), precision=N.ES_PRECISION_SPLIT)

    def init(s):
        s["sim"].InitSample(grid, st, False)

    def field(b):
        def run(s):
            sm = SampleMetrics()
            sig = s["sim"].ComputeSigmas(b, TEMPS, sample_metrics=sm)
            return _sigmas(sig) + _metrics(sm)
        return run

    def images(s):
        its = s["sim"].ComputeSigmasWithImages(40.0, TEMPS)
        return np.concatenate([np.concatenate([it.particle_lifetimes, it.xx_buffer, it.xy_buffer, [it.result.xx, it.result.xy]])
                               for it in its])

    def lifetimes(s):
        return s["sim"].ReadLifetimes(5, 300)

    def average(s):
        v = C.c_double()
        s["sim"]._check(N.cuda_lib().es_average_lifetime(s["sim"].ctx, C.byref(v)))
        return [v.value]

    return [("create", create), ("init", init), ("field 20 T", field(20.0)), ("field 7 T", field(7.0)),
            ("images", images), ("read lifetimes", lifetimes), ("average", average)]


def steps_fp64_noalloc():
    """A plain FP64 context, its lifetimes handed to the no-alloc entry point."""
    import torch

    grid, st = _grid(1), _settings()

    def create(s):
        s["sim"] = SimulationCUDA(DIM, PPQ, grid.info(), precision=N.ES_PRECISION_FP64)

    def init(s):
        s["sim"].InitSample(grid, st, True)

    def lifetimes(s):
        lt, m = s["sim"].ComputeLifetimes(10.0)
        s["d_lt"] = torch.from_numpy(lt).to("cuda:0")
        torch.cuda.synchronize()
        return np.concatenate([lt, [m[k] for k in sorted(m)]])

    def noalloc(s):
        temps = np.ascontiguousarray(TEMPS, dtype=np.float64)
        d_out = torch.full((2 * len(temps),), float("nan"), dtype=torch.float64, device="cuda:0")
        status = N.cuda_lib().es_derive_temperatures_noalloc(C.c_void_p(s["d_lt"].data_ptr()), DIM, PPQ, C.byref(st),
                                                             1, 10.0, temps.ctypes.data, len(temps),
                                                             C.c_void_p(d_out.data_ptr()), None)
        torch.cuda.synchronize()
        N.check(status, None)
        return d_out.cpu().numpy()

    return [("create", create), ("init", init), ("lifetimes", lifetimes), ("noalloc", noalloc)]


def steps_batch():
    """A batched sweep over a host grid and a GPU-built grid: the per-pass
    kernels mode twice (the second replay reuses the graph), then the
    persistent mode."""
    st = _settings()
    host_grid = _grid(2)

    def create(s):
        s["b"] = BatchSweep(precision=N.ES_PRECISION_SPLIT, mode=N.ES_BATCH_PASS_KERNELS)

    def dgrid(s):
        s["dg"] = DeviceGrid.from_seed(300, L, EXT, DENSITY, R_IMP, 12)

    def add(which):
        def run(s):
            g = host_grid if which == "host" else s["dg"]
            s.setdefault("ids", {})[which] = s["b"].add_grid(g)
            s.setdefault("cells", {})[which] = g.info().cell_size
        return run

    def passes(s):
        ps = [BatchPass(s["ids"][w], DIM, PPQ, coh, L, s["cells"][w], b, st, list(TEMPS))
              for w in ("host", "device") for b in (7.0, 30.0) for coh in (True, False)]
        s["b"].set_passes(ps)

    def run(s):
        out, mets = s["b"].run()
        return np.concatenate([out.ravel(), [m[k] for m in mets for k in sorted(m)]])

    def persistent(s):
        s["b"].set_tuning(mode=N.ES_BATCH_PERSISTENT)
        return run(s)

    return [("create", create), ("device grid", dgrid), ("add host grid", add("host")),
            ("add device grid", add("device")), ("instances", passes), ("run", run), ("replay", run),
            ("persistent", persistent)]


def steps_dgrid():
    """A GPU grid build and its download."""

    def build(s):
        s["dg"] = DeviceGrid.from_seed(77, L, EXT, 1e16, R_IMP, 12)

    def download(s):
        return np.concatenate([s["dg"].GetImpurities().ravel(), s["dg"].GetIndex().astype(np.float64)])

    return [("build", build), ("download", download)]


SCENARIOS = {"pass": steps_pass, "fp64_noalloc": steps_fp64_noalloc, "batch": steps_batch, "dgrid": steps_dgrid}


def run_scenario(steps):
    """Runs the steps in order; a step that raises EsError is repeated once with
    injection disarmed. Returns everything the steps returned, the failures, and
    the operation counts at the end (since the last arming or disarming)."""
    state, out, failures = {}, [], []
    try:
        for name, fn in steps:
            try:
                r = fn(state)
            except N.EsError as e:
                failures.append((name, e.status, str(e)))
                N.fault_inject(None)
                r = fn(state)
            if r is not None:
                out.append(np.asarray(r, dtype=np.float64).ravel())
        counts = N.fault_counts()
    finally:
        N.fault_inject(None)
        for key in ("b", "sim", "dg"):
            if key in state:
                state[key].close()
    return np.concatenate(out), failures, counts


@pytest.mark.parametrize("kind", sorted(KINDS))
@pytest.mark.parametrize("scenario", sorted(SCENARIOS))
def test_every_failure_point_is_reported_and_recoverable(cuda_device, scenario, kind):
    N.fault_inject("")  # disarmed, counters at zero
    ref, failures, counts = run_scenario(SCENARIOS[scenario]())
    assert not failures
    n_ops = counts[kind]
    assert n_ops >= 1, (scenario, kind)
    for k in range(1, n_ops + 1):
        N.fault_inject(f"{kind}:{k}")
        got, failures, _ = run_scenario(SCENARIOS[scenario]())
        assert len(failures) == 1, (scenario, kind, k, failures)
        assert failures[0][1] == KINDS[kind], (scenario, kind, k, failures)
        assert np.array_equal(got, ref, equal_nan=True), (scenario, kind, k, failures[0][0])


def test_repeating_failures_and_counts(cuda_device):
    """"launch:N+" fails every launch from the N-th on; the counts say how many
    operations ran and failed; disarming restores normal operation."""
    grid, st = _grid(), _settings()
    with SimulationCUDA(DIM, PPQ, grid.info(), precision=N.ES_PRECISION_SPLIT) as sim:
        sim.InitSample(grid, st, False)
        ref = sim.ComputeSigmas(20.0, TEMPS)
        N.fault_inject("launch:1+")
        for _ in range(3):
            with pytest.raises(N.EsError) as e:
                sim.ComputeSigmas(20.0, TEMPS)
            assert e.value.status == N.ES_ERR_LAUNCH
        c = N.fault_counts()
        assert c["launch"] == 3 and c["failed"] == 3
        N.fault_inject(None)
        assert _sigmas(sim.ComputeSigmas(20.0, TEMPS)) == _sigmas(ref)
