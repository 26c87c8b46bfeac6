"""Autotuner for batched sweeps: impurity-cell size and launch shape.

No reference counterpart: the reference fixes its cell size through the
`target_cell_population` config value (cells per row = round(sqrt(N / tcp)),
src/sim/Grid.cpp:40) and its OpenCL launch shape in code
(src/sim/SimulationCL.cpp:412-431). The batched path leaves both to this tuner:

1. Pilot passes stand in for the sweep: per density class of the workload one
   impurity sample at the class's geometric-mean density, on a reduced start
   grid (the cost of an orbit depends on density, radius and field, not on
   how many start positions there are), at the sweep's smallest, middle and
   largest field, both sectors, all of its temperatures.
2. Cell size: for every candidate `target_cell_population`, the pilot grids
   are rebuilt and run with the default launch shape; each density class keeps
   the fastest.
3. Launch shape: with those grids, every (mode, blocks per SM, work-item size)
   candidate is timed; the fastest wins.

Every timing is the minimum over repeats of a CUDA-event-timed graph replay.
Results are cached as JSON, keyed by device and workload signature, so a sweep
pays for tuning once.

The cell size changes the grid (and, through GridInformation::cell_size, the
start-position offset, src/sim/Simulation.h:142-143): a tuned sweep is compared
with plain FP64 on the same tuned grids.
"""
from __future__ import annotations

import json
import math
import os
import time
from dataclasses import asdict, dataclass, field
from pathlib import Path

from . import _native as N
from .batch import BatchPass, BatchSweep, incoherent_temperature
from .simulation import Grid, make_settings

TCP_CANDIDATES = (4, 8, 12, 20, 32)
SHAPE_CANDIDATES = (
    {"mode": N.ES_BATCH_PERSISTENT, "blocks_per_sm": 4, "chunk_iters": 16},
    {"mode": N.ES_BATCH_PERSISTENT, "blocks_per_sm": 4, "chunk_iters": 32},
    {"mode": N.ES_BATCH_PERSISTENT, "blocks_per_sm": 4, "chunk_iters": 64},
    {"mode": N.ES_BATCH_PERSISTENT, "blocks_per_sm": 3, "chunk_iters": 32},
    {"mode": N.ES_BATCH_PASS_KERNELS, "blocks_per_sm": 4, "chunk_iters": 32},
)
PILOT_DIM = 65
TUNER_VERSION = 3


def default_cache() -> Path:
    base = os.environ.get("ES_B200_TUNE_CACHE")
    if base:
        return Path(base)
    return Path.home() / ".cache" / "elasticscattering_b200" / "tuning.json"


@dataclass
class TuneResult:
    key: str
    density_edges: list          # class k covers [edges[k], edges[k+1])
    tcp: list                    # chosen target_cell_population per class
    shape: dict                  # es_batch_tuning fields (mode, blocks_per_sm, chunk_iters)
    pilot_orbits: int = 0
    seconds: float = 0.0
    trials: list = field(default_factory=list)

    def tcp_for(self, density: float) -> int:
        for k in range(len(self.tcp)):
            if density < self.density_edges[k + 1] or k == len(self.tcp) - 1:
                return int(self.tcp[k])
        return int(self.tcp[-1])


def _device_name(device: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return f"cuda:{device}"


def signature(wl, n_classes: int) -> str:
    dens = [s.density for s in wl.samples]
    return (f"v{TUNER_VERSION}|ppq{wl.phi_steps}|ri{wl.impurity_radius:.3g}|ext{wl.region_extends:.4g}"
            f"|L{wl.region_size:.3g}|B{min(wl.fields):.3g}-{max(wl.fields):.3g}x{len(wl.fields)}"
            f"|T{len(wl.temperatures)}|n{min(dens):.3g}-{max(dens):.3g}x{n_classes}")


def _pilot_passes(wl, grid_ids: dict, cell_sizes: dict, densities: list) -> list:
    fields = sorted(wl.fields)
    pick = sorted({fields[0], fields[len(fields) // 2], fields[-1]})
    temps = [incoherent_temperature(t) for t in wl.temperatures]
    out = []
    for k, dens in enumerate(densities):
        if k not in grid_ids:
            continue
        st = make_settings(wl.tau, wl.alpha, wl.clockwise, wl.particle_speed, wl.region_size, wl.region_extends,
                           dens, wl.impurity_radius, wl.target_cell_population)
        for b in pick:
            for coherent in (True, False):
                out.append(BatchPass(grid_ids[k], PILOT_DIM, wl.phi_steps, coherent, wl.region_size, cell_sizes[k],
                                     float(b), st, list(temps)))
    return out


def _time_batch(bs: BatchSweep, repeats: int = 2) -> float:
    import torch
    stream = torch.cuda.ExternalStream(bs.stream_handle())
    bs.run(with_metrics=False)  # records the graph, warms up
    best = math.inf
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bs.enqueue()
        e1.record(stream)
        bs.collect(with_metrics=False)
        best = min(best, e0.elapsed_time(e1))
    return best


def tune_sweep(wl, device: int = 0, n_classes: int = 3, cache: Path | None = None, force: bool = False,
               tcp_candidates=TCP_CANDIDATES, shape_candidates=SHAPE_CANDIDATES) -> TuneResult:
    """Cell sizes per density class and the launch shape for a BatchWorkload."""
    cache = default_cache() if cache is None else Path(cache)
    key = f"{_device_name(device)}|{signature(wl, n_classes)}"
    store = {}
    if cache.exists():
        try:
            store = json.loads(cache.read_text())
        except (OSError, json.JSONDecodeError):
            store = {}
    if not force and key in store:
        return TuneResult(**store[key])

    t_start = time.time()
    dens = sorted(s.density for s in wl.samples)
    lo, hi = math.log(dens[0]), math.log(dens[-1]) + 1e-12
    edges = [math.exp(lo + (hi - lo) * k / n_classes) for k in range(n_classes + 1)]
    centres = [math.exp(0.5 * (math.log(edges[k]) + math.log(edges[k + 1]))) for k in range(n_classes)]
    seeds = [wl.samples[0].seed + 7919 * k for k in range(n_classes)]
    trials = []

    def run(grids_by_class, shape) -> tuple[float, int]:
        with BatchSweep(device, precision=N.ES_PRECISION_SPLIT, **shape) as bs:
            ids = {k: bs.add_grid(g) for k, g in grids_by_class.items()}
            cells = {k: g.info().cell_size for k, g in grids_by_class.items()}
            bs.set_passes(_pilot_passes(wl, ids, cells, centres))
            return _time_batch(bs), bs.total_orbits

    # 1. cell size per density class, default launch shape
    base_shape = dict(shape_candidates[min(1, len(shape_candidates) - 1)])
    best_tcp = [None] * n_classes
    best_ms = [math.inf] * n_classes
    pilot_orbits = 0
    for tcp in tcp_candidates:
        for k in range(n_classes):
            g = Grid.from_seed(seeds[k], wl.region_size, wl.region_extends, centres[k], wl.impurity_radius, tcp)
            ms, orbits = run({k: g}, base_shape)
            trials.append({"stage": "cell", "class": k, "tcp": tcp, "ms": ms, "orbits": orbits})
            pilot_orbits = max(pilot_orbits, orbits)
            if ms < best_ms[k]:
                best_ms[k], best_tcp[k] = ms, tcp

    # 2. launch shape on the chosen grids
    grids = {k: Grid.from_seed(seeds[k], wl.region_size, wl.region_extends, centres[k], wl.impurity_radius,
                               best_tcp[k]) for k in range(n_classes)}
    best_shape, best = base_shape, math.inf
    for shape in shape_candidates:
        ms, orbits = run(grids, dict(shape))
        trials.append({"stage": "shape", **shape, "ms": ms, "orbits": orbits})
        if ms < best:
            best, best_shape = ms, dict(shape)

    res = TuneResult(key=key, density_edges=edges, tcp=[int(x) for x in best_tcp], shape=best_shape,
                     pilot_orbits=pilot_orbits, seconds=time.time() - t_start, trials=trials)
    store[key] = asdict(res)
    try:
        cache.parent.mkdir(parents=True, exist_ok=True)
        tmp = cache.with_suffix(f".{os.getpid()}.tmp")  # ranks of a multi-GPU run tune at once
        tmp.write_text(json.dumps(store, indent=1))
        tmp.replace(cache)
    except OSError:
        pass
    return res
