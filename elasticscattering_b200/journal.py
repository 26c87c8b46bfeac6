"""The per-pass results journal of a .config sweep (`journal <path>`; the
writer is host/journal.cpp): one JSON object per finished (sample, sector,
field) pass with its sigma at every temperature and its metrics. A sweep that
stopped part way resumes from it; this module reads it, for instance to look
at the passes a partial sweep has finished.

No reference counterpart: the reference has no resume
(src/SimulationRunner.cpp:88-98).
"""
from __future__ import annotations

import json
import struct

FNV_OFFSET = 1469598103934665603
FNV_PRIME = 1099511628211
TAG = b"es-journal-1\0"


def _fnv(data: bytes, h: int = FNV_OFFSET) -> int:
    for c in data:
        h = ((h ^ c) * FNV_PRIME) & 0xFFFFFFFFFFFFFFFF
    return h


def run_key(cfg: dict) -> int:
    """The run key of a parsed config (the JSON of es_config_describe): FNV-1a
    over the inputs that decide a pass's sigma, in host/journal.cpp's order --
    start grid, phases, precision, per-pass or batched mode, the Settings
    fields and the temperatures."""
    i = lambda v: struct.pack("<q", int(v))  # noqa: E731
    d = lambda v: struct.pack("<d", float(v))  # noqa: E731
    data = (TAG + i(cfg["dimension"]) + i(cfg["phi_steps"]) + i(cfg["precision"]) + i(cfg["batched"])
            + d(cfg["tau"]) + d(cfg["alpha"])
            + i(cfg["clockwise"]) + d(cfg["particle_speed"]) + d(cfg["region_size"]) + d(cfg["region_extends"])
            + d(cfg["impurity_density"]) + d(cfg["impurity_radius"]) + i(cfg["target_cell_population"])
            + i(len(cfg["temperatures"])) + b"".join(d(t) for t in cfg["temperatures"]))
    return _fnv(data)


def read(path, key: int | None = None) -> list[dict]:
    """The complete entries of the journal at `path` (of run `key` only, if
    given), in file order; torn or foreign lines are skipped."""
    out = []
    with open(path, encoding="utf-8") as f:
        for line in f:
            try:
                e = json.loads(line)
            except json.JSONDecodeError:
                continue
            if not isinstance(e, dict) or e.get("journal") != 1:
                continue
            if key is not None and e.get("run") != f"{key:016x}":
                continue
            out.append(e)
    return out


def format_entry(key: int, sample: int, seed: int, coherent: bool, field: float, sigma, metrics: dict,
                 real_particles: int, avg_particle_lifetime: float = 0.0, time_lifetimes: float = 0.0,
                 time_temperatures: float = 0.0) -> str:
    """One journal line (without the newline) in the writer's layout; sigma is
    [(xx, xy)] per temperature, metrics the ten es_metrics counters."""
    names = ("cells_passed", "impurities_tested", "particles_inside_impurity", "particles_escaped",
             "particles_at_bound", "max_impurities_tested", "max_cells_passed", "crossings_tested",
             "start_cell_tests", "retraced_fp64")
    g = lambda x: repr(float(x))  # noqa: E731  (shortest round-trip form)
    sig = ",".join(f"[{g(xx)},{g(xy)}]" for xx, xy in sigma)
    met = ",".join(f'"{n}":{int(metrics.get(n, 0))}' for n in names)
    return (f'{{"journal":1,"run":"{key:016x}","sample":{sample},"seed":{seed},"coherent":{1 if coherent else 0},'
            f'"field":{g(field)},"sigma":[{sig}],"metrics":{{{met}}},"real_particles":{int(real_particles)},'
            f'"avg_particle_lifetime":{g(avg_particle_lifetime)},"time_lifetimes":{g(time_lifetimes)},'
            f'"time_temperatures":{g(time_temperatures)}}}')
