"""The reference's own CPU build (oracle/_ref/libes_ref.so) run over many processes.

TEST INFRASTRUCTURE ONLY (the oracle of the full-size parity tests). The
reference is single-threaded (src/sim/SimulationCPU.cpp:112-135); a full
config-1 sector pass takes ~30 s on one core. Here the start-position rows of
each pass are split into disjoint ranges, each range runs the body of the
reference's SimulationCPU::ComputeLifetimes in its own process
(ref_sim_lifetimes_rows), and the results land in one file per pass, in the
reference's [j][i][q][p] order. The reference's DeriveTemperature
(src/sim/SimulationCPU.cpp:143-155) then turns each whole pass into sigma, one
process per (pass, temperature). Nothing here is a product path.

The pool uses the `spawn` start method, so it is safe to create after CUDA was
initialised in the parent.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import shutil
import tempfile
from dataclasses import dataclass, field

import numpy as np

METRIC_NAMES = ("cells_passed", "impurities_tested", "particles_inside_impurity", "particles_escaped",
                "particles_at_bound", "max_impurities_tested", "max_cells_passed")


@dataclass(frozen=True)
class PassSpec:
    """One sector pass: the Grid(seed, ...) it runs on (src/sim/Grid.cpp:28-46),
    the Simulation constructor and Settings values, the sector and the field."""
    seed: int
    region_size: float
    region_extends: float
    density: float
    impurity_radius: float
    target_cell_population: int
    dim: int
    phi_steps: int
    tau: float
    alpha: float
    clockwise: bool
    particle_speed: float
    coherent: bool
    field_b: float

    @property
    def per_row(self) -> int:
        return self.dim * 4 * self.phi_steps

    def grid_key(self):
        return (self.seed, self.region_size, self.region_extends, self.density, self.impurity_radius,
                self.target_cell_population)


def spec_of(w, seed: int, coherent: bool, field_b: float, dim: int | None = None, density: float | None = None,
            phi_steps: int | None = None) -> PassSpec:
    """A PassSpec from a workload (elasticscattering_b200.workloads)."""
    return PassSpec(seed, w.region_size, w.region_extends, w.density if density is None else density,
                    w.impurity_radius, w.target_cell_population, w.dim if dim is None else dim,
                    w.phi_steps if phi_steps is None else phi_steps, w.tau, w.alpha, bool(w.clockwise),
                    w.particle_speed, bool(coherent), float(field_b))


# ---- worker side -----------------------------------------------------------

_GRIDS: dict = {}


def _sim(spec: PassSpec):
    import oracle_lib as O
    lib = O.ref()
    g = _GRIDS.get(spec.grid_key())
    if g is None:
        for old in list(_GRIDS.values()):  # one grid per worker at a time (a few hundred MB at most)
            lib.ref_grid_free(old)
        _GRIDS.clear()
        g = lib.ref_grid_new_seed(spec.seed & 0xFFFFFFFF, spec.region_size, spec.region_extends, spec.density,
                                  spec.impurity_radius, spec.target_cell_population)
        _GRIDS[spec.grid_key()] = g
    sim = lib.ref_sim_new(g, spec.dim, spec.phi_steps, spec.tau, spec.alpha, int(spec.clockwise),
                          spec.particle_speed, spec.region_size, spec.region_extends)
    lib.ref_sim_init_sample(sim, int(spec.coherent))
    return lib, sim


def _rows_task(args):
    spec, j0, j1, path, first_row = args
    lib, sim = _sim(spec)
    out = np.zeros((j1 - j0) * spec.per_row)
    m = np.zeros(7, dtype=np.int32)
    lib.ref_sim_lifetimes_rows(sim, spec.field_b, j0, j1, out.ctypes.data, m.ctypes.data)
    lib.ref_sim_free(sim)
    with open(path, "r+b") as f:
        f.seek((j0 - first_row) * spec.per_row * 8)
        f.write(out.tobytes())
    return path, [int(v) for v in m]


def _derive_task(args):
    spec, path, temperature = args
    lib, sim = _sim(spec)
    raw = np.fromfile(path, dtype=np.float64)
    out = np.zeros(2)
    lib.ref_sim_derive(sim, spec.field_b, float(temperature), raw.ctypes.data, out.ctypes.data)
    lib.ref_sim_free(sim)
    return path, float(temperature), (float(out[0]), float(out[1]))


# ---- parent side -----------------------------------------------------------

@dataclass
class PassResult:
    spec: PassSpec
    rows: tuple
    path: str
    metrics: dict = field(default_factory=dict)
    sigmas: dict = field(default_factory=dict)  # temperature -> (xx, xy)

    def lifetimes(self) -> np.ndarray:
        return np.fromfile(self.path, dtype=np.float64)


class RefPool:
    """A spawn pool of processes running the reference's CPU build."""

    def __init__(self, procs: int | None = None):
        self.procs = procs or min(64, len(os.sched_getaffinity(0)))
        self._pool = mp.get_context("spawn").Pool(self.procs)
        self._dir = tempfile.mkdtemp(prefix="es_refpool_")
        self._files = 0

    def close(self) -> None:
        self._pool.terminate()
        self._pool.join()
        shutil.rmtree(self._dir, ignore_errors=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, passes, temperatures=(), rows=None, rows_per_task: int | None = None) -> list[PassResult]:
        """Lifetimes of every pass over start rows [rows[0], rows[1]) (default:
        all rows), and -- for passes over all rows -- the reference's sigma at
        each temperature. Returns one PassResult per pass, in order."""
        results, tasks = [], []
        for k, spec in enumerate(passes):
            j0, j1 = rows if rows else (0, spec.dim)
            path = os.path.join(self._dir, f"pass{self._files}.f64")
            self._files += 1
            with open(path, "wb") as f:
                f.truncate((j1 - j0) * spec.per_row * 8)
            res = PassResult(spec, (j0, j1), path, {n: 0 for n in METRIC_NAMES})
            results.append(res)
            step = rows_per_task or max(1, (j1 - j0) * len(passes) // (6 * self.procs))
            for a in range(j0, j1, step):
                tasks.append((spec, a, min(j1, a + step), path, j0))
        by_path = {r.path: r for r in results}
        for path, m in self._pool.imap_unordered(_rows_task, tasks):
            r = by_path[path]
            for n, v in zip(METRIC_NAMES, m):
                r.metrics[n] = max(r.metrics[n], v) if n.startswith("max_") else r.metrics[n] + v
        full = [r for r in results if r.rows == (0, r.spec.dim)]
        dtasks = [(r.spec, r.path, T) for r in full for T in temperatures]
        for path, T, sig in self._pool.imap_unordered(_derive_task, dtasks):
            by_path[path].sigmas[T] = sig
        return results

    def discard(self, results) -> None:
        for r in results:
            try:
                os.remove(r.path)
            except OSError:
                pass
