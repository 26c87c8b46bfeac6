"""Named workloads of the conductivity path, as concrete reference inputs.

Each workload is a set of reference `.config` values (src/SimulationConfiguration.h)
plus the field and temperature lists of its sweep. Conventions used to turn
the physical descriptions into reference inputs:

- phase samples N_phi -> phi_steps = the odd integer nearest N_phi/4 (the
  reference integrates each quarter separately, src/sim/Simulation.h:115-125);
- "padded by one orbit diameter" -> region_extends = 2 v m* / (e B_min);
- "cell size ~5e-8 m" -> the integer target_cell_population whose
  cells_per_row = round(sqrt(N_imp / tcp)) gives the nearest cell size;
- seed s -> start_seed s, so sample k uses Grid seed (s + 100) * (k + 1)
  (src/SimulationConfiguration.h:209-210);
- T = 0 cannot be expressed by the reference (its parser drops T <= 0,
  src/SimulationConfiguration.h:193-195, and tau_inc = hbar / (k_B T) diverges).
  The "T = 0" row is the coherent sigma at the configured tau plus the
  incoherent sigma at T_ZERO_STANDIN kelvin.
"""
from __future__ import annotations

from dataclasses import dataclass, field

# src/sim/es/constants.h:23-26
M0 = 9.10938188e-31
M_EFF = 5.0 * M0
E_CHARGE = 1.60217646e-19

T_ZERO_STANDIN = 1e-3  # kelvin


def orbit_diameter(speed: float, b_min: float) -> float:
    """2 r = 2 v m* / (e B) at the smallest field of the sweep."""
    return 2.0 * speed * M_EFF / (E_CHARGE * b_min)


@dataclass
class Workload:
    name: str
    dim: int                 # `dimension`: start positions per row (odd)
    phi_steps: int           # `phi_steps`: phases per quadrant (odd)
    region_size: float
    region_extends: float
    density: float
    impurity_radius: float
    target_cell_population: int
    fields: list = field(default_factory=list)
    temperatures: list = field(default_factory=list)
    start_seed: int = 0
    num_samples: int = 1
    particle_speed: float = 1.68e5
    alpha: float = 0.3
    tau: float = 1e-12
    clockwise: bool = True

    @property
    def orbits_per_pass(self) -> int:
        return self.dim * self.dim * 4 * self.phi_steps

    def seed(self, sample: int) -> int:
        return (self.start_seed + 100) * (sample + 1)

    def config_text(self) -> str:
        """The workload as a reference .config file."""
        temps = " ".join(repr(float(t)) for t in self.temperatures)
        lines = [
            f"num_samples {self.num_samples}", f"dimension {self.dim}", f"phi_steps {self.phi_steps}",
            f"temperatures {temps}",
        ]
        if len(self.fields) == 1:
            lines.append(f"magnetic_field {self.fields[0]!r}")
        else:
            lo, hi = self.fields[0], self.fields[-1]
            step = (hi - lo) / (len(self.fields) - 1)
            if any(abs(b - (lo + k * step)) > 1e-12 * max(abs(hi), 1.0) for k, b in enumerate(self.fields)):
                # src/SimulationConfiguration.h:150-176: one field, or min/max/n uniformly spaced
                raise ValueError("a .config file holds one magnetic field or a uniformly spaced range")
            lines += [f"magnetic_field_min {lo!r}", f"magnetic_field_max {hi!r}", f"magnetic_field_n {len(self.fields)}"]
        lines += [
            f"particle_speed {self.particle_speed!r}", f"clockwise {1 if self.clockwise else 0}",
            f"alpha {self.alpha!r}", f"tau {self.tau!r}", f"region_size {self.region_size!r}",
            f"region_extends {self.region_extends!r}", f"impurity_density {self.density!r}",
            f"impurity_radius {self.impurity_radius!r}", f"target_cell_population {self.target_cell_population}",
            f"start_seed {self.start_seed}",
        ]
        return "\n".join(lines) + "\n"


def config0() -> Workload:
    """Plain method, CPU-runnable: 65x65 positions x 101 phase samples, 1e15 m^-2, B = 20 T."""
    return Workload("config0-65x65x100-B20", dim=65, phi_steps=25, region_size=1e-6,
                    region_extends=orbit_diameter(1.68e5, 20.0), density=1e15, impurity_radius=2e-9,
                    target_cell_population=3, fields=[20.0], temperatures=[T_ZERO_STANDIN])


def config1() -> Workload:
    """Plain method at scale: 257x257 positions x 513 phase samples (34.08 M orbits per
    sector pass), 5e15 m^-2, B in {1, 5, 10, 20, 40} T, one sample."""
    return Workload("config1-257x257x516-5B", dim=257, phi_steps=129, region_size=1e-6,
                    region_extends=orbit_diameter(1.68e5, 1.0), density=5e15, impurity_radius=2e-9,
                    target_cell_population=12, fields=[1.0, 5.0, 10.0, 20.0, 40.0], temperatures=[T_ZERO_STANDIN])


def config3() -> Workload:
    """Precision stress: 1025x1025 positions x 1025 phases, 1e16 m^-2, r_i = 5e-9, B = 40 T."""
    return Workload("config3-1025x1025x1028-B40", dim=1025, phi_steps=257, region_size=1e-6,
                    region_extends=orbit_diameter(1.68e5, 40.0), density=1e16, impurity_radius=5e-9,
                    target_cell_population=25, fields=[40.0], temperatures=[T_ZERO_STANDIN])


@dataclass
class SweepSample:
    """One impurity sample of a batched sweep: its Grid seed, start grid and density."""
    index: int
    seed: int
    dim: int
    density: float


@dataclass
class BatchWorkload:
    """A sweep over samples x fields x temperatures with per-sample start grids and
    densities (both sectors per (sample, field), as SimulationRunner runs them,
    src/SimulationRunner.cpp:91-92)."""
    name: str
    samples: list
    fields: list
    temperatures: list
    phi_steps: int
    region_size: float
    region_extends: float
    impurity_radius: float
    target_cell_population: int
    draw_seed: int
    particle_speed: float = 1.68e5
    alpha: float = 0.3
    tau: float = 1e-12
    clockwise: bool = True

    @property
    def orbits(self) -> int:
        return sum(s.dim * s.dim for s in self.samples) * 4 * self.phi_steps * 2 * len(self.fields)

    @property
    def sigma_points(self) -> int:
        """One point = one (sample, field, temperature) with both sectors."""
        return len(self.samples) * len(self.fields) * len(self.temperatures)


def config2(n_samples: int = 64, n_fields: int = 32, dims=(129, 257, 513), phi_steps: int = 129,
            draw_seed: int = 12345, start_seed: int = 0) -> BatchWorkload:
    """Batched sweep: 64 samples (Grid seeds of start_seed 0, samples 0-63) x 32 fields
    uniformly spaced 1-40 T x T in {0, 10, 40} K. Per sample, the start grid is drawn from
    {129^2, 257^2, 513^2} and the density log-uniformly from 1e15-1e16 m^-2, with a
    fixed draw seed (12345) so that the instance set is reproducible."""
    import numpy as np
    rng = np.random.default_rng(draw_seed)
    dim_draw = rng.choice(np.asarray(dims), size=n_samples)
    dens_draw = 10.0 ** rng.uniform(15.0, 16.0, size=n_samples)
    samples = [SweepSample(k, (start_seed + 100) * (k + 1), int(dim_draw[k]), float(dens_draw[k]))
               for k in range(n_samples)]
    fields = [float(b) for b in np.linspace(1.0, 40.0, n_fields)]
    return BatchWorkload(f"config2-{n_samples}x{n_fields}x3", samples, fields, [0.0, 10.0, 40.0], phi_steps,
                         region_size=1e-6, region_extends=orbit_diameter(1.68e5, min(fields)),
                         impurity_radius=2e-9, target_cell_population=12, draw_seed=draw_seed)


def shard_samples(wl: BatchWorkload, rank: int, world: int, per_rank: int) -> BatchWorkload:
    """The samples one GPU of a multi-GPU sweep runs: rank r takes samples
    [r * per_rank, (r + 1) * per_rank) of the draw (weak scaling: every GPU runs
    `per_rank` samples; the passes share no data, so the only exchange is the
    gather of the sigma results)."""
    import copy
    if not 0 <= rank < world or per_rank < 1:
        raise ValueError("bad shard")
    if (rank + 1) * per_rank > len(wl.samples):
        raise ValueError(f"the draw holds {len(wl.samples)} samples; {world} x {per_rank} requested")
    out = copy.copy(wl)
    out.samples = wl.samples[rank * per_rank:(rank + 1) * per_rank]
    out.name = f"{wl.name.split('-')[0]}-{per_rank}x{len(wl.fields)}x{len(wl.temperatures)}"
    return out


def representative_slice(wl: BatchWorkload, k: int = 0) -> BatchWorkload:
    """Three samples of the draw, one per start grid (129^2, 257^2, 513^2), with
    every field and temperature: the draw picks each start grid with probability
    1/3, so the slice holds the orbits of three average samples. The samples are
    matched greedily so that the slice's estimated cost per orbit (sample_cost)
    is as close as possible to the whole draw's: slice 0 takes the best triple,
    slice 1 the best of the remaining samples, and so on, so slices k = 0, 1, ...
    are disjoint (the per-GPU work of a weak-scaling run) and each times like
    the sweep it stands for."""
    import copy
    import itertools
    dims = sorted({s.dim for s in wl.samples})
    by_dim = {d: [s for s in wl.samples if s.dim == d] for d in dims}
    cost = {s.index: sample_cost(wl, s) for s in wl.samples}
    per_pass = 4 * wl.phi_steps * 2 * len(wl.fields)
    target = sum(cost.values()) / (sum(s.dim * s.dim for s in wl.samples) * per_pass)
    used: set = set()
    picked = None
    for _ in range(k + 1):
        best, best_key = None, None
        for trio in itertools.product(*[[s for s in by_dim[d] if s.index not in used] for d in dims]):
            cpo = sum(cost[s.index] for s in trio) / (sum(s.dim * s.dim for s in trio) * per_pass)
            key = (abs(cpo - target), [s.index for s in trio])
            if best_key is None or key < best_key:
                best, best_key = trio, key
        if best is None:
            raise ValueError(f"the draw holds too few samples of each start grid for slice {k}")
        used |= {s.index for s in best}
        picked = list(best)
    out = copy.copy(wl)
    out.samples = picked
    out.name = f"{wl.name.split('-')[0]}-slice{k}-{len(picked)}x{len(wl.fields)}x{len(wl.temperatures)}"
    return out


def expected_cells(density: float, impurity_radius: float, magnetic_field: float, cell_size: float,
                   speed: float = 1.68e5) -> float:
    """Cell steps an orbit takes on average before its first impurity hit: the
    straight-line mean free path 1 / (2 r_i n), capped by the orbit's
    circumference 2 pi v m* / (e B), in cells, plus the start cell."""
    import math
    mfp = 1.0 / (2.0 * impurity_radius * density)
    circ = 2.0 * math.pi * speed * M_EFF / (E_CHARGE * magnetic_field)
    return 1.0 + min(mfp, circ) / cell_size


def sample_cost(wl: BatchWorkload, s: SweepSample) -> float:
    """Estimated cost of one sample's sweep: orbits x expected cell steps, summed
    over the fields and both sectors (the walk dominates every pass)."""
    import math
    n_imp = s.density * (wl.region_size + 2 * wl.region_extends) ** 2
    cpr = max(1, round(math.sqrt(n_imp / wl.target_cell_population)))
    cell = (wl.region_size + 2 * wl.region_extends) / cpr
    orbits = s.dim * s.dim * 4 * wl.phi_steps
    return sum(2 * orbits * expected_cells(s.density, wl.impurity_radius, b, cell, wl.particle_speed)
               for b in wl.fields)


def lpt_partition(costs: list, world: int) -> list:
    """Longest processing time first: items in decreasing cost (ties by index)
    go to the rank with the smallest load so far (ties to the lowest rank).
    Returns, per rank, the item indices in increasing order. Deterministic."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def lpt_shard(wl: BatchWorkload, rank: int, world: int) -> BatchWorkload:
    """The samples rank `rank` runs when the whole draw is split over `world`
    GPUs by LPT on sample_cost (strong scaling: the total work is fixed)."""
    import copy
    if not 0 <= rank < world:
        raise ValueError("bad shard")
    parts = lpt_partition([sample_cost(wl, s) for s in wl.samples], world)
    out = copy.copy(wl)
    out.samples = [wl.samples[i] for i in parts[rank]]
    out.name = f"{wl.name.split('-')[0]}-lpt{rank}of{world}-{len(out.samples)}x{len(wl.fields)}x{len(wl.temperatures)}"
    return out


def row_split(dim: int, rank: int, world: int) -> tuple:
    """Start rows [j0, j1) of one sector pass that rank `rank` of `world` GPUs
    computes when a single pass is split (the rows hold equal orbit counts)."""
    if not 0 <= rank < world or world > dim:
        raise ValueError("bad row split")
    return (rank * dim) // world, ((rank + 1) * dim) // world


WORKLOADS = {"config0": config0, "config1": config1, "config3": config3}
