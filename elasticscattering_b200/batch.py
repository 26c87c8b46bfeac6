"""Batched sweeps: many (sample, field, sector) passes in one graph replay.

The reference runs a sweep as nested loops (SimulationRunner::RunSample,
src/SimulationRunner.cpp:86-151): per sample one Grid, per field and sector one
Simulation::ComputeSigmas call. `BatchSweep` takes the whole list of those calls
at once and runs them through the es_batch_* C ABI (include/es_cuda.h),
recorded once as a CUDA graph and replayed. The default mode
(ES_BATCH_PASS_KERNELS) runs the single-pass kernels for each pass in turn;
ES_BATCH_PERSISTENT fuses stages (b) and (c) into one persistent lifetime kernel
over all passes (faster for sweeps of many small passes). Each pass returns what
ComputeSigmas returns for it (one Sigma per temperature) plus its metrics.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .simulation import DeviceGrid, Grid, Sigma


@dataclass
class BatchPass:
    """One ComputeSigmas call: grid (index into BatchSweep.add_grid), start grid,
    phases, field, sector and temperatures."""
    grid: int
    positions_per_row: int
    phi_steps: int
    coherent: bool
    region_size: float
    grid_cell_size: float
    magnetic_field: float
    settings: N.Settings
    temperatures: list = field(default_factory=list)

    @property
    def n_orbits(self) -> int:
        return self.positions_per_row ** 2 * 4 * self.phi_steps

    def to_c(self) -> N.BatchInstance:
        if not 1 <= len(self.temperatures) <= N.ES_BATCH_MAX_T:
            raise ValueError(f"1..{N.ES_BATCH_MAX_T} temperatures per pass")
        t = (C.c_double * N.ES_BATCH_MAX_T)(*[float(x) for x in self.temperatures])
        return N.BatchInstance(int(self.grid), int(self.positions_per_row), int(self.phi_steps),
                               1 if self.coherent else 0, float(self.region_size), float(self.grid_cell_size),
                               float(self.magnetic_field), self.settings, len(self.temperatures), t)


def incoherent_temperature(t: float) -> float:
    """The reference cannot take T <= 0 (src/SimulationConfiguration.h:193-195); a
    T = 0 row uses the T_ZERO_STANDIN temperature for the incoherent sector."""
    from .workloads import T_ZERO_STANDIN
    return float(t) if t > 0 else T_ZERO_STANDIN


def sweep_passes(wl, grid_ids: list, grid_cell_sizes: list, samples=None, fields=None) -> list:
    """The BatchPass list of a BatchWorkload: per sample, per field, coherent then
    incoherent (src/SimulationRunner.cpp:91-92), each with the full temperature list."""
    from .simulation import make_settings
    samples = wl.samples if samples is None else samples
    fields = wl.fields if fields is None else fields
    temps = [incoherent_temperature(t) for t in wl.temperatures]
    out = []
    for s in samples:
        st = make_settings(wl.tau, wl.alpha, wl.clockwise, wl.particle_speed, wl.region_size, wl.region_extends,
                           s.density, wl.impurity_radius, wl.target_cell_population)
        for b in fields:
            for coherent in (True, False):
                out.append(BatchPass(grid_ids[s.index], s.dim, wl.phi_steps, coherent, wl.region_size,
                                     grid_cell_sizes[s.index], float(b), st, list(temps)))
    return out


class BatchSweep:
    """Owner of one es_batch (device buffers, stream, recorded graph)."""

    def __init__(self, device: int = 0, chunk_iters: int = 32, blocks_per_sm: int = 4,
                 precision: int = N.ES_PRECISION_SPLIT, mode: int = N.ES_BATCH_PASS_KERNELS):
        lib = N.cuda_lib()
        h = C.c_void_p()
        st = lib.es_batch_create(int(device), C.byref(h))
        if st != N.ES_OK:
            N.check(st, None)
        self._b = h
        self.passes: list[BatchPass] = []
        self.set_tuning(chunk_iters=chunk_iters, blocks_per_sm=blocks_per_sm, precision=precision,
                        mode=mode)

    def close(self) -> None:
        if getattr(self, "_b", None) and self._b.value:
            N.cuda_lib().es_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library handles may already be gone
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int) -> None:
        N.check_batch(st, self._b)

    def get_tuning(self) -> dict:
        t = N.BatchTuning()
        self._check(N.cuda_lib().es_batch_get_tuning(self._b, C.byref(t)))
        return {name: int(getattr(t, name)) for name, _ in N.BatchTuning._fields_}

    def set_tuning(self, **fields) -> None:
        cur = self.get_tuning()
        cur.update(fields)
        t = N.BatchTuning(*[int(cur[name]) for name, _ in N.BatchTuning._fields_])
        self._check(N.cuda_lib().es_batch_set_tuning(self._b, C.byref(t)))
        self._tuned = True

    def add_grid(self, grid) -> int:
        """Copies a Grid (host) or DeviceGrid to the batch's device memory; returns
        its index for BatchPass.grid."""
        out = C.c_int32()
        if isinstance(grid, DeviceGrid):
            self._check(N.cuda_lib().es_batch_add_dgrid(self._b, grid.handle, C.byref(out)))
            return int(out.value)
        # the host Grid's own arrays, read in place by the library
        xy, n, idx = grid.arrays()
        s = grid.GetSettings()
        self._check(N.cuda_lib().es_batch_add_grid(self._b, xy, n, idx, C.byref(s), C.byref(out)))
        return int(out.value)

    def clear(self) -> None:
        self._check(N.cuda_lib().es_batch_clear(self._b))
        self.passes = []

    def set_passes(self, passes: list[BatchPass]) -> None:
        arr = (N.BatchInstance * len(passes))(*[p.to_c() for p in passes])
        self._check(N.cuda_lib().es_batch_set_instances(self._b, arr, len(passes)))
        self.passes = list(passes)

    def enqueue(self) -> None:
        self._check(N.cuda_lib().es_batch_enqueue(self._b))

    def collect(self, with_metrics: bool = True):
        """Waits for the last enqueue; returns (sigma [n, ES_BATCH_MAX_T, 2], metrics list)."""
        n = len(self.passes)
        out = np.zeros((n, N.ES_BATCH_MAX_T, 2))
        mets = (N.Metrics * n)() if with_metrics else None
        self._check(N.cuda_lib().es_batch_collect(self._b, out.ctypes.data, mets))
        return out, ([m.as_dict() for m in mets] if with_metrics else None)

    def run(self, with_metrics: bool = True):
        self.enqueue()
        return self.collect(with_metrics)

    def sigmas(self, out: np.ndarray) -> list[list[Sigma]]:
        """Per pass, one Sigma per temperature (ComputeSigmas' return value)."""
        return [[Sigma(float(out[k, t, 0]), float(out[k, t, 1])) for t in range(len(p.temperatures))]
                for k, p in enumerate(self.passes)]

    @property
    def total_orbits(self) -> int:
        return int(N.cuda_lib().es_batch_total_orbits(self._b))

    def stream_handle(self) -> int:
        return int(N.cuda_lib().es_batch_stream(self._b) or 0)

    def launch_count(self) -> int:
        return int(N.cuda_lib().es_batch_launch_count(self._b))

    def graph_kernels(self) -> int:
        """Kernels one replay of the recorded graph launches."""
        return int(N.cuda_lib().es_batch_graph_kernels(self._b))


def finish_results(coherent: np.ndarray, incoherent: np.ndarray) -> dict:
    """SimulationRunner::FinishResults (src/SimulationRunner.cpp:153-198) on the
    per-sample sigmas of a sweep: `coherent` and `incoherent` are
    [sample][field][temperature][xx, xy]. Returns the sample means of each sector
    and delta_xx = std(sigma_xx_coh + sigma_xx_inc) / mean per (field,
    temperature), summed over the samples in sample order as the reference does,
    so the result does not depend on which GPU computed which sample."""
    coh = np.asarray(coherent, dtype=np.float64)
    inc = np.asarray(incoherent, dtype=np.float64)
    S = coh.shape[0]
    c_sum = np.zeros(coh.shape[1:])
    i_sum = np.zeros(inc.shape[1:])
    dxx_sq = np.zeros(coh.shape[1:3])
    for s in range(S):
        c_sum = c_sum + coh[s]
        i_sum = i_sum + inc[s]
        t = coh[s, :, :, 0] + inc[s, :, :, 0]
        dxx_sq = dxx_sq + t * t
    c_mean = c_sum / float(S)
    i_mean = i_sum / float(S)
    if S == 1:
        xxd = np.zeros(coh.shape[1:3])
    else:
        sq_exp = dxx_sq / float(S)
        exp = c_mean[:, :, 0] + i_mean[:, :, 0]
        xxd = np.sqrt((sq_exp - exp * exp) / (float(S) - 1.0)) / exp
    return {"coherent": c_mean, "incoherent": i_mean, "delta_xx": xxd}


def gather_sweep(local: dict, n_samples: int, dist=None) -> tuple:
    """The one exchange of a multi-GPU sweep: every rank holds the sigmas of its
    own samples, {sample index: (coherent [field][T][2], incoherent [field][T][2])};
    all of them are gathered (torch.distributed all_gather_object, any backend)
    and returned as dense [sample][field][T][2] arrays in sample order. With
    dist None (one process) the local results are returned as they are."""
    parts = [local]
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, local)
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise ValueError(f"sample {k} was computed by more than one rank")
            merged[k] = v
    if sorted(merged) != list(range(n_samples)):
        raise ValueError(f"gathered samples {sorted(merged)} are not 0..{n_samples - 1}")
    coh = np.stack([np.asarray(merged[k][0], dtype=np.float64) for k in range(n_samples)])
    inc = np.stack([np.asarray(merged[k][1], dtype=np.float64) for k in range(n_samples)])
    return coh, inc


def per_sample_sigmas(passes: list, out: np.ndarray, sample_of_grid: dict, n_fields: int, n_t: int) -> dict:
    """Regroups a batch's results ([pass][T][2], passes as sweep_passes orders
    them: per sample, per field, coherent then incoherent) into
    {sample index: (coherent [field][T][2], incoherent [field][T][2])}."""
    res = {}
    for k, p in enumerate(passes):
        s = sample_of_grid[p.grid]
        if s not in res:
            res[s] = (np.zeros((n_fields, n_t, 2)), np.zeros((n_fields, n_t, 2)))
        f = (k // 2) % n_fields
        res[s][0 if p.coherent else 1][f] = out[k, :n_t, :]
    return res
