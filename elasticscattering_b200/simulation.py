"""Python mirror of the reference's plugin interface for the conductivity path.

The reference drives a backend through `class Simulation`
(src/sim/Simulation.h:56-147): a constructor taking (positions_per_row,
phi_steps, GridInformation), `InitSample(grid, settings, coherent)`, and
`ComputeSigmas` / `ComputeSigmasWithImages(B, temperatures, grid,
sample_metrics)`, fed by a `Grid` (src/sim/Grid.h:55-94). The classes here keep
those names and argument meanings and call the CUDA backend through its C ABI
(include/es_cuda.h). Errors raise EsError instead of the reference's
print-and-exit (src/utils/ErrorMacros.h:22-38).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from ._native import EsError, ImpuritySettings, Metrics, Settings


@dataclass
class Sigma:
    """Sigma, reference src/SimulationResult.h:24-52."""
    xx: float = 0.0
    xy: float = 0.0

    def __add__(self, o: "Sigma") -> "Sigma":
        return Sigma(o.xx + self.xx, o.xy + self.xy)

    def __iadd__(self, o: "Sigma") -> "Sigma":
        self.xx += o.xx
        self.xy += o.xy
        return self


@dataclass
class IterationResult:
    """IterationResult, reference src/SimulationResult.h:80-87: per-position maps
    (dim*dim, row-major [j][i]) of the truncated lifetime and of sigma_xx/xy
    integrated over phase, plus the sigmas."""
    particle_lifetimes: np.ndarray
    xx_buffer: np.ndarray
    xy_buffer: np.ndarray
    result: Sigma


@dataclass
class SampleMetrics:
    """SampleMetrics, reference src/Metrics.h:50-80."""
    sample_index: int = 0
    coherent: bool = False
    total_particles: int = 0
    total_cells: int = 0
    impurity_count: int = 0
    seed: int = 0
    total_indexed_impurities: int = 0
    iteration_metrics: list = field(default_factory=list)


def make_settings(tau: float, alpha: float, is_clockwise: bool, particle_speed: float, region_size: float,
                  region_extends: float, impurity_density: float, impurity_radius: float,
                  target_cell_population: int = 15) -> Settings:
    """Settings, reference src/ConfigSettings.h:22-34."""
    return Settings(tau, alpha, 1 if is_clockwise else 0, particle_speed, region_size, region_extends,
                    impurity_density, impurity_radius, int(target_cell_population))


class Grid:
    """Impurity field + cell index (reference Grid, src/sim/Grid.cpp), built by
    the host C++ runtime (libes_host.so)."""

    def __init__(self, handle: int, region_size: float, region_extends: float):
        self._h = C.c_void_p(handle)
        self.region_size = region_size
        self.region_extends = region_extends

    @classmethod
    def from_seed(cls, seed: int, region_size: float, region_extends: float, density: float,
                  impurity_radius: float, target_cell_population: int, max_impurities: int = 0) -> "Grid":
        lib = N.host_lib()
        h = C.c_void_p()
        N.check_host(lib.es_grid_create_seeded(seed & 0xFFFFFFFF, region_size, region_extends, density,
                                               impurity_radius, int(target_cell_population), int(max_impurities),
                                               C.byref(h)))
        return cls(h.value, region_size, region_extends)

    @classmethod
    def from_list(cls, impurities, region_size: float, region_extends: float, impurity_radius: float,
                  target_cell_population: int) -> "Grid":
        xy = np.ascontiguousarray(impurities, dtype=np.float64).reshape(-1, 2)
        lib = N.host_lib()
        h = C.c_void_p()
        N.check_host(lib.es_grid_create_from_list(xy.ctypes.data, len(xy), region_size, region_extends,
                                                  impurity_radius, int(target_cell_population), C.byref(h)))
        return cls(h.value, region_size, region_extends)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            try:
                N.host_lib().es_grid_destroy(self._h)
            except Exception:  # interpreter shutdown: the library may already be gone
                pass
            self._h = C.c_void_p()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def GetTotalImpurityCount(self) -> int:
        return int(N.host_lib().es_grid_indexed_count(self._h))

    def GetUniqueImpurityCount(self) -> int:
        return int(N.host_lib().es_grid_unique_count(self._h))

    def GetCellsPerRow(self) -> int:
        return int(N.host_lib().es_grid_cells_per_row(self._h))

    def GetSeed(self) -> int:
        return int(N.host_lib().es_grid_seed(self._h))

    def GetSettings(self) -> ImpuritySettings:
        s = ImpuritySettings()
        N.host_lib().es_grid_settings(self._h, C.byref(s))
        return s

    def GetImpurities(self) -> np.ndarray:
        n = self.GetTotalImpurityCount()
        if n == 0:
            return np.zeros((0, 2))
        p = N.host_lib().es_grid_impurities(self._h)
        return np.ctypeslib.as_array(p, shape=(n * 2,)).reshape(n, 2).copy()

    def GetIndex(self) -> np.ndarray:
        c = self.GetCellsPerRow()
        p = N.host_lib().es_grid_index(self._h)
        return np.ctypeslib.as_array(p, shape=(c * c,)).copy()

    def arrays(self) -> tuple:
        """(impurity x,y pairs, their count, cell index) as pointers into this
        Grid's own host memory, valid while the Grid lives: what es_upload_grid
        and es_batch_add_grid read, without a copy."""
        n = self.GetTotalImpurityCount()
        xy = C.cast(N.host_lib().es_grid_impurities(self._h), C.c_void_p) if n else None
        idx = C.cast(N.host_lib().es_grid_index(self._h), C.c_void_p)
        return xy, n, idx

    def info(self) -> "GridInformation":
        return GridInformation(self.region_size, self.region_extends, self.GetSettings().cell_size,
                               self.GetTotalImpurityCount(), self.GetCellsPerRow() ** 2)


class DeviceGrid:
    """The seeded Grid built on the GPU (es_dgrid_create_seeded): the host Grid's
    impurity positions, ordered array and cell index, bit for bit, without the
    host build or the upload. Same getters as Grid (copies to the host)."""

    def __init__(self, handle: int, region_size: float, region_extends: float, seed: int, device: int):
        self._h = C.c_void_p(handle)
        self.region_size = region_size
        self.region_extends = region_extends
        self.seed = seed
        self.device = device

    @classmethod
    def from_seed(cls, seed: int, region_size: float, region_extends: float, density: float,
                  impurity_radius: float, target_cell_population: int, max_impurities: int = 0,
                  device: int = 0) -> "DeviceGrid":
        h = C.c_void_p()
        N.check(N.cuda_lib().es_dgrid_create_seeded(int(device), seed & 0xFFFFFFFF, region_size, region_extends,
                                                    density, impurity_radius, int(target_cell_population),
                                                    int(max_impurities), C.byref(h)), None)
        return cls(h.value, region_size, region_extends, seed, device)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            N.cuda_lib().es_dgrid_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may already be gone
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def _info(self):
        s = ImpuritySettings()
        n_idx, n_unique = C.c_int64(), C.c_int64()
        N.check(N.cuda_lib().es_dgrid_info(self._h, C.byref(s), C.byref(n_idx), C.byref(n_unique)), None)
        return s, int(n_idx.value), int(n_unique.value)

    def GetTotalImpurityCount(self) -> int:
        return self._info()[1]

    def GetUniqueImpurityCount(self) -> int:
        return self._info()[2]

    def GetCellsPerRow(self) -> int:
        return int(self._info()[0].cells_per_row)

    def GetSeed(self) -> int:
        return self.seed

    def GetSettings(self) -> ImpuritySettings:
        return self._info()[0]

    def GetImpurities(self) -> np.ndarray:
        n = self.GetTotalImpurityCount()
        out = np.zeros((n, 2))
        if n:
            N.check(N.cuda_lib().es_dgrid_download(self._h, out.ctypes.data, None), None)
        return out

    def GetIndex(self) -> np.ndarray:
        c = self.GetCellsPerRow()
        out = np.zeros(c * c, dtype=np.int32)
        N.check(N.cuda_lib().es_dgrid_download(self._h, None, out.ctypes.data), None)
        return out

    def info(self) -> "GridInformation":
        s, n_idx, _ = self._info()
        return GridInformation(self.region_size, self.region_extends, s.cell_size, n_idx, s.cells_per_row ** 2)


@dataclass
class GridInformation:
    """GridInformation, reference src/sim/es/settings.h:65-73."""
    region_size: float
    region_extends: float
    cell_size: float
    indexed_impurity_count: int
    index_size: int


class SimulationCUDA:
    """The B200 backend behind the reference's Simulation interface
    (src/sim/Simulation.h:56-147), one CUDA context + stream per instance."""

    def __init__(self, positions_per_row: int, phi_steps: int, grid_info: GridInformation, device: int = 0,
                 precision: int = N.ES_PRECISION_FP64):
        lib = N.cuda_lib()
        desc = N.SimDesc(int(positions_per_row), int(phi_steps), grid_info.region_size, grid_info.region_extends,
                         grid_info.cell_size, int(device), int(precision))
        h = C.c_void_p()
        N.check(lib.es_create(C.byref(desc), C.byref(h)), None)
        self._ctx = h
        self.positions_per_row = int(positions_per_row)
        self.phi_steps = int(phi_steps)
        self.n_orbits = self.positions_per_row ** 2 * 4 * self.phi_steps

    def close(self) -> None:
        if getattr(self, "_ctx", None) and self._ctx.value:
            N.cuda_lib().es_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library handles may already be gone
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def ctx(self) -> C.c_void_p:
        return self._ctx

    def _check(self, st: int) -> None:
        N.check(st, self._ctx)

    def _upload(self, grid) -> None:
        if isinstance(grid, DeviceGrid):
            self._check(N.cuda_lib().es_upload_dgrid(self._ctx, grid.handle))
            return
        xy, n, idx = grid.arrays()
        s = grid.GetSettings()
        gen = int(N.host_lib().es_grid_generation(grid.handle))
        self._check(N.cuda_lib().es_upload_grid(self._ctx, xy, n, idx, C.byref(s), gen))

    def upload_grid(self, grid: Grid) -> None:
        self._upload(grid)

    def InitSample(self, grid: Grid, settings: Settings, coherent: bool) -> None:
        """Simulation::InitSample, src/sim/Simulation.h:111-126."""
        self._upload(grid)
        self._check(N.cuda_lib().es_init_sample(self._ctx, C.byref(settings), 1 if coherent else 0))

    def ComputeSigmas(self, magnetic_field: float, temperatures, grid: Grid | None = None,
                      sample_metrics: SampleMetrics | None = None) -> list[Sigma]:
        """Simulation::ComputeSigmas, src/sim/Simulation.h:128."""
        ts = np.ascontiguousarray(temperatures, dtype=np.float64)
        out = np.zeros(2 * len(ts))
        m = Metrics()
        self._check(N.cuda_lib().es_compute_sigmas(self._ctx, float(magnetic_field), ts.ctypes.data, len(ts),
                                                   out.ctypes.data, C.byref(m)))
        if sample_metrics is not None:
            sample_metrics.iteration_metrics.append(m.as_dict())
        return [Sigma(float(out[2 * t]), float(out[2 * t + 1])) for t in range(len(ts))]

    def ComputeSigmasWithImages(self, magnetic_field: float, temperatures, grid: Grid | None = None,
                                sample_metrics: SampleMetrics | None = None) -> list[IterationResult]:
        """Simulation::ComputeSigmasWithImages, src/sim/Simulation.h:129."""
        ts = np.ascontiguousarray(temperatures, dtype=np.float64)
        nt, npos = len(ts), self.positions_per_row ** 2
        out = np.zeros(2 * nt)
        lt, xx, xy = (np.zeros(nt * npos) for _ in range(3))
        m = Metrics()
        self._check(N.cuda_lib().es_compute_sigmas_images(self._ctx, float(magnetic_field), ts.ctypes.data, nt,
                                                          out.ctypes.data, lt.ctypes.data, xx.ctypes.data,
                                                          xy.ctypes.data, C.byref(m)))
        if sample_metrics is not None:
            sample_metrics.iteration_metrics.append(m.as_dict())
        return [IterationResult(lt[t * npos:(t + 1) * npos].copy(), xx[t * npos:(t + 1) * npos].copy(),
                                xy[t * npos:(t + 1) * npos].copy(), Sigma(float(out[2 * t]), float(out[2 * t + 1])))
                for t in range(nt)]

    def ComputeLifetimes(self, magnetic_field: float, copy: bool = True) -> tuple[np.ndarray | None, dict]:
        """SimulationCL::ComputeLifetimes (src/sim/SimulationCL.cpp:113-177) with the
        raw lifetimes copied out ([j][i][q][p] order) and the metrics. copy=False
        leaves them on the device only (ReadLifetimes reads a range)."""
        out = np.zeros(self.n_orbits) if copy else None
        m = Metrics()
        self._check(N.cuda_lib().es_compute_lifetimes(self._ctx, float(magnetic_field),
                                                      out.ctypes.data if copy else None, C.byref(m)))
        return out, m.as_dict()

    def SetRows(self, j0: int, j1: int) -> None:
        """es_set_rows: the following passes cover start rows [j0, j1) only, and
        their sigmas are those rows' share (shares of a row partition add up)."""
        self._check(N.cuda_lib().es_set_rows(self._ctx, int(j0), int(j1)))

    def ReadLifetimes(self, first: int, count: int) -> np.ndarray:
        """es_read_lifetimes: `count` resident lifetimes from orbit `first` on."""
        out = np.zeros(int(count))
        self._check(N.cuda_lib().es_read_lifetimes(self._ctx, int(first), int(count), out.ctypes.data))
        return out

    def DeriveTemperatures(self, temperatures) -> list[Sigma]:
        ts = np.ascontiguousarray(temperatures, dtype=np.float64)
        out = np.zeros(2 * len(ts))
        self._check(N.cuda_lib().es_derive_temperatures(self._ctx, ts.ctypes.data, len(ts), out.ctypes.data))
        return [Sigma(float(out[2 * t]), float(out[2 * t + 1])) for t in range(len(ts))]

    def enqueue_sigmas(self, magnetic_field: float, temperatures: np.ndarray, d_out_ptr: int) -> None:
        """es_enqueue_sigmas: asynchronous pass writing 2*n_t doubles to device memory."""
        ts = np.ascontiguousarray(temperatures, dtype=np.float64)
        self._check(N.cuda_lib().es_enqueue_sigmas(self._ctx, float(magnetic_field), ts.ctypes.data, len(ts),
                                                   C.c_void_p(d_out_ptr)))

    def enqueue_derive_temperatures(self, temperatures: np.ndarray, d_out_ptr: int) -> None:
        """es_enqueue_derive_temperatures: stages (b)+(c) on the resident lifetimes,
        2*n_t doubles to device memory, no host wait."""
        ts = np.ascontiguousarray(temperatures, dtype=np.float64)
        self._check(N.cuda_lib().es_enqueue_derive_temperatures(self._ctx, ts.ctypes.data, len(ts),
                                                                C.c_void_p(d_out_ptr)))

    def synchronize(self) -> None:
        self._check(N.cuda_lib().es_synchronize(self._ctx))

    def read_metrics(self, reset: bool = True) -> dict:
        m = Metrics()
        self._check(N.cuda_lib().es_read_metrics(self._ctx, C.byref(m), 1 if reset else 0))
        return m.as_dict()

    def get_tuning(self) -> dict:
        t = N.Tuning()
        self._check(N.cuda_lib().es_get_tuning(self._ctx, C.byref(t)))
        return {name: int(getattr(t, name)) for name, _ in N.Tuning._fields_}

    def set_tuning(self, **fields) -> None:
        t = N.Tuning()
        self._check(N.cuda_lib().es_get_tuning(self._ctx, C.byref(t)))
        for k, v in fields.items():
            setattr(t, k, int(v))
        self._check(N.cuda_lib().es_set_tuning(self._ctx, C.byref(t)))

    def stream_handle(self) -> int:
        return int(N.cuda_lib().es_stream(self._ctx) or 0)

    def launch_count(self) -> int:
        return int(N.cuda_lib().es_launch_count(self._ctx))


__all__ = ["EsError", "Grid", "GridInformation", "IterationResult", "SampleMetrics", "Settings", "Sigma",
           "SimulationCUDA", "make_settings"]
