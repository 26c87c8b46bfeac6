"""ctypes access to oracle/_ref/libes_refbind.so (test infrastructure only): the
reference's own sweep loop over a `Simulation*` that is either the reference's
SimulationCPU (backend 0) or the reference-side binding SimulationCUDA
(elasticscattering_b200/refbind/SimulationCUDA.h, backend 1)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
REFBIND_SO = ROOT / "oracle" / "_ref" / "libes_refbind.so"
_lib = None


def available() -> bool:
    return REFBIND_SO.exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(REFBIND_SO))
        _vp, _d, _i = C.c_void_p, C.c_double, C.c_int
        _lib.rb_sweep.restype = _i
        _lib.rb_sweep.argtypes = [_i, _vp, _i, _d, _d, _d, _d, _i, _i, _i, _d, _d, _i, _d, _vp, _i, _vp, _i, _i,
                                  _vp, _vp, _vp, _vp]
    return _lib


def sweep(backend: int, w, seeds, dim: int, ppq: int, fields, temps, images: bool = False):
    """RunSimulation's loop (samples x sectors x fields) through the chosen backend.
    Returns sigma [sample][sector][field][T][2], metrics [..][7], avg lifetime [..],
    and with images the maps [sample][sector][field][T][3][dim*dim]."""
    seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
    fields = np.ascontiguousarray(fields, dtype=np.float64)
    temps = np.ascontiguousarray(temps, dtype=np.float64)
    S, F, T = len(seeds), len(fields), len(temps)
    out = np.zeros((S, 2, F, T, 2))
    met = np.zeros((S, 2, F, 7), dtype=np.int32)
    avg = np.zeros((S, 2, F))
    maps = np.zeros((S, 2, F, T, 3, dim * dim)) if images else None
    rc = lib().rb_sweep(backend, seeds.ctypes.data, S, w.region_size, w.region_extends, w.density,
                        w.impurity_radius, w.target_cell_population, dim, ppq, w.tau, w.alpha, int(w.clockwise),
                        w.particle_speed, fields.ctypes.data, F, temps.ctypes.data, T, int(images), out.ctypes.data,
                        met.ctypes.data, avg.ctypes.data, maps.ctypes.data if images else None)
    assert rc == 0
    return out, met, avg, maps
