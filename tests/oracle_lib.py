"""ctypes access to the CPU oracles (test infrastructure only).

- liboracle.so : the C restatement of the reference's FP64 path (oracle/es_oracle.c)
- libes_ref.so : the reference's own CPU sources compiled in place (oracle/_ref)

Only tests, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
import hashlib
from dataclasses import dataclass
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_SO = ROOT / "oracle" / "liboracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "libes_ref.so"

_vp, _d, _i32, _i64, _u32 = C.c_void_p, C.c_double, C.c_int32, C.c_int64, C.c_uint32


class OrcIS(C.Structure):
    _fields_ = [("spawn_region_start", _d), ("spawn_region_size", _d), ("cell_size", _d),
                ("cells_per_row", _i32), ("impurity_radius", _d)]


class OrcMetrics(C.Structure):
    _fields_ = [("cells_passed", _i64), ("impurities_tested", _i64), ("particles_inside_impurity", _i64),
                ("particles_escaped", _i64), ("particles_at_bound", _i64), ("max_impurities_tested", _i64),
                ("max_cells_passed", _i64)]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class OrcSim(C.Structure):
    _fields_ = [("positions_per_row", _i32), ("particles_per_quadrant", _i32), ("region_size", _d),
                ("grid_cell_size", _d), ("particle_speed", _d), ("alpha", _d), ("tau", _d),
                ("is_clockwise", _i32), ("is_coherent", _i32)]


_oracle = None
_ref = None


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        lib = C.CDLL(str(ORACLE_SO))
        lib.orc_generate_impurities.argtypes = [_u32, _i64, _d, _d, _vp]
        lib.orc_grid_seed_sizes.argtypes = [_d, _d, _d, _i32, _vp, _vp]
        lib.orc_grid_build.restype = _i64
        lib.orc_grid_build.argtypes = [_vp, _i64, _d, _d, _d, _i32, _vp, _vp]
        lib.orc_grid_settings.argtypes = [_d, _d, _d, _i32, C.POINTER(OrcIS)]
        lib.orc_lifetimes.argtypes = [C.POINTER(OrcSim), C.POINTER(OrcIS), _vp, _vp, _d, _i32, _i32, _vp,
                                      C.POINTER(OrcMetrics)]
        lib.orc_trace_one.restype = _d
        lib.orc_trace_one.argtypes = [C.POINTER(OrcSim), C.POINTER(OrcIS), _vp, _vp, _d, _d, _d, _i32, _i32,
                                      C.POINTER(OrcMetrics)]
        lib.orc_trace_explicit.restype = _d
        lib.orc_trace_explicit.argtypes = [C.POINTER(OrcIS), _vp, _vp, _d, _d, _d, _i32, _i32, _d, _d, _d, _d,
                                           _i32, _i32]
        lib.orc_derive_temperature.argtypes = [C.POINTER(OrcSim), _d, _d, _vp, _vp]
        lib.orc_derive_temperature_images.argtypes = [C.POINTER(OrcSim), _d, _d, _vp, _vp, _vp, _vp, _vp]
        lib.orc_get_angle.restype = _d
        lib.orc_get_angle.argtypes = [_d, _d, _d, _d, _d, C.c_int]
        lib.orc_angle_in_range.restype = C.c_int
        lib.orc_angle_in_range.argtypes = [_d, _d, _d, C.c_int]
        lib.orc_cross_angle.restype = _d
        lib.orc_cross_angle.argtypes = [_d, _d, C.c_int]
        lib.orc_bound_time.restype = _d
        lib.orc_bound_time.argtypes = [_d, _d, _d, C.c_int, C.c_int, C.c_int]
        lib.orc_circles_cross.restype = C.c_int
        lib.orc_circles_cross.argtypes = [_d, _d, _d, _d, _d, _d]
        lib.orc_first_cross_time.restype = _d
        lib.orc_first_cross_time.argtypes = [_d, _d, _d, C.c_int, _d, _d, _d, _d, _d, _d, _d]
        lib.orc_simpson_weight.restype = _d
        lib.orc_simpson_weight.argtypes = [C.c_int, C.c_int]
        lib.orc_next_cell.restype = C.c_int
        lib.orc_next_cell.argtypes = [_d, _d, _d, C.c_int, _d, C.POINTER(OrcIS), _vp, _vp]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return REF_SO.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REF_SO))
        lib.ref_grid_new_seed.restype = _vp
        lib.ref_grid_new_seed.argtypes = [_u32, _d, _d, _d, _d, C.c_int]
        lib.ref_grid_new_list.restype = _vp
        lib.ref_grid_new_list.argtypes = [_vp, C.c_int, _d, _d, _d, C.c_int]
        lib.ref_grid_free.argtypes = [_vp]
        lib.ref_grid_info.argtypes = [_vp] + [_vp] * 7
        lib.ref_grid_copy.argtypes = [_vp, _vp, _vp]
        lib.ref_sim_new.restype = _vp
        lib.ref_sim_new.argtypes = [_vp, C.c_int, C.c_int, _d, _d, C.c_int, _d, _d, _d]
        lib.ref_sim_free.argtypes = [_vp]
        lib.ref_sim_init_sample.argtypes = [_vp, C.c_int]
        lib.ref_sim_lifetimes.argtypes = [_vp, _d, _vp, _vp]
        lib.ref_sim_lifetimes_rows.restype = C.c_longlong
        lib.ref_sim_lifetimes_rows.argtypes = [_vp, _d, C.c_int, C.c_int, _vp, _vp]
        lib.ref_sim_sigmas.argtypes = [_vp, _d, _vp, C.c_int, _vp, _vp]
        lib.ref_sim_sigmas_images.argtypes = [_vp, _d, _vp, C.c_int, _vp, _vp, _vp, _vp]
        lib.ref_sim_derive.argtypes = [_vp, _d, _d, _vp, _vp]
        _ref = lib
    return _ref


@dataclass
class OracleGrid:
    xy: np.ndarray        # (n, 2) ordered impurities
    cell_end: np.ndarray  # int32 cumulative ends
    settings: OrcIS
    unique: int


def oracle_grid_seeded(seed: int, region_size: float, region_extends: float, density: float, radius: float,
                       tcp: int) -> OracleGrid:
    lib = oracle()
    u, c = C.c_int64(), C.c_int32()
    rc = lib.orc_grid_seed_sizes(region_size, region_extends, density, tcp, C.byref(u), C.byref(c))
    if rc != 0:
        raise ValueError("Woah!" if rc == 1 else "No impurities")
    imps = np.zeros(2 * u.value)
    lib.orc_generate_impurities(seed & 0xFFFFFFFF, u.value, -region_extends, region_size + region_extends,
                                imps.ctypes.data)
    return _oracle_bin(imps.reshape(-1, 2), region_size, region_extends, radius, c.value, u.value)


def oracle_grid_list(xy, region_size: float, region_extends: float, radius: float, tcp: int) -> OracleGrid:
    xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1, 2)
    n = len(xy)
    # Grid(vector<v2>, ...), src/sim/Grid.cpp:53: C round() rounds half away from zero.
    v = float(np.sqrt(n / float(tcp)))
    r = int(np.floor(v))
    cpr = max(r + 1 if v - r >= 0.5 else r, 1)
    return _oracle_bin(xy, region_size, region_extends, radius, cpr, n)


def _oracle_bin(xy, region_size, region_extends, radius, cpr, unique) -> OracleGrid:
    lib = oracle()
    xy = np.ascontiguousarray(xy, dtype=np.float64)
    n_idx = lib.orc_grid_build(xy.ctypes.data, len(xy), region_extends, region_size, radius, cpr, None, None)
    out = np.zeros(2 * n_idx)
    ce = np.zeros(cpr * cpr, dtype=np.int32)
    lib.orc_grid_build(xy.ctypes.data, len(xy), region_extends, region_size, radius, cpr, out.ctypes.data,
                       ce.ctypes.data)
    s = OrcIS()
    lib.orc_grid_settings(region_size, region_extends, radius, cpr, C.byref(s))
    return OracleGrid(out.reshape(-1, 2), ce, s, unique)


def oracle_lifetimes(g: OracleGrid, dim: int, ppq: int, region_size: float, speed: float, alpha: float, tau: float,
                     clockwise: bool, coherent: bool, B: float, rows: tuple[int, int] | None = None):
    lib = oracle()
    sim = OrcSim(dim, ppq, region_size, g.settings.cell_size, speed, alpha, tau, int(clockwise), int(coherent))
    j0, j1 = rows if rows else (0, dim)
    out = np.zeros((j1 - j0) * dim * 4 * ppq)
    m = OrcMetrics()
    xy = np.ascontiguousarray(g.xy)
    lib.orc_lifetimes(C.byref(sim), C.byref(g.settings), xy.ctypes.data, g.cell_end.ctypes.data, B, j0, j1,
                      out.ctypes.data, C.byref(m))
    return out, m.as_dict()


def oracle_sigmas(g: OracleGrid, dim: int, ppq: int, region_size: float, speed: float, alpha: float, tau: float,
                  clockwise: bool, coherent: bool, B: float, temperatures, lifetimes=None):
    lib = oracle()
    sim = OrcSim(dim, ppq, region_size, g.settings.cell_size, speed, alpha, tau, int(clockwise), int(coherent))
    if lifetimes is None:
        lifetimes, _ = oracle_lifetimes(g, dim, ppq, region_size, speed, alpha, tau, clockwise, coherent, B)
    lifetimes = np.ascontiguousarray(lifetimes)
    res = []
    for T in temperatures:
        o = np.zeros(2)
        lib.orc_derive_temperature(C.byref(sim), B, float(T), lifetimes.ctypes.data, o.ctypes.data)
        res.append((float(o[0]), float(o[1])))
    return res


def oracle_images(g: OracleGrid, dim: int, ppq: int, region_size: float, speed: float, alpha: float, tau: float,
                  clockwise: bool, coherent: bool, B: float, T: float, lifetimes):
    lib = oracle()
    sim = OrcSim(dim, ppq, region_size, g.settings.cell_size, speed, alpha, tau, int(clockwise), int(coherent))
    lifetimes = np.ascontiguousarray(lifetimes)
    o = np.zeros(2)
    lt, xx, xy = (np.zeros(dim * dim) for _ in range(3))
    lib.orc_derive_temperature_images(C.byref(sim), B, float(T), lifetimes.ctypes.data, o.ctypes.data,
                                      lt.ctypes.data, xx.ctypes.data, xy.ctypes.data)
    return (float(o[0]), float(o[1])), lt, xx, xy


def sha256(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def parse_config_text(text: str) -> dict:
    """Key/value lines as the reference's SimulationConfiguration::ParseFromeFile
    reads them (src/SimulationConfiguration.h:90-106): skip empty, '#' and ':/'
    lines; key up to the first space; the first occurrence of a key wins."""
    values: dict[str, str] = {}
    for line in text.splitlines():
        if not line or line[0] == "\n" or line[0] == "#" or (len(line) > 1 and line[0] == ":" and line[1] == "/"):
            continue
        pos = line.find(" ")
        key = line if pos < 0 else line[:pos]
        val = "" if pos < 0 else line[pos + 1:]
        values.setdefault(key, val.strip())
    return values
