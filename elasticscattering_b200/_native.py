"""ctypes declarations of the two in-tree native libraries.

libes_cuda.so (include/es_cuda.h) is the CUDA backend; libes_host.so
(include/es_host.h) is the host runtime (Grid, .config runner). Both are built
in-tree by elasticscattering_b200/build.py. There is no fallback: if a library
is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG = Path(__file__).resolve().parent

ES_OK = 0
ES_ERR_BAD_ARG = 1
ES_ERR_OOM = 2
ES_ERR_LAUNCH = 3
STATUS_NAMES = {
    0: "ES_OK", 1: "ES_ERR_BAD_ARG", 2: "ES_ERR_OOM", 3: "ES_ERR_LAUNCH", 4: "ES_ERR_WALK_CAP",
    5: "ES_ERR_DEVICE", 6: "ES_ERR_NO_GRID", 7: "ES_ERR_NO_SAMPLE", 8: "ES_ERR_TIMEOUT",
}
ES_PRECISION_FP64 = 0
ES_PRECISION_SPLIT = 1
ES_PRECISION_SPLIT_EXACT = 2


class EsError(RuntimeError):
    """A non-OK es_status, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class ImpuritySettings(C.Structure):
    """ImpuritySettings, reference src/sim/es/settings.h:76-85."""
    _fields_ = [("spawn_region_start", C.c_double), ("spawn_region_size", C.c_double),
                ("cell_size", C.c_double), ("cells_per_row", C.c_int32), ("impurity_radius", C.c_double)]


class Settings(C.Structure):
    """Settings, reference src/ConfigSettings.h:22-34 (bool widened to int32)."""
    _fields_ = [("tau", C.c_double), ("alpha", C.c_double), ("is_clockwise", C.c_int32),
                ("particle_speed", C.c_double), ("region_size", C.c_double), ("region_extends", C.c_double),
                ("impurity_density", C.c_double), ("impurity_radius", C.c_double),
                ("target_cell_population", C.c_int32)]


class Metrics(C.Structure):
    """ParticleMetrics, reference src/sim/es/particle_metrics.h:22-44, 64-bit."""
    _fields_ = [("cells_passed", C.c_int64), ("impurities_tested", C.c_int64),
                ("particles_inside_impurity", C.c_int64), ("particles_escaped", C.c_int64),
                ("particles_at_bound", C.c_int64), ("max_impurities_tested", C.c_int64),
                ("max_cells_passed", C.c_int64), ("crossings_tested", C.c_int64),
                ("start_cell_tests", C.c_int64), ("retraced_fp64", C.c_int64)]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class Tuning(C.Structure):
    """es_tuning: kernel choices of a context."""
    _fields_ = [("lifetime_variant", C.c_int32)]


ES_BATCH_MAX_T = 8
ES_BATCH_PERSISTENT = 2
ES_BATCH_PASS_KERNELS = 3


class BatchInstance(C.Structure):
    """es_batch_instance: one (sample, field, sector) pass of a batch."""
    _fields_ = [("grid", C.c_int32), ("positions_per_row", C.c_int32), ("particles_per_quadrant", C.c_int32),
                ("coherent", C.c_int32), ("region_size", C.c_double), ("grid_cell_size", C.c_double),
                ("magnetic_field", C.c_double), ("settings", Settings), ("n_t", C.c_int32),
                ("temperatures", C.c_double * ES_BATCH_MAX_T)]


class QueryMap(C.Structure):
    """es_mlp_query_map: feature maps and sigma scale of a surrogate's queries."""
    _fields_ = [("g_lo", C.c_double * 5), ("g_hi", C.c_double * 5), ("log_scale", C.c_int32 * 5),
                ("sigma0_per_tau", C.c_double), ("w_per_b", C.c_double)]


class BatchTuning(C.Structure):
    """es_batch_tuning: launch choices of a batch."""
    _fields_ = [("chunk_iters", C.c_int32), ("blocks_per_sm", C.c_int32), ("precision", C.c_int32),
                ("mode", C.c_int32)]


class SimDesc(C.Structure):
    _fields_ = [("positions_per_row", C.c_int32), ("particles_per_quadrant", C.c_int32),
                ("region_size", C.c_double), ("region_extends", C.c_double), ("grid_cell_size", C.c_double),
                ("device_ordinal", C.c_int32), ("precision", C.c_int32)]


# Every symbol include/es_cuda.h declares: name -> (restype, argtypes).
_vp, _d, _i32, _i64, _u32, _u64 = C.c_void_p, C.c_double, C.c_int32, C.c_int64, C.c_uint32, C.c_uint64
CUDA_API = {
    "es_create": (_i32, [C.POINTER(SimDesc), C.POINTER(_vp)]),
    "es_destroy": (_i32, [_vp]),
    "es_get_tuning": (_i32, [_vp, C.POINTER(Tuning)]),
    "es_set_tuning": (_i32, [_vp, C.POINTER(Tuning)]),
    "es_last_error": (C.c_char_p, [_vp]),
    "es_upload_grid": (_i32, [_vp, _vp, _i64, _vp, C.POINTER(ImpuritySettings), _u64]),
    "es_init_sample": (_i32, [_vp, C.POINTER(Settings), _i32]),
    "es_compute_sigmas": (_i32, [_vp, _d, _vp, _i32, _vp, C.POINTER(Metrics)]),
    "es_compute_sigmas_images": (_i32, [_vp, _d, _vp, _i32, _vp, _vp, _vp, _vp, C.POINTER(Metrics)]),
    "es_compute_lifetimes": (_i32, [_vp, _d, _vp, C.POINTER(Metrics)]),
    "es_derive_temperatures": (_i32, [_vp, _vp, _i32, _vp]),
    "es_read_lifetimes": (_i32, [_vp, _i64, _i64, _vp]),
    "es_set_rows": (_i32, [_vp, _i32, _i32]),
    "es_enqueue_derive_temperatures": (_i32, [_vp, _vp, _i32, _vp]),
    "es_enqueue_sigmas": (_i32, [_vp, _d, _vp, _i32, _vp]),
    "es_enqueue_lifetimes": (_i32, [_vp, _d]),
    "es_synchronize": (_i32, [_vp]),
    "es_average_lifetime": (_i32, [_vp, C.POINTER(_d)]),
    "es_read_metrics": (_i32, [_vp, C.POINTER(Metrics), _i32]),
    "es_stream": (_vp, [_vp]),
    "es_launch_count": (_i64, [_vp]),
    "es_probe_fp64_fma": (_i32, [_i32, C.POINTER(_d)]),
    "es_probe_fp32_fma": (_i32, [_i32, C.POINTER(_d)]),
    "es_fault_inject": (_i32, [C.c_char_p]),
    "es_fault_counts": (_i32, [C.POINTER(_i64)]),
    "es_derive_temperatures_noalloc": (_i32, [_vp, _i32, _i32, C.POINTER(Settings), _i32, _d, _vp, _i32, _vp, _vp]),
    "es_batch_create": (_i32, [_i32, C.POINTER(_vp)]),
    "es_batch_destroy": (_i32, [_vp]),
    "es_batch_last_error": (C.c_char_p, [_vp]),
    "es_batch_get_tuning": (_i32, [_vp, C.POINTER(BatchTuning)]),
    "es_batch_set_tuning": (_i32, [_vp, C.POINTER(BatchTuning)]),
    "es_batch_add_grid": (_i32, [_vp, _vp, _i64, _vp, C.POINTER(ImpuritySettings), C.POINTER(_i32)]),
    "es_batch_clear": (_i32, [_vp]),
    "es_batch_set_instances": (_i32, [_vp, C.POINTER(BatchInstance), _i32]),
    "es_batch_run": (_i32, [_vp, _vp, _vp]),
    "es_batch_enqueue": (_i32, [_vp]),
    "es_batch_collect": (_i32, [_vp, _vp, _vp]),
    "es_batch_stream": (_vp, [_vp]),
    "es_batch_launch_count": (_i64, [_vp]),
    "es_batch_graph_kernels": (_i64, [_vp]),
    "es_batch_total_orbits": (_i64, [_vp]),
    "es_dgrid_create_seeded": (_i32, [_i32, _u32, _d, _d, _d, _d, _i32, _i64, C.POINTER(_vp)]),
    "es_dgrid_destroy": (_i32, [_vp]),
    "es_dgrid_info": (_i32, [_vp, C.POINTER(ImpuritySettings), C.POINTER(_i64), C.POINTER(_i64)]),
    "es_dgrid_download": (_i32, [_vp, _vp, _vp]),
    "es_upload_dgrid": (_i32, [_vp, _vp]),
    "es_batch_add_dgrid": (_i32, [_vp, _vp, C.POINTER(_i32)]),
    "es_mlp_param_count": (_i64, []),
    "es_mlp_create": (_i32, [_i32, _i32, C.POINTER(_vp)]),
    "es_mlp_destroy": (_i32, [_vp]),
    "es_mlp_last_error": (C.c_char_p, [_vp]),
    "es_mlp_set_params": (_i32, [_vp, _vp]),
    "es_mlp_get_params": (_i32, [_vp, _vp]),
    "es_mlp_set_dataset": (_i32, [_vp, _vp, _vp, _i64]),
    "es_mlp_train": (_i32, [_vp, _i32, _i32, C.c_float, _u64, _vp]),
    "es_mlp_gradients": (_i32, [_vp, _vp, _vp, _i32, _vp, _vp]),
    "es_mlp_predict": (_i32, [_vp, _vp, _i64, _vp, _vp, _vp]),
    "es_mlp_query": (_i32, [_vp, C.POINTER(QueryMap), _vp, _i64, _vp, _vp, _vp]),
    "es_mlp_launch_count": (_i64, [_vp]),
    "es_mlp_stream": (_vp, [_vp]),
    "es_debug_trace": (_i32, [_vp, _d, _d, _i32, _i32, _d, _d, _d, _d, _d, _i32, _i32, C.POINTER(_d)]),
    "es_debug_finish_retrace": (_i32, [_vp, _i32]),
    "es_debug_next_cell": (_i32, [_vp, _d, _d, _d, _i32, _d, C.POINTER(ImpuritySettings), _vp, _vp,
                                  C.POINTER(_i32)]),
}

HOST_API = {
    "es_grid_create_seeded": (_i32, [_u32, _d, _d, _d, _d, _i32, _i64, C.POINTER(_vp)]),
    "es_grid_create_from_list": (_i32, [_vp, _i64, _d, _d, _d, _i32, C.POINTER(_vp)]),
    "es_grid_destroy": (None, [_vp]),
    "es_grid_impurities": (C.POINTER(C.c_double), [_vp]),
    "es_grid_index": (C.POINTER(C.c_int32), [_vp]),
    "es_grid_indexed_count": (_i64, [_vp]),
    "es_grid_unique_count": (_i64, [_vp]),
    "es_grid_cells_per_row": (_i32, [_vp]),
    "es_grid_seed": (_u32, [_vp]),
    "es_grid_generation": (_u64, [_vp]),
    "es_grid_settings": (None, [_vp, C.POINTER(ImpuritySettings)]),
    "es_run_config": (_i32, [C.c_char_p, C.c_char_p, _i32, _i32]),
    "es_config_describe": (_i32, [C.c_char_p, C.c_char_p, _i32]),
    "es_host_last_error": (C.c_char_p, []),
}

_libs: dict[str, C.CDLL] = {}


def _load(name: str, api: dict) -> C.CDLL:
    if name in _libs:
        return _libs[name]
    path = PKG / name
    if not path.exists():
        raise ImportError(f"{path} is not built; run `python -m elasticscattering_b200.build`")
    lib = C.CDLL(str(path), mode=C.RTLD_GLOBAL)
    for sym, (res, args) in api.items():
        if not hasattr(lib, sym):
            continue
        fn = getattr(lib, sym)
        fn.restype = res
        fn.argtypes = args
    _libs[name] = lib
    return lib


def cuda_lib() -> C.CDLL:
    return _load("libes_cuda.so", CUDA_API)


def host_lib() -> C.CDLL:
    cuda_lib()
    return _load("libes_host.so", HOST_API)


def fault_inject(spec: str | None) -> None:
    """Arms host-side fault injection (es_fault_inject): "alloc:N", "copy:N",
    "launch:N" items, comma-separated, "+" after N for "and every later one";
    None or "" disarms."""
    st = cuda_lib().es_fault_inject(spec.encode() if spec else None)
    if st != ES_OK:
        raise EsError(st, cuda_lib().es_last_error(None).decode())


def fault_counts() -> dict:
    """Operations counted since the last fault_inject, and how many failed."""
    out = (_i64 * 4)()
    cuda_lib().es_fault_counts(out)
    return {"alloc": out[0], "copy": out[1], "launch": out[2], "failed": out[3]}


def check(status: int, ctx=None) -> None:
    if status != ES_OK:
        msg = cuda_lib().es_last_error(ctx)
        raise EsError(status, msg.decode() if msg else "")


def check_batch(status: int, batch) -> None:
    if status != ES_OK:
        msg = cuda_lib().es_batch_last_error(batch)
        raise EsError(status, msg.decode() if msg else "")


def check_mlp(status: int, mlp) -> None:
    if status != ES_OK:
        msg = cuda_lib().es_mlp_last_error(mlp)
        raise EsError(status, msg.decode() if msg else "")


def check_host(status: int) -> None:
    if status != ES_OK:
        msg = host_lib().es_host_last_error()
        raise EsError(status, msg.decode() if msg else "")
