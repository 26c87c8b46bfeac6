"""Host runtime and C ABI, on the CPU (no kernel is launched here).

- The C++ Grid (libes_host.so) reproduces the reference's Grid bit for bit
  (reference tests/sim/GridGenerationTests.h properties + the oracle + the
  reference's own CPU build via the committed fixture).
- libes_cuda.so / libes_host.so load and export every symbol include/*.h declares.
- Argument validation fails loudly before any device work.
"""
from __future__ import annotations

import re

import numpy as np
import pytest

import oracle_lib as O
from conftest import ROOT, gpu_available
from elasticscattering_b200 import EsError, Grid, GridInformation, SimulationCUDA, _native, workloads


def declared_symbols(header: str) -> list[str]:
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(es_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("header,loader", [("es_cuda.h", _native.cuda_lib), ("es_host.h", _native.host_lib)])
def test_library_exports_every_declared_symbol(header, loader):
    lib = loader()
    syms = declared_symbols(header)
    assert len(syms) >= 10
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_python_constants_match_header_enums():
    """Every ES_* enumerator and #define of include/es_cuda.h that the Python
    binding names has the header's value (batch modes, precisions, status codes)."""
    text = (ROOT / "include" / "es_cuda.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    values = {}
    for body in re.findall(r"enum\s+\w*\s*\{(.*?)\}", text, flags=re.S):
        nxt = 0
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            name, _, val = item.partition("=")
            nxt = int(val.strip(), 0) if val.strip() else nxt
            values[name.strip()] = nxt
            nxt += 1
    for name, val in re.findall(r"#define\s+(ES_[A-Z0-9_]+)\s+(-?\d+)", text):
        values[name] = int(val)
    checked = [n for n in values if hasattr(_native, n)]
    assert {"ES_BATCH_PASS_KERNELS", "ES_BATCH_PERSISTENT", "ES_PRECISION_SPLIT", "ES_OK"} <= set(checked)
    for n in checked:
        assert getattr(_native, n) == values[n], (n, getattr(_native, n), values[n])


def test_python_binding_declares_every_symbol():
    for header, api in (("es_cuda.h", _native.CUDA_API), ("es_host.h", _native.HOST_API)):
        assert set(declared_symbols(header)) == set(api), header


def test_grid_seeded_matches_oracle_and_reference_fixture(golden):
    w = workloads.config0()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    o = O.oracle_grid_seeded(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                             w.target_cell_population)
    assert np.array_equal(g.GetImpurities(), o.xy) and np.array_equal(g.GetIndex(), o.cell_end)
    ref = golden("ref_outputs.json")["config0_grid"]
    assert O.sha256(g.GetImpurities()) == ref["impurities_sha256"]
    assert O.sha256(g.GetIndex()) == ref["index_sha256"]
    assert g.GetUniqueImpurityCount() == ref["unique"] and g.GetCellsPerRow() == ref["cells_per_row"]
    s = g.GetSettings()
    assert (s.spawn_region_start, s.spawn_region_size, s.cells_per_row, s.impurity_radius) == \
        (o.settings.spawn_region_start, o.settings.spawn_region_size, o.settings.cells_per_row,
         o.settings.impurity_radius)
    assert s.cell_size == o.settings.cell_size


@pytest.mark.parametrize("name", ["test_impurities.npy", "real_case_impurities.npy", "test_impurities_lt.npy"])
def test_grid_from_list_matches_oracle(golden, name):
    xy = golden(name)
    for ext, ri, tcp in ((1e-7, 2e-9, 10), (1e-6, 1e-8, 10), (1e-7, 1.11e-9, 3)):
        g = Grid.from_list(xy, 1e-7, ext, ri, tcp)
        o = O.oracle_grid_list(xy, 1e-7, ext, ri, tcp)
        assert np.array_equal(g.GetImpurities(), o.xy) and np.array_equal(g.GetIndex(), o.cell_end)


@pytest.mark.parametrize("seed", [0, 1, 12345, 2 ** 31 + 7, 2 ** 32 - 1])
def test_grid_seed_int_conversion_matches_oracle(seed):
    # Grid::GenerateImpurities takes the seed through an int (reference src/sim/Grid.cpp:61).
    g = Grid.from_seed(seed, 1.0, 0.0, 1e3, 1e-3, 16)
    o = O.oracle_grid_seeded(seed, 1.0, 0.0, 1e3, 1e-3, 16)
    assert np.array_equal(g.GetImpurities(), o.xy)


def test_grid_generation_properties():
    """tests/sim/GridGenerationTests.h: monotone index, every impurity in its own or an
    overlapped cell, one cell holds all, diagonal duplication."""
    g = Grid.from_seed(0, 1.0, 0.0, 1e2, 1e-2, int(1e2 / 16))
    idx = g.GetIndex()
    assert np.all(np.diff(idx) >= 0)
    g4 = Grid.from_seed(0, 1.0, 0.0, 1e2, 1e-3, 4)
    assert len(g4.GetIndex()) == 25
    g1 = Grid.from_seed(0, 1.0, 0.0, 1e2, 1e-3, 101)
    assert list(g1.GetIndex()) == [100]
    for pos in ((0.5, 0.5), (0.505, 0.4999), (0.508, 0.4999), (0.492, 0.4999), (0.508, 0.501), (0.492, 0.501)):
        gd = Grid.from_list([pos, (0.1, 0.1), (0.9, 0.9), (0.9, 0.8)], 1, 0, 1e-2, 1)
        assert gd.GetCellsPerRow() == 2 and gd.GetTotalImpurityCount() == 7


def test_grid_arrays_point_at_the_grid_itself():
    """Grid.arrays(): the pointers es_upload_grid and es_batch_add_grid read in
    place hold what GetImpurities / GetIndex copy out, and stay the same pointers
    across calls (no copy is made)."""
    import ctypes as C

    g = Grid.from_seed(7, 1e-6, 3.8e-7, 5e15, 2e-9, 12)
    xy, n, idx = g.arrays()
    assert n == g.GetTotalImpurityCount() > 0
    cells = g.GetCellsPerRow() ** 2
    got_xy = np.ctypeslib.as_array(C.cast(xy, C.POINTER(C.c_double)), shape=(2 * n,))
    got_idx = np.ctypeslib.as_array(C.cast(idx, C.POINTER(C.c_int32)), shape=(cells,))
    assert np.array_equal(got_xy, g.GetImpurities().ravel())
    assert np.array_equal(got_idx, g.GetIndex())
    xy2, _, idx2 = g.arrays()
    assert xy2.value == xy.value and idx2.value == idx.value
    empty = Grid.from_list([], 1e-6, 0.0, 2e-9, 12)
    assert empty.arrays()[:2] == (None, 0)


def test_grid_config_errors_raise():
    with pytest.raises(EsError, match="Woah"):
        Grid.from_seed(1, 1e-5, 1e-5, 1e20, 2e-9, 10)
    with pytest.raises(EsError, match="No impurities"):
        Grid.from_seed(1, 1e-9, 0, 1.0, 2e-9, 10)


def test_create_validates_before_device_work():
    info = GridInformation(1e-6, 1e-7, 5e-8, 100, 100)
    with pytest.raises(EsError) as e:
        SimulationCUDA(64, 7, info)      # even dimension (src/SimulationConfiguration.h:154-155)
    assert e.value.status == 1
    with pytest.raises(EsError) as e:
        SimulationCUDA(65, 8, info)      # even phi_steps (src/SimulationConfiguration.h:151-152)
    assert e.value.status == 1


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    info = GridInformation(1e-6, 1e-7, 5e-8, 100, 100)
    with pytest.raises(EsError) as e:
        SimulationCUDA(65, 7, info)
    assert e.value.status == 5 and "device" in str(e.value).lower()


def test_fault_injection_plan_syntax():
    """es_fault_inject accepts "alloc|copy|launch:N[+]" items and rejects
    anything else without touching the armed plan; the counters start at zero
    with each call. No device is needed: the plan lives on the host."""
    for spec in ("alloc:1", "copy:3,launch:2+", " launch:10 , alloc:2+ ", "", None):
        _native.fault_inject(spec)
        assert _native.fault_counts() == {"alloc": 0, "copy": 0, "launch": 0, "failed": 0}
    for bad in ("alloc", "alloc:0", "alloc:-1", "free:1", "copy:x", "launch:1++", "copy:1,bogus"):
        with pytest.raises(EsError) as e:
            _native.fault_inject(bad)
        assert e.value.status == 1
    _native.fault_inject(None)


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_fault_injection_counts_nothing_without_a_device():
    """Argument and device checks come before the first counted operation."""
    _native.fault_inject("alloc:1")
    info = GridInformation(1e-6, 1e-7, 5e-8, 100, 100)
    with pytest.raises(EsError) as e:
        SimulationCUDA(65, 7, info)
    assert e.value.status == 5
    assert _native.fault_counts()["alloc"] == 0
    _native.fault_inject(None)
