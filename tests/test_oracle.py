"""Pins the oracle (oracle/es_oracle.c) before the GPU tests trust it.

1. Known answers of the reference's unit tests (tests/es/*.h, tests/sim/SimpsonWeightsTest.h).
2. The reference's golden sigma tables (tests/sim/SigmaIntegrationTest.h:84-138) at the
   reference's own tolerance, 1e-5 / B relative (tests/TestMacros.h:17).
3. Bit-exact agreement with outputs of the reference's own CPU build, from the committed
   fixture (ref_outputs.json) and, where oracle/_ref exists, live on random configurations.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import oracle_lib as O
from elasticscattering_b200 import workloads

PI = 3.141592653589793238463
HALF_PI = 1.570796326794896619231
E = 1.60217646e-19
M = 5.0 * 9.10938188e-31


# ---- 1. geometry known answers (tests/es/AngleTests.h, OrbitDetailsTest.h) ----

@pytest.mark.parametrize("pos,cw,expected", [
    ((1, 0), True, HALF_PI), ((-1, 0), True, 3 * HALF_PI), ((0, 1), True, PI), ((0, -1), True, 0.0),
    ((-1, 0), False, HALF_PI), ((0, 1), False, 0.0), ((1, 0), False, 3 * HALF_PI), ((0, -1), False, PI),
])
def test_get_angle_unit_circle(pos, cw, expected):
    got = O.oracle().orc_get_angle(pos[0], pos[1], 0.0, 0.0, 1.0, int(cw))
    assert abs(got - expected) < 1e-6


def test_get_angle_offset_orbit():
    lib = O.oracle()
    assert abs(lib.orc_get_angle(5, 5, 6, 6, math.sqrt(2), 1) - 7 * PI / 4) < 1e-6
    assert abs(lib.orc_get_angle(5, 5, 6, 6, math.sqrt(2), 0) - 3 * PI / 4) < 1e-6


@pytest.mark.parametrize("phi,lo,hi,cw,expected", [
    (1, 0.5, 1.5, False, True), (1, 0.5, 1.5, True, False), (2, 0.5, 1.5, True, True),
    (0.1, 0.5, 1.5, True, True), (1, 1.5, 0.5, False, False), (1, 1.5, 0.5, True, True),
    (1, 1, 1, True, True), (2, 1, 1, True, True),
])
def test_angle_in_range(phi, lo, hi, cw, expected):
    assert bool(O.oracle().orc_angle_in_range(phi, lo, hi, int(cw))) == expected


def test_cross_angle():
    lib = O.oracle()
    assert lib.orc_cross_angle(6.1, 0.1, 1) == 6
    assert abs(lib.orc_cross_angle(6.1, 0.1, 0) - (2 * PI - 6.0)) < 1e-6


@pytest.mark.parametrize("phi,is_electron,is_future,expected", [
    (-0.25, False, True, 0.25), (-0.25, True, True, 0.75), (-0.25, True, False, 0.25), (-0.25, False, False, 0.75),
    (PI / 2 - 0.25, False, True, 0.25), (PI - 0.25, False, True, 0.25), (3 * PI / 2 - 0.25, False, True, 0.25),
    (0.5, False, True, 1.0), (0.5, False, False, 0.0),
])
def test_bound_time(phi, is_electron, is_future, expected):
    # The reference's tests pass (phi, w=0.5, alpha=1) into the (phi, alpha, w) slots.
    assert O.oracle().orc_bound_time(phi, 0.5, 1.0, 0, int(is_electron), int(is_future)) == expected


def test_circles_cross():
    lib = O.oracle()
    assert not lib.orc_circles_cross(1, 2, 1, 5, 5, 1)
    assert not lib.orc_circles_cross(1, 2, 1, 1, 3, 5)
    assert lib.orc_circles_cross(0, 0, 1, 0, 0.5, 0.6)
    assert lib.orc_circles_cross(0, 0, 1000, 2, 0, 1001)


def test_cross_time():
    lib = O.oracle()
    a1 = lib.orc_get_angle(3, 4, 0, 0, 5, 1)
    a2 = lib.orc_get_angle(3, 4, 0, 0, 5, 0)
    t = lib.orc_first_cross_time(0, 0, 5, 1, a1, 5, 0, 0.1, 2, 0, 0)
    t2 = lib.orc_first_cross_time(0, 0, 5, 0, a2, 5, 0, 0.1, 2, 0, 0)
    assert abs(t - 0.907 / 2) < 0.01
    assert abs(t + t2 - (2 * PI - 0.1 * 2.0 / 5) / 2) < 1e-6
    t = lib.orc_first_cross_time(0, 0, 5, 1, a1, 5, 0, 0.059, 100, 0, 0)
    t2 = lib.orc_first_cross_time(0, 0, 5, 0, a2, 5, 0, 0.059, 100, 0, 0)
    assert abs(t + t2 - (2 * PI - 0.059 * 2.0 / 5) / 100) < 1e-6


def test_simpson_weights():
    w = O.oracle().orc_simpson_weight
    assert [w(i, 7) for i in range(7)] == [1, 4, 2, 4, 2, 4, 1]
    assert w(1, 7) * w(1, 7) == 16 and w(1, 7) * w(2, 7) == 8


# ---- GetNextCell sequences (tests/es/GridMovementTests.h) ----

def walk_oracle(case, grid):
    lib = O.oracle()
    s = O.OrcIS()
    lo, hi = grid["spawn_range"]
    s.spawn_region_start, s.spawn_region_size, s.cells_per_row = lo, hi - lo, grid["cells_per_row"]
    s.cell_size = s.spawn_region_size / s.cells_per_row
    cur = np.array([*case["start_position"], case["start_angle"], 2 * PI, *case["start_cell"]], dtype=np.float64)
    out = []
    for _ in range(100):
        nxt = np.zeros(6)
        avail = lib.orc_next_cell(case["center"][0], case["center"][1], case["radius"], int(case["clockwise"]), 0.0,
                                  C.byref(s), cur.ctypes.data, nxt.ctypes.data)
        if not avail:
            break
        out.append(nxt.copy())
        cur = nxt
    return out


def test_grid_movement_known_answers(golden):
    gm = golden("grid_movement.json")
    for case in gm["cases"]:
        got = walk_oracle(case, gm["grid"])
        exp = case["expected_pos_x_pos_y_cell_x_cell_y_angle"]
        assert len(got) == len(exp), case["name"]
        for g, e in zip(got, exp):
            assert abs(g[0] - e[0]) < 1e-13 and abs(g[1] - e[1]) < 1e-13, case["name"]
            assert abs(g[2] - e[4]) < 1e-13, case["name"]
            assert (int(g[4]), int(g[5])) == (e[2], e[3]), case["name"]


# ---- TraceOrbit known answers (tests/es/LifetimeTests.h) ----

def lifetime_case_values(golden):
    lc = golden("lifetime_cases.json")
    imps = golden(lc["grid"]["impurities"])
    gd = lc["grid"]
    g = O.oracle_grid_list(imps, gd["region_size"], gd["region_extends"], gd["impurity_radius"],
                           gd["target_cell_population"])
    return lc, g


def check_lifetime(value, checks):
    for op, v in checks:
        if op == ">":
            assert value > v
        elif op == "<":
            assert value < v
        elif op == "==":
            assert value == v
        elif op == "almost":
            assert abs(value - v) < 1e-13


def test_lifetime_known_answers(golden):
    lc, g = lifetime_case_values(golden)
    xy = np.ascontiguousarray(g.xy)
    for c in lc["cases"]:
        st = lc["settings"][c["settings"]]
        combos = [(c["is_clockwise"], c["is_coherent"])] if c["is_clockwise"] is not None else \
            [(a, b) for a in (0, 1) for b in (0, 1)]
        for cw, coh in combos:
            lt = O.oracle().orc_trace_explicit(C.byref(g.settings), xy.ctypes.data, g.cell_end.ctypes.data, st["B"],
                                               c["position"][0], c["position"][1], c["q"], c["p"], 0.0,
                                               st["phi_step_size"], lc["common"]["alpha"],
                                               lc["common"]["particle_speed"], cw, coh)
            check_lifetime(E * st["B"] / M * lt, c["checks"])


# ---- 2. golden sigma tables ----

def golden_config(tables, key, golden):
    c = tables[key]["config"]
    xy = golden(tables[key]["impurities"])
    n_b = int(c["magnetic_field_n"])
    lo, hi = float(c["magnetic_field_min"]), float(c["magnetic_field_max"])
    fields = [lo + i * ((hi - lo) / (n_b - 1)) for i in range(n_b)]
    temps = [float(t) for t in c["temperatures"].split() if float(t) > 0]
    return c, xy, fields, temps


@pytest.mark.parametrize("key", ["file1", "file2"])
def test_oracle_matches_golden_sigma_tables(golden, key):
    tables = golden("sigma_tables.json")
    c, xy, fields, temps = golden_config(tables, key, golden)
    L, ext, ri, tcp = (float(c["region_size"]), float(c["region_extends"]), float(c["impurity_radius"]),
                       int(c["target_cell_population"]))
    g = O.oracle_grid_list(xy, L, ext, ri, tcp)
    dim, ppq = int(c["dimension"]), int(c["phi_steps"])
    args = (dim, ppq, L, float(c["particle_speed"]), float(c["alpha"]), float(c["tau"]), int(c["clockwise"]))
    rows = tables[key]["rows_T_B_cohxx_cohxy_incxx_incxy"]
    for bi, B in enumerate(fields):
        coh = O.oracle_sigmas(g, *args, True, B, temps)
        lt_inc, m = O.oracle_lifetimes(g, *args, False, B)
        assert m["particles_escaped"] == 0  # SigmaIntegrationTest.h:50-53
        inc = O.oracle_sigmas(g, *args, False, B, temps, lifetimes=lt_inc)
        for ti in range(len(temps)):
            row = rows[bi * len(temps) + ti]
            assert abs(row[1] - B) < 1e-13 and abs(row[0] - temps[ti]) < 1e-13
            tol = 1e-5 / B
            for got, exp in ((coh[ti][0], row[2]), (coh[ti][1], row[3]), (inc[ti][0], row[4]), (inc[ti][1], row[5])):
                assert abs((got - exp) / exp) < tol


# ---- 3. bit-exact against the reference's own CPU build ----

def ref_cases(golden):
    tables = golden("sigma_tables.json")
    out = golden("ref_outputs.json")
    for key in ("file1", "file2"):
        c, xy, fields, temps = golden_config(tables, key, golden)
        L, ext, ri, tcp = (float(c["region_size"]), float(c["region_extends"]), float(c["impurity_radius"]),
                           int(c["target_cell_population"]))
        g = O.oracle_grid_list(xy, L, ext, ri, tcp)
        args = (int(c["dimension"]), int(c["phi_steps"]), L, float(c["particle_speed"]), float(c["alpha"]),
                float(c["tau"]), int(c["clockwise"]))
        yield key, g, args, out[key]
    w = workloads.config0()
    g = O.oracle_grid_seeded(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                             w.target_cell_population)
    yield "config0", g, (w.dim, w.phi_steps, w.region_size, w.particle_speed, w.alpha, w.tau, int(w.clockwise)), \
        out["config0"]


def test_oracle_bit_exact_vs_reference_fixture(golden):
    for key, g, args, entries in ref_cases(golden):
        for e in entries:
            lt, m = O.oracle_lifetimes(g, *args, bool(e["coherent"]), e["B"])
            assert O.sha256(lt) == e["lifetimes_sha256"], (key, e["coherent"], e["B"])
            for k, v in e["metrics"].items():
                assert m[k] == v, (key, k)
            sig = O.oracle_sigmas(g, *args, bool(e["coherent"]), e["B"], e["temperatures"], lifetimes=lt)
            flat = [v for pair in sig for v in pair]
            assert ["%.17g" % v for v in flat] == e["sigma_xx_xy"], (key, e["coherent"], e["B"])


def test_oracle_grid_matches_reference_fixture(golden):
    ref = golden("ref_outputs.json")["config0_grid"]
    w = workloads.config0()
    g = O.oracle_grid_seeded(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                             w.target_cell_population)
    assert g.settings.cells_per_row == ref["cells_per_row"] and len(g.xy) == ref["indexed"]
    assert O.sha256(g.xy) == ref["impurities_sha256"] and O.sha256(g.cell_end) == ref["index_sha256"]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference tree absent)")
@pytest.mark.parametrize("seed", range(6))
def test_oracle_bit_exact_vs_live_reference(seed):
    """Random small configurations: the oracle and the reference's own CPU code agree bit for bit
    on the grid, every lifetime, every metric counter and the sigmas."""
    rng = np.random.default_rng(1000 + seed)
    L = 1e-6
    B = float(rng.uniform(2.0, 50.0))
    speed = 1.68e5
    ext = 2 * speed * M / (E * B) * float(rng.uniform(1.0, 1.5))
    density = float(10 ** rng.uniform(14.8, 16.0))
    ri = float(rng.choice([1e-9, 2e-9, 5e-9]))
    tcp = int(rng.integers(2, 20))
    dim = int(rng.choice([9, 15, 21]))
    ppq = int(rng.choice([3, 5, 7]))
    alpha = float(rng.choice([0.1, 0.3, PI / 4]))
    cw = int(rng.integers(0, 2))
    gseed = int(rng.integers(0, 2 ** 32))
    lib = O.ref()
    area = (L + 2 * ext) ** 2 * density
    if area > 1e7 or area < 1:
        pytest.skip("configuration outside the reference's Grid limits")
    gp = lib.ref_grid_new_seed(gseed, L, ext, density, ri, tcp)
    g = O.oracle_grid_seeded(gseed, L, ext, density, ri, tcp)
    cpr, tot, uniq = C.c_int(), C.c_int(), C.c_int()
    st, sz, cs, r = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    lib.ref_grid_info(gp, C.byref(cpr), C.byref(tot), C.byref(uniq), C.byref(st), C.byref(sz), C.byref(cs), C.byref(r))
    rxy = np.zeros(2 * tot.value)
    rce = np.zeros(cpr.value ** 2, dtype=np.int32)
    lib.ref_grid_copy(gp, rxy.ctypes.data, rce.ctypes.data)
    assert np.array_equal(rxy, g.xy.ravel()) and np.array_equal(rce, g.cell_end)
    temps = [0.5, 7.0]
    for coh in (1, 0):
        sim = lib.ref_sim_new(gp, dim, ppq, 1e-12, alpha, cw, speed, L, ext)
        lib.ref_sim_init_sample(sim, coh)
        n = dim * dim * 4 * ppq
        rlt = np.zeros(n)
        rm = np.zeros(7, dtype=np.int32)
        lib.ref_sim_lifetimes(sim, B, rlt.ctypes.data, rm.ctypes.data)
        olt, om = O.oracle_lifetimes(g, dim, ppq, L, speed, alpha, 1e-12, cw, coh, B)
        assert np.array_equal(rlt.view(np.int64), olt.view(np.int64))
        assert list(rm) == [om[k] for k in ("cells_passed", "impurities_tested", "particles_inside_impurity",
                                             "particles_escaped", "particles_at_bound", "max_impurities_tested",
                                             "max_cells_passed")]
        ts = np.array(temps)
        rs = np.zeros(4)
        lib.ref_sim_sigmas(sim, B, ts.ctypes.data, 2, rs.ctypes.data, None)
        os_ = O.oracle_sigmas(g, dim, ppq, L, speed, alpha, 1e-12, cw, coh, B, temps, lifetimes=olt)
        assert list(rs) == [v for p in os_ for v in p]
        # images path: per-position maps equal the reference's IntegratePosition
        ro, rl, rx, ry = np.zeros(2), np.zeros(dim * dim), np.zeros(dim * dim), np.zeros(dim * dim)
        lib.ref_sim_sigmas_images(sim, B, ts[:1].ctypes.data, 1, ro.ctypes.data, rl.ctypes.data, rx.ctypes.data,
                                  ry.ctypes.data)
        (ox, oy), ol, oxx, oxy = O.oracle_images(g, dim, ppq, L, speed, alpha, 1e-12, cw, coh, B, temps[0], olt)
        assert np.array_equal(rl, ol) and np.array_equal(rx, oxx) and np.array_equal(ry, oxy)
        assert (ro[0], ro[1]) == (ox, oy)
        lib.ref_sim_free(sim)
    lib.ref_grid_free(gp)
