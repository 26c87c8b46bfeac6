"""Parity of the CUDA path (libes_cuda.so, called through its C ABI) with the oracle.

Bars (the parity target): the same hit/no-hit decision for every orbit, and sigma within
1e-9 relative of the reference's FP64 results on the same seeded inputs.
Per-orbit lifetimes are additionally held to 1e-9 relative (they differ from the
CPU only through the last bits of asin; the phase constants are tabulated with
the host libm).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from elasticscattering_b200 import EsError, Grid, SampleMetrics, SimulationCUDA, make_settings, workloads
from elasticscattering_b200 import _native as N

pytestmark = pytest.mark.gpu

SIGMA_RTOL = 1e-9      # plain-path sigma tolerance, relative
LIFETIME_RTOL = 1e-9   # per-orbit lifetime tolerance, relative
E = 1.60217646e-19
M = 5.0 * 9.10938188e-31


def classes(lt: np.ndarray, bound: np.ndarray | None) -> np.ndarray:
    """0 = no lifetime (start inside, escape, full circle), 1 = hit, 2 = clamped to the sector bound."""
    c = np.where(lt == 0, 0, 1)
    if bound is not None:
        c = np.where((lt != 0) & (lt == bound), 2, c)
    return c


def bound_times(w, coherent: bool, B: float) -> np.ndarray | None:
    if coherent:
        return None
    omega = E * B / M
    alpha = w.alpha
    ppq = w.phi_steps
    area = alpha * 2.0
    phi_start, step = -alpha, area / (ppq - 1)
    half_pi = 1.570796326794896619231
    out = []
    for q in range(4):
        for p in range(ppq):
            phi = phi_start + q * half_pi + p * step
            rem = (phi + alpha) - half_pi * np.floor((phi + alpha) / half_pi)
            dphi = rem if w.clockwise else (2.0 * alpha - rem)
            out.append(dphi / omega)
    return np.tile(np.array(out), w.dim * w.dim)


def settings_of(w):
    return make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends,
                         w.density, w.impurity_radius, w.target_cell_population)


def compare_lifetimes(gpu: np.ndarray, orc: np.ndarray, bound) -> dict:
    cg, co = classes(gpu, bound), classes(orc, bound)
    flips = int((cg != co).sum())
    nz = (orc != 0) & (cg == co)
    rel = np.abs(gpu[nz] - orc[nz]) / np.abs(orc[nz])
    return {"flips": flips, "max_rel": float(rel.max()) if rel.size else 0.0,
            "bit_identical": float((gpu.view(np.int64) == orc.view(np.int64)).mean())}


@pytest.fixture(scope="module")
def config0_setup(cuda_device):
    w = workloads.config0()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    og = O.oracle_grid_seeded(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                              w.target_cell_population)
    assert np.array_equal(g.GetImpurities(), og.xy)
    sim = SimulationCUDA(w.dim, w.phi_steps, g.info(), device=cuda_device)
    yield w, g, og, sim
    sim.close()


@pytest.mark.parametrize("coherent", [True, False])
@pytest.mark.parametrize("B", [20.0, 5.0])
def test_lifetimes_per_orbit_config0(config0_setup, coherent, B):
    w, g, og, sim = config0_setup
    sim.InitSample(g, settings_of(w), coherent)
    gpu, gm = sim.ComputeLifetimes(B)
    orc, om = O.oracle_lifetimes(og, w.dim, w.phi_steps, w.region_size, w.particle_speed, w.alpha, w.tau,
                                 w.clockwise, coherent, B)
    r = compare_lifetimes(gpu, orc, bound_times(w, coherent, B))
    assert r["flips"] == 0, r
    assert r["max_rel"] <= LIFETIME_RTOL, r
    for k in ("cells_passed", "impurities_tested", "particles_inside_impurity", "particles_escaped",
              "particles_at_bound", "max_impurities_tested", "max_cells_passed"):
        assert gm[k] == om[k], (k, gm[k], om[k])


def test_sigma_config0_vs_reference(config0_setup, golden):
    w, g, og, sim = config0_setup
    ref = golden("ref_outputs.json")["config0"]
    for e in ref:
        sim.InitSample(g, settings_of(w), bool(e["coherent"]))
        got = sim.ComputeSigmas(e["B"], e["temperatures"])
        exp = [float(v) for v in e["sigma_xx_xy"]]
        for t, s in enumerate(got):
            for a, b in ((s.xx, exp[2 * t]), (s.xy, exp[2 * t + 1])):
                assert abs(a - b) <= SIGMA_RTOL * abs(b), (e["coherent"], e["B"], a, b)


def golden_case(golden, key):
    tables = golden("sigma_tables.json")
    c = tables[key]["config"]
    xy = golden(tables[key]["impurities"])
    n_b = int(c["magnetic_field_n"])
    lo, hi = float(c["magnetic_field_min"]), float(c["magnetic_field_max"])
    fields = [lo + i * ((hi - lo) / (n_b - 1)) for i in range(n_b)]
    temps = [float(t) for t in c["temperatures"].split() if float(t) > 0]
    L, ext, ri, tcp = (float(c["region_size"]), float(c["region_extends"]), float(c["impurity_radius"]),
                       int(c["target_cell_population"]))
    g = Grid.from_list(xy, L, ext, ri, tcp)
    s = make_settings(float(c["tau"]), float(c["alpha"]), int(c["clockwise"]) > 0, float(c["particle_speed"]), L, ext,
                      float(c["impurity_density"]), ri, tcp)
    return c, g, s, fields, temps, tables[key]["rows_T_B_cohxx_cohxy_incxx_incxy"]


@pytest.mark.parametrize("key", ["file1", "file2"])
def test_sigma_golden_tables(cuda_device, golden, key):
    """The reference's integration test through the C ABI: golden rows at the reference's
    tolerance (1e-5 / B) and the reference's own CPU outputs at 1e-9."""
    c, g, s, fields, temps, rows = golden_case(golden, key)
    ref = golden("ref_outputs.json")[key]
    with SimulationCUDA(int(c["dimension"]), int(c["phi_steps"]), g.info(), device=cuda_device) as sim:
        res = {}
        for coh in (True, False):
            sim.InitSample(g, s, coh)
            for B in fields:
                metrics = SampleMetrics()
                res[(coh, B)] = sim.ComputeSigmas(B, temps, g, metrics)
                assert metrics.iteration_metrics[0]["particles_escaped"] == 0
        for bi, B in enumerate(fields):
            for ti in range(len(temps)):
                row = rows[bi * len(temps) + ti]
                coh, inc = res[(True, B)][ti], res[(False, B)][ti]
                for got, exp in ((coh.xx, row[2]), (coh.xy, row[3]), (inc.xx, row[4]), (inc.xy, row[5])):
                    assert abs((got - exp) / exp) < 1e-5 / B
        for e in ref:
            got = res[(bool(e["coherent"]), e["B"])]
            exp = [float(v) for v in e["sigma_xx_xy"]]
            for t, sg in enumerate(got):
                for a, b in ((sg.xx, exp[2 * t]), (sg.xy, exp[2 * t + 1])):
                    assert abs(a - b) <= SIGMA_RTOL * abs(b), (key, e["coherent"], e["B"], a, b)


def test_images_match_oracle(cuda_device, golden):
    """ComputeSigmasWithImages: the per-position maps of IntegratePosition, and its sigma
    equal to ComputeSigmas' within 1e-13 (the reference's own check,
    tests/sim/SigmaIntegrationTest.h:144-169; the two paths sum in different orders)."""
    c, g, s, fields, temps, _ = golden_case(golden, "file1")
    dim, ppq = int(c["dimension"]), int(c["phi_steps"])
    xy = golden("test_impurities.npy")
    og = O.oracle_grid_list(xy, float(c["region_size"]), float(c["region_extends"]), float(c["impurity_radius"]),
                            int(c["target_cell_population"]))
    with SimulationCUDA(dim, ppq, g.info(), device=cuda_device) as sim:
        for coh in (True, False):
            sim.InitSample(g, s, coh)
            B = fields[2]
            its = sim.ComputeSigmasWithImages(B, temps)
            plain = sim.ComputeSigmas(B, temps)
            lt, _ = O.oracle_lifetimes(og, dim, ppq, float(c["region_size"]), float(c["particle_speed"]),
                                       float(c["alpha"]), float(c["tau"]), int(c["clockwise"]), coh, B)
            for t, T in enumerate(temps):
                (ox, oy), ol, oxx, oxy = O.oracle_images(og, dim, ppq, float(c["region_size"]),
                                                         float(c["particle_speed"]), float(c["alpha"]),
                                                         float(c["tau"]), int(c["clockwise"]), coh, B, T, lt)
                for got, exp in ((its[t].particle_lifetimes, ol), (its[t].xx_buffer, oxx), (its[t].xy_buffer, oxy)):
                    scale = np.abs(exp).max()
                    assert np.allclose(got, exp, rtol=SIGMA_RTOL, atol=1e-12 * scale)
                assert abs(its[t].result.xx - plain[t].xx) <= 1e-13 * abs(plain[t].xx)
                assert abs(its[t].result.xy - plain[t].xy) <= 1e-13 * abs(plain[t].xy)
                assert abs(its[t].result.xx - ox) <= SIGMA_RTOL * abs(ox)


def test_grid_movement_on_device(cuda_device, golden):
    gm = golden("grid_movement.json")
    lo, hi = gm["grid"]["spawn_range"]
    s = N.ImpuritySettings(lo, hi - lo, (hi - lo) / gm["grid"]["cells_per_row"], gm["grid"]["cells_per_row"], 0.0)
    g = Grid.from_list([(0.5e-6, 0.5e-6)], 1e-6, 1e-6, 1e-9, 1)
    with SimulationCUDA(3, 3, g.info(), device=cuda_device) as sim:
        lib = N.cuda_lib()
        for case in gm["cases"]:
            cur = np.array([*case["start_position"], case["start_angle"], 2 * np.pi, *case["start_cell"]])
            got = []
            for _ in range(100):
                nxt = np.zeros(6)
                avail = C.c_int32()
                N.check(lib.es_debug_next_cell(sim.ctx, case["center"][0], case["center"][1], case["radius"],
                                               int(case["clockwise"]), 0.0, C.byref(s), cur.ctypes.data,
                                               nxt.ctypes.data, C.byref(avail)), sim.ctx)
                if not avail.value:
                    break
                got.append(nxt.copy())
                cur = nxt
            exp = case["expected_pos_x_pos_y_cell_x_cell_y_angle"]
            assert len(got) == len(exp), case["name"]
            for a, e in zip(got, exp):
                assert abs(a[0] - e[0]) < 1e-13 and abs(a[1] - e[1]) < 1e-13 and abs(a[2] - e[4]) < 1e-13
                assert (int(a[4]), int(a[5])) == (e[2], e[3])


def test_lifetime_known_answers_on_device(cuda_device, golden):
    lc = golden("lifetime_cases.json")
    gd = lc["grid"]
    g = Grid.from_list(golden(gd["impurities"]), gd["region_size"], gd["region_extends"], gd["impurity_radius"],
                       gd["target_cell_population"])
    with SimulationCUDA(3, 3, g.info(), device=cuda_device) as sim:
        sim.upload_grid(g)
        lib = N.cuda_lib()
        for c in lc["cases"]:
            st = lc["settings"][c["settings"]]
            combos = [(c["is_clockwise"], c["is_coherent"])] if c["is_clockwise"] is not None else \
                [(a, b) for a in (0, 1) for b in (0, 1)]
            for cw, coh in combos:
                out = C.c_double()
                N.check(lib.es_debug_trace(sim.ctx, c["position"][0], c["position"][1], c["q"], c["p"], st["B"], 0.0,
                                           st["phi_step_size"], lc["common"]["alpha"], lc["common"]["particle_speed"],
                                           cw, coh, C.byref(out)), sim.ctx)
                v = E * st["B"] / M * out.value
                for op, val in c["checks"]:
                    assert {"<": v < val, ">": v > val, "==": v == val, "almost": abs(v - val) < 1e-13}[op], \
                        (c["name"], v, op, val)


@pytest.mark.parametrize("coherent", [True, False])
def test_lifetime_variants_agree_bitwise(config0_setup, coherent):
    """The FP64 kernel's register budgets and its deferred crossing form run the
    same arithmetic: lifetimes and every metric counter are identical. Removed
    variant numbers are rejected."""
    w, g, og, sim = config0_setup
    sim.InitSample(g, settings_of(w), coherent)
    default = sim.get_tuning()
    runs = {}
    for variant in (0, 2, 6):
        sim.set_tuning(lifetime_variant=variant)
        runs[variant] = sim.ComputeLifetimes(5.0)
    for variant in (1, 3, 4, 5, 7, -1):
        with pytest.raises(EsError):
            sim.set_tuning(lifetime_variant=variant)
    sim.set_tuning(**default)
    for variant in (2, 6):
        assert np.array_equal(runs[0][0].view(np.int64), runs[variant][0].view(np.int64)), variant
        assert runs[0][1] == runs[variant][1], variant


def test_results_are_bit_reproducible(config0_setup):
    w, g, og, sim = config0_setup
    sim.InitSample(g, settings_of(w), False)
    a = sim.ComputeSigmas(20.0, [1e-3, 1.0, 10.0])
    b = sim.ComputeSigmas(20.0, [1e-3, 1.0, 10.0])
    assert [(s.xx, s.xy) for s in a] == [(s.xx, s.xy) for s in b]


def test_many_temperatures_span_groups(config0_setup):
    """More than one temperature group (8 per integration launch) gives the same values."""
    w, g, og, sim = config0_setup
    sim.InitSample(g, settings_of(w), False)
    temps = [0.5 + 0.7 * k for k in range(19)]
    many = sim.ComputeSigmas(20.0, temps)
    for k in (0, 8, 18):
        one = sim.ComputeSigmas(20.0, [temps[k]])[0]
        assert (one.xx, one.xy) == (many[k].xx, many[k].xy)


def test_enqueue_matches_blocking(config0_setup):
    import torch
    w, g, og, sim = config0_setup
    sim.InitSample(g, settings_of(w), True)
    ref = sim.ComputeSigmas(20.0, [1e-3])
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    sim.enqueue_sigmas(20.0, np.array([1e-3]), out.data_ptr())
    sim.synchronize()
    assert out.cpu().tolist() == [ref[0].xx, ref[0].xy]
    m = sim.read_metrics()
    assert m["cells_passed"] > 0


def test_error_paths(cuda_device):
    w = workloads.config0()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    with SimulationCUDA(w.dim, w.phi_steps, g.info(), device=cuda_device) as sim:
        with pytest.raises(EsError) as e:
            sim.ComputeSigmas(20.0, [1.0])
        assert e.value.status == 6  # no grid
        sim.upload_grid(g)
        with pytest.raises(EsError) as e:
            sim.ComputeSigmas(20.0, [1.0])
        assert e.value.status == 7  # no sample
        sim.InitSample(g, settings_of(w), False)
        with pytest.raises(EsError):
            sim.ComputeSigmas(0.0, [1.0])
        with pytest.raises(EsError):
            sim.ComputeSigmas(20.0, [0.0])  # incoherent tau = hbar / (k_B T) needs T > 0
        assert sim.ComputeSigmas(20.0, [1.0])[0].xx > 0  # the context stays usable
    # region_extends below the start-grid offset (0.01 cell): the last row of
    # start positions falls outside the impurity grid.
    small = Grid.from_seed(5, 1e-6, 1e-11, 1e15, 2e-9, 3)
    with SimulationCUDA(w.dim, w.phi_steps, small.info(), device=cuda_device) as sim:
        with pytest.raises(EsError, match="outside the impurity grid"):
            sim.InitSample(small, settings_of(w), True)


def test_config1_full_size_rows_and_properties(cuda_device):
    """Full config-1 size (257 x 257 x 516 = 34.08 M orbits per pass) at one field: parity on
    three start-position rows against the oracle, plus size-independent properties of the
    whole pass (no escapes, no negative lifetimes, incoherent lifetimes never past the bound,
    reproducible sigma)."""
    w = workloads.config1()
    B = 20.0
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    og = O.OracleGrid(g.GetImpurities(), g.GetIndex(), O.OrcIS(*[getattr(g.GetSettings(), f) for f, _ in
                                                                  N.ImpuritySettings._fields_]),
                      g.GetUniqueImpurityCount())
    per_row = w.dim * 4 * w.phi_steps
    with SimulationCUDA(w.dim, w.phi_steps, g.info(), device=cuda_device) as sim:
        for coh in (True, False):
            sim.InitSample(g, settings_of(w), coh)
            lt, m = sim.ComputeLifetimes(B)
            # The reference counts an orbit as escaped whenever GetNextCell makes no
            # progress (src/sim/es/cell_grid.h:177-180), e.g. grazing a cell edge, so
            # a handful occur at this size even with a large region extension.
            assert m["particles_escaped"] <= 1e-6 * w.orbits_per_pass and (lt >= 0).all()
            bt = bound_times(w, coh, B)
            if bt is not None:
                assert (lt <= bt).all()
            for j in (0, w.dim // 2, w.dim - 1):
                orc, _ = O.oracle_lifetimes(og, w.dim, w.phi_steps, w.region_size, w.particle_speed, w.alpha,
                                            w.tau, w.clockwise, coh, B, rows=(j, j + 1))
                part = lt[j * per_row:(j + 1) * per_row]
                r = compare_lifetimes(part, orc, None if bt is None else bt[j * per_row:(j + 1) * per_row])
                assert r["flips"] == 0 and r["max_rel"] <= LIFETIME_RTOL, (coh, j, r)
            a = sim.DeriveTemperatures([1e-3, 10.0])
            b = sim.DeriveTemperatures([1e-3, 10.0])
            assert [(s.xx, s.xy) for s in a] == [(s.xx, s.xy) for s in b]
            assert all(np.isfinite([s.xx, s.xy]).all() for s in a)
