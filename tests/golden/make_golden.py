"""Generates the committed golden fixtures of tests/golden/ from the reference.

Run here, where the reference tree and its CPU build (oracle/_ref, see
oracle/Makefile) exist:

    python tests/golden/make_golden.py REFERENCE_ROOT

REFERENCE_ROOT is the root of the reference's source tree (required).

It writes
  sigma_tables.json     the golden sigma rows of the reference's integration test
                        (tests/sim/SigmaIntegrationTest.h:84-138), read as text,
                        with the .config values they were made with
  *.npy                 the impurity lists those tests load (tests/data/*.dat)
  grid_movement.json    the GetNextCell crossing sequences (tests/es/GridMovementTests.h)
  lifetime_cases.json   the TraceOrbit known answers (tests/es/LifetimeTests.h)
  ref_outputs.json      outputs of the reference's own CPU code (oracle/_ref):
                        sigmas printed to 17 digits, lifetime SHA-256 digests and
                        metrics, for the golden configurations and config 0
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle_lib as O  # noqa: E402
from elasticscattering_b200 import workloads  # noqa: E402

NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"


def read_dat(path: Path) -> np.ndarray:
    """tests/TestUtils.h:13-44: skip '#' lines, two numbers split at the first space."""
    rows = []
    for line in path.read_text().splitlines():
        if not line or line[0] == "#" or line.startswith(":/"):
            continue
        pos = line.find(" ")
        rows.append((float(line[:pos]), float(line[pos + 1:])))
    return np.array(rows, dtype=np.float64)


def sigma_tables(ref_root: Path) -> dict:
    text = (ref_root / "tests/sim/SigmaIntegrationTest.h").read_text()
    row_re = re.compile(rf"DataRow\(\s*({NUM})\s*,\s*({NUM}),\s*Sigma\(\s*({NUM})\s*,\s*({NUM})\s*\),\s*"
                        rf"Sigma\(\s*({NUM})\s*,\s*({NUM})\s*\)\s*\)")
    f1 = text.index('SUBCASE("File 1")')
    f2 = text.index('SUBCASE("File 2")')
    out = {}
    for key, seg, cfg, imps in (("file1", text[f1:f2], "test_smaller_case.config", "test_impurities.dat"),
                                ("file2", text[f2:], "real_case.config", "real_case_impurities.dat")):
        rows = [[float(x) for x in m.groups()] for m in row_re.finditer(seg)]
        cfg_values = O.parse_config_text((ref_root / "tests/data" / cfg).read_text())
        out[key] = {"config": cfg_values, "impurities": imps.replace(".dat", ".npy"),
                    "rows_T_B_cohxx_cohxy_incxx_incxy": rows,
                    "source": "tests/sim/SigmaIntegrationTest.h", "tolerance": "rel < 1e-5 / B (tests/TestMacros.h:17)"}
    return out


def grid_movement(ref_root: Path) -> list:
    text = (ref_root / "tests/es/GridMovementTests.h").read_text()
    body = text[text.index('TEST_CASE("GetNextCell")'):]
    body = body[:body.index("/* Todo")]
    cases = []
    for block in re.split(r'SUBCASE\("', body)[1:]:
        name = block[:block.index('"')]
        m = re.search(rf"Orbit o\(\{{\s*({NUM})\s*,\s*({NUM})\s*\}},\s*({NUM}),\s*(true|false)\)", block)
        cx, cy, r, cw = float(m.group(1)), float(m.group(2)), float(m.group(3)), m.group(4) == "true"
        mp = re.search(rf"exit\.position = v2\(\s*({NUM})\s*,\s*({NUM})\s*\)", block)
        pos = (float(mp.group(1)), float(mp.group(2))) if mp else (0.0, 0.0)
        mc = re.search(r"exit\.entering_cell = \{\s*(\d+),\s*(\d+)\s*\}", block)
        ma = re.search(rf"exit\.incident_angle = ({NUM});", block)
        expected = [[float(a), float(b), int(c), int(d), float(e)] for a, b, c, d, e in re.findall(
            rf"Intersection\(\{{\s*({NUM})\s*,\s*({NUM})\s*\}},\s*\{{\s*(\d+),\s*(\d+)\s*\}},\s*({NUM})\)", block)]
        cases.append({"name": name, "center": [cx, cy], "radius": r, "clockwise": cw, "start_position": list(pos),
                      "start_cell": [int(mc.group(1)), int(mc.group(2))], "start_angle": float(ma.group(1)),
                      "expected_pos_x_pos_y_cell_x_cell_y_angle": expected})
    return {"grid": {"cells_per_row": 10, "spawn_range": [-1e-6, 2e-6]}, "phi": 0.0, "tolerance": 1e-13,
            "source": "tests/es/GridMovementTests.h", "cases": cases}


def lifetime_cases(ref_root: Path) -> dict:
    """tests/es/LifetimeTests.h: Grid(imps, 1e-6, 1e-6, 1e-8, 10) and ps/ps50/ps8."""
    text = (ref_root / "tests/es/LifetimeTests.h").read_text()
    cases = []
    for block in re.split(r'SUBCASE\("', text)[1:]:
        name = block[:block.index('"')]
        mcp = re.search(rf"CreateParticle\((\d+),\s*(\d+),\s*v2\(\s*({NUM})\s*,\s*({NUM})\s*\),\s*&(ps\w*)\)", block)
        var = mcp.group(5)
        sets = dict(re.findall(r"(ps\w*\.is_(?:clockwise|coherent))\s*=\s*(\d+);", block))
        checks = []
        for op, val in re.findall(rf"CHECK\(lt ([<>=]=?) ({NUM})\)", block):
            checks.append([op, float(val)])
        if re.search(r"CHECK_ALMOST\(lt, \(PI / 4\)\)", block):
            checks.append(["almost", 3.141592653589793238463 / 4])
        cw = sets.get(f"{var}.is_clockwise")
        coh = sets.get(f"{var}.is_coherent")
        cases.append({"name": name, "q": int(mcp.group(1)), "p": int(mcp.group(2)),
                      "position": [float(mcp.group(3)), float(mcp.group(4))], "settings": var,
                      "is_clockwise": None if cw is None else int(cw), "is_coherent": None if coh is None else int(coh),
                      "checks": checks})
    return {"grid": {"region_size": 1e-6, "region_extends": 1e-6, "impurity_radius": 1e-8,
                     "target_cell_population": 10, "impurities": "test_impurities_lt.npy"},
            "settings": {"ps": {"B": 10.0, "phi_step_size": 0.0}, "ps50": {"B": 50.0, "phi_step_size": 0.0},
                         "ps8": {"B": 8.0, "phi_step_size": 1.57079633e+00}},
            "common": {"alpha": 3.141592653589793238463 / 4.0, "particle_speed": 1.68e5, "phi_start": 0.0},
            "note": ("The reference's 'Edge case 1' sets ps.* but traces with ps8, whose is_clockwise and "
                     "is_coherent it never initialises; the fixture leaves them null."),
            "source": "tests/es/LifetimeTests.h", "cases": cases}


def ref_outputs(tables: dict, imps: dict) -> dict:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libes_ref.so is missing: run `make -C oracle` first")
    lib = O.ref()
    import ctypes as C
    res = {}

    def run(key, grid_ptr, dim, ppq, tau, alpha, cw, speed, L, ext, fields, temps):
        entry = []
        for coh in (1, 0):
            sim = lib.ref_sim_new(grid_ptr, dim, ppq, tau, alpha, cw, speed, L, ext)
            lib.ref_sim_init_sample(sim, coh)
            for B in fields:
                n = dim * dim * 4 * ppq
                lt = np.zeros(n)
                m = np.zeros(7, dtype=np.int32)
                lib.ref_sim_lifetimes(sim, float(B), lt.ctypes.data, m.ctypes.data)
                ts = np.array(temps, dtype=np.float64)
                out = np.zeros(2 * len(ts))
                lib.ref_sim_sigmas(sim, float(B), ts.ctypes.data, len(ts), out.ctypes.data, None)
                entry.append({"coherent": coh, "B": float(B), "temperatures": [float(t) for t in ts],
                              "sigma_xx_xy": ["%.17g" % v for v in out],
                              "lifetimes_sha256": O.sha256(lt), "zero_lifetimes": int((lt == 0).sum()),
                              "metrics": dict(zip(["cells_passed", "impurities_tested", "particles_inside_impurity",
                                                   "particles_escaped", "particles_at_bound",
                                                   "max_impurities_tested", "max_cells_passed"],
                                                  [int(x) for x in m]))})
            lib.ref_sim_free(sim)
        res[key] = entry

    for key in ("file1", "file2"):
        c = tables[key]["config"]
        xy = imps[tables[key]["impurities"]]
        L, ext, ri, tcp = float(c["region_size"]), float(c["region_extends"]), float(c["impurity_radius"]), int(c["target_cell_population"])
        g = lib.ref_grid_new_list(xy.ctypes.data, len(xy), L, ext, ri, tcp)
        n_b = int(c["magnetic_field_n"])
        lo, hi = float(c["magnetic_field_min"]), float(c["magnetic_field_max"])
        step = (hi - lo) / (n_b - 1)
        fields = [lo + i * step for i in range(n_b)]
        temps = [float(t) for t in c["temperatures"].split() if float(t) > 0]
        run(key, g, int(c["dimension"]), int(c["phi_steps"]), float(c["tau"]), float(c["alpha"]),
            int(c["clockwise"]), float(c["particle_speed"]), L, ext, fields, temps)
        lib.ref_grid_free(g)

    w = workloads.config0()
    g = lib.ref_grid_new_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                              w.target_cell_population)
    run("config0", g, w.dim, w.phi_steps, w.tau, w.alpha, int(w.clockwise), w.particle_speed, w.region_size,
        w.region_extends, w.fields + [5.0], w.temperatures + [1.0, 10.0])
    cpr, tot, uniq = C.c_int(), C.c_int(), C.c_int()
    st, sz, cs, r = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    lib.ref_grid_info(g, C.byref(cpr), C.byref(tot), C.byref(uniq), C.byref(st), C.byref(sz), C.byref(cs), C.byref(r))
    xy = np.zeros(2 * tot.value)
    ce = np.zeros(cpr.value ** 2, dtype=np.int32)
    lib.ref_grid_copy(g, xy.ctypes.data, ce.ctypes.data)
    res["config0_grid"] = {"seed": w.seed(0), "cells_per_row": cpr.value, "indexed": tot.value, "unique": uniq.value,
                           "impurities_sha256": O.sha256(xy), "index_sha256": O.sha256(ce)}
    lib.ref_grid_free(g)
    return res


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py REFERENCE_ROOT")
    ref_root = Path(sys.argv[1])
    imps = {}
    for name in ("test_impurities.dat", "real_case_impurities.dat", "test_impurities_lt.dat"):
        a = read_dat(ref_root / "tests/data" / name)
        np.save(HERE / name.replace(".dat", ".npy"), a)
        imps[name.replace(".dat", ".npy")] = a
    tables = sigma_tables(ref_root)
    (HERE / "sigma_tables.json").write_text(json.dumps(tables, indent=1))
    (HERE / "grid_movement.json").write_text(json.dumps(grid_movement(ref_root), indent=1))
    (HERE / "lifetime_cases.json").write_text(json.dumps(lifetime_cases(ref_root), indent=1))
    (HERE / "ref_outputs.json").write_text(json.dumps(ref_outputs(tables, imps), indent=1))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
