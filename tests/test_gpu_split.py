"""Split precision (ES_PRECISION_SPLIT) against the plain FP64 path, through the C ABI.

North-star bar for the split path: sigma within 1e-6 relative of plain FP64, error stated
per result. The split kernel recomputes every winning crossing with the reference's FP64
arithmetic and re-traces in FP64 every orbit whose FP32 decisions lack margin, so the
tests also hold it to the plain path's per-orbit bars: the same hit/no-hit/at-bound class
for every orbit and lifetimes within 1e-9.
"""
from __future__ import annotations

import numpy as np
import pytest

from elasticscattering_b200 import Grid, SimulationCUDA, make_settings, workloads
from elasticscattering_b200 import _native as N

pytestmark = pytest.mark.gpu

SPLIT_SIGMA_RTOL = 1e-6
LIFETIME_RTOL = 1e-9


def settings_of(w):
    return make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends,
                         w.density, w.impurity_radius, w.target_cell_population)


def pair(w, grid, device):
    plain = SimulationCUDA(w.dim, w.phi_steps, grid.info(), device=device, precision=N.ES_PRECISION_FP64)
    split = SimulationCUDA(w.dim, w.phi_steps, grid.info(), device=device, precision=N.ES_PRECISION_SPLIT)
    return plain, split


def compare(a: np.ndarray, b: np.ndarray) -> dict:
    ca, cb = (a == 0), (b == 0)
    flips = int((ca != cb).sum())
    nz = ~ca & ~cb
    rel = np.abs(a[nz] - b[nz]) / np.abs(a[nz])
    return {"flips": flips, "max_rel": float(rel.max()) if rel.size else 0.0,
            "bit_identical": float((a.view(np.int64) == b.view(np.int64)).mean())}


@pytest.mark.parametrize("wname,fields", [("config0", (20.0, 5.0, 40.0)), ("config3", (40.0,))])
def test_split_matches_plain_per_orbit(cuda_device, wname, fields):
    w = workloads.WORKLOADS[wname]()
    if wname == "config3":
        w.dim, w.phi_steps = 129, 33  # the stress-case geometry at a test-sized start grid
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    plain, split = pair(w, g, cuda_device)
    try:
        for coherent in (True, False):
            plain.InitSample(g, settings_of(w), coherent)
            split.InitSample(g, settings_of(w), coherent)
            for B in fields:
                a, ma = plain.ComputeLifetimes(B)
                b, mb = split.ComputeLifetimes(B)
                r = compare(a, b)
                assert r["flips"] == 0 and r["max_rel"] <= LIFETIME_RTOL, (coherent, B, r, mb["retraced_fp64"])
                assert mb["retraced_fp64"] < 0.05 * len(a)
                for k in ("cells_passed", "impurities_tested", "crossings_tested", "particles_inside_impurity",
                          "particles_escaped", "particles_at_bound"):
                    assert ma[k] == mb[k], (coherent, B, k, ma[k], mb[k])
                temps = [1e-3, 10.0, 40.0]
                sa, sb = plain.DeriveTemperatures(temps), split.DeriveTemperatures(temps)
                for x, y in zip(sa, sb):
                    assert abs(x.xx - y.xx) <= SPLIT_SIGMA_RTOL * abs(x.xx)
                    assert abs(x.xy - y.xy) <= SPLIT_SIGMA_RTOL * abs(x.xy)
    finally:
        plain.close()
        split.close()


def test_split_config1_full_size(cuda_device):
    """config 1 at full size (34.08 M orbits per pass): every orbit compared with the plain path."""
    w = workloads.config1()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    plain, split = pair(w, g, cuda_device)
    try:
        for coherent in (True, False):
            plain.InitSample(g, settings_of(w), coherent)
            split.InitSample(g, settings_of(w), coherent)
            for B in (1.0, 20.0):
                a, _ = plain.ComputeLifetimes(B)
                b, mb = split.ComputeLifetimes(B)
                r = compare(a, b)
                assert r["flips"] == 0 and r["max_rel"] <= LIFETIME_RTOL, (coherent, B, r, mb["retraced_fp64"])
                sa = plain.DeriveTemperatures([1e-3])[0]
                sb = split.DeriveTemperatures([1e-3])[0]
                assert abs(sa.xx - sb.xx) <= SPLIT_SIGMA_RTOL * abs(sa.xx)
                assert abs(sa.xy - sb.xy) <= SPLIT_SIGMA_RTOL * abs(sa.xy)
    finally:
        plain.close()
        split.close()


# (sample, sector, field index) of config-2 passes where the reference's own
# rounding decides orbits: found by scanning split against plain FP64.
REFERENCE_ROUNDING_CASES = [
    # a vertical cell edge within ~1e-14 m of the orbit centre's x: the reference's
    # GetAngle takes asin of a ratio that rounds past -1, gets NaN and drops that
    # edge crossing, so the walk stops (an escape, lifetime 0)
    (2, False, 3), (2, False, 6),
    # an exit point within 1e-7 L of a perpendicular edge while the orbit runs almost
    # parallel to it: GetNextCell's corner rule moves diagonally and the walk
    # doubles back on itself
    (0, True, 24), (2, False, 25), (2, True, 22),
]


@pytest.mark.parametrize("sample,coherent,field_index", REFERENCE_ROUNDING_CASES)
def test_split_reproduces_reference_rounding_cases(cuda_device, sample, coherent, field_index):
    """Config-2 passes (513^2 starts, 7-9e15 m^-2, cells of target population 8)
    that contain orbits decided by the reference's rounding: the split path must
    hand them to the FP64 re-trace, so every lifetime equals the plain path's,
    bit for bit, and so do the walk metrics."""
    wl = workloads.config2(n_samples=64)
    s = wl.samples[sample]
    B = wl.fields[field_index]
    g = Grid.from_seed(s.seed, wl.region_size, wl.region_extends, s.density, wl.impurity_radius, 8)
    st = make_settings(wl.tau, wl.alpha, wl.clockwise, wl.particle_speed, wl.region_size, wl.region_extends,
                       s.density, wl.impurity_radius, 8)
    plain = SimulationCUDA(s.dim, wl.phi_steps, g.info(), device=cuda_device, precision=N.ES_PRECISION_FP64)
    split = SimulationCUDA(s.dim, wl.phi_steps, g.info(), device=cuda_device, precision=N.ES_PRECISION_SPLIT)
    try:
        plain.InitSample(g, st, coherent)
        split.InitSample(g, st, coherent)
        a, ma = plain.ComputeLifetimes(B)
        b, mb = split.ComputeLifetimes(B)
        r = compare(a, b)
        assert r["bit_identical"] == 1.0, (B, r, mb["retraced_fp64"])
        for k in ("cells_passed", "impurities_tested", "particles_inside_impurity", "particles_escaped",
                  "particles_at_bound"):
            assert ma[k] == mb[k], (B, k, ma[k], mb[k])
    finally:
        plain.close()
        split.close()


def test_split_images_and_fp32_integration(cuda_device):
    """Split contexts integrate in FP32 (FP64 sums): sigma and the per-position
    maps of ComputeSigmasWithImages stay within the split bar of the plain path;
    the lifetime map (no GetSigma) is the plain one."""
    w = workloads.config0()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    plain, split = pair(w, g, cuda_device)
    temps = [1e-3, 4.0, 40.0]
    try:
        for coherent in (True, False):
            plain.InitSample(g, settings_of(w), coherent)
            split.InitSample(g, settings_of(w), coherent)
            for B in (2.0, 20.0):
                a = plain.ComputeSigmasWithImages(B, temps)
                b = split.ComputeSigmasWithImages(B, temps)
                for x, y in zip(a, b):
                    assert abs(x.result.xx - y.result.xx) <= SPLIT_SIGMA_RTOL * abs(x.result.xx)
                    assert abs(x.result.xy - y.result.xy) <= SPLIT_SIGMA_RTOL * abs(x.result.xy)
                    assert np.array_equal(x.particle_lifetimes, y.particle_lifetimes)
                    for u, v in ((x.xx_buffer, y.xx_buffer), (x.xy_buffer, y.xy_buffer)):
                        assert np.abs(u - v).max() <= SPLIT_SIGMA_RTOL * np.abs(u).max()
    finally:
        plain.close()
        split.close()


def test_split_exact_sigma_equals_fp64(cuda_device):
    """ES_PRECISION_SPLIT_EXACT: the split walk (lifetimes the FP64 walk's bit for
    bit) with the FP64 integration gives the plain FP64 path's sigma and
    per-position maps bit for bit, at B = 1 and 20 T, both sectors, three
    temperatures; the counters are equal apart from the re-trace count."""
    w = workloads.config1()
    dim = 129
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    s = make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                      w.impurity_radius, w.target_cell_population)
    temps = [1e-3, 10.0, 40.0]
    keys = ("cells_passed", "impurities_tested", "particles_inside_impurity", "particles_escaped",
            "particles_at_bound", "max_cells_passed", "max_impurities_tested")
    with SimulationCUDA(dim, w.phi_steps, g.info(), device=cuda_device, precision=N.ES_PRECISION_FP64) as plain, \
            SimulationCUDA(dim, w.phi_steps, g.info(), device=cuda_device,
                           precision=N.ES_PRECISION_SPLIT_EXACT) as exact:
        for coh in (True, False):
            plain.InitSample(g, s, coh)
            exact.InitSample(g, s, coh)
            for B in (1.0, 20.0):
                lp, mp = plain.ComputeLifetimes(B)
                le, me = exact.ComputeLifetimes(B)
                assert np.array_equal(lp.view(np.int64), le.view(np.int64)), (coh, B)
                assert all(mp[k] == me[k] for k in keys), (coh, B)
                sp, se = plain.DeriveTemperatures(temps), exact.DeriveTemperatures(temps)
                assert [(x.xx, x.xy) for x in sp] == [(x.xx, x.xy) for x in se], (coh, B)
                ip, ie = plain.ComputeSigmasWithImages(B, temps), exact.ComputeSigmasWithImages(B, temps)
                for a, b in zip(ip, ie):
                    assert np.array_equal(a.particle_lifetimes, b.particle_lifetimes)
                    assert np.array_equal(a.xx_buffer, b.xx_buffer) and np.array_equal(a.xy_buffer, b.xy_buffer)


@pytest.mark.parametrize("every", [5, 13])  # the re-trace list holds a quarter of the pass
def test_finish_retrace_keeps_lifetimes_and_counters(cuda_device, every):
    """The finish kernel hands a winner whose crossing point the reference drops
    (NaN) to the FP64 re-trace, which subtracts the walk's counters of that orbit
    before adding its own. es_debug_finish_retrace forces that path for the hit
    of every `every`-th orbit on a long-walk (config-1) grid: the lifetimes must
    stay bit-identical and every counter but retraced_fp64 unchanged, with more
    orbits re-traced."""
    w = workloads.config1()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    lib = N.cuda_lib()
    with SimulationCUDA(65, 33, g.info(), device=cuda_device, precision=N.ES_PRECISION_SPLIT) as sim:
        assert lib.es_debug_finish_retrace(sim.ctx, -1) == N.ES_ERR_BAD_ARG
        for coherent in (True, False):
            sim.InitSample(g, settings_of(w), coherent)
            for B in (1.0, 20.0):
                N.check(lib.es_debug_finish_retrace(sim.ctx, 0), sim.ctx)
                ref, mref = sim.ComputeLifetimes(B)
                N.check(lib.es_debug_finish_retrace(sim.ctx, every), sim.ctx)
                got, mgot = sim.ComputeLifetimes(B)
                assert np.array_equal(ref.view(np.int64), got.view(np.int64)), (coherent, B)
                for k in mref:
                    if k != "retraced_fp64":
                        assert mgot[k] == mref[k], (coherent, B, k, mgot[k], mref[k])
                assert mgot["retraced_fp64"] > mref["retraced_fp64"]
        N.check(lib.es_debug_finish_retrace(sim.ctx, 0), sim.ctx)
