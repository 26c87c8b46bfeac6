"""es_derive_temperatures_noalloc: stages (b)+(c) for callers that cannot allocate.

Callers that own all device memory through their own pool, or that run where a
driver allocation is not allowed, pass the lifetimes and the output as device
pointers; the entry point's scratch is a fixed array inside the library. This
file checks, through the C ABI, that two calls in a row give the sigmas of the
allocating entry point (es_derive_temperatures) within the sigma tolerance of the
parity tests, for both sectors, with more temperatures than one integration
group holds and at the stated maximum phi_steps, and that bad arguments and
sizes beyond the maximum are rejected before anything is enqueued. It is
collected last so that a run stopping at the first failure has run every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from elasticscattering_b200 import Grid, SimulationCUDA, make_settings, workloads
from elasticscattering_b200 import _native as N

pytestmark = pytest.mark.gpu

SIGMA_RTOL = 1e-9  # the sigma tolerance of tests/test_gpu_parity.py
MAX_PHI_STEPS = 1025  # the entry point's stated scratch maximum


def _noalloc(d_lt, dim, ppq, s, coherent, B, temps, d_out):
    temps = np.ascontiguousarray(temps, dtype=np.float64)
    return N.cuda_lib().es_derive_temperatures_noalloc(C.c_void_p(d_lt.data_ptr()), dim, ppq, C.byref(s),
                                                       int(coherent), B, temps.ctypes.data, len(temps),
                                                       C.c_void_p(d_out.data_ptr()), None)


def _check_against(expected, got, tag):
    for t, e in enumerate(expected):
        assert abs(got[2 * t] - e.xx) <= SIGMA_RTOL * abs(e.xx), (tag, t, got[2 * t], e.xx)
        assert abs(got[2 * t + 1] - e.xy) <= SIGMA_RTOL * abs(e.xy), (tag, t, got[2 * t + 1], e.xy)


def _setup(w):
    grid = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                          w.target_cell_population)
    s = make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                      w.impurity_radius, w.target_cell_population)
    return grid, s


def test_noalloc_matches_allocating_entry_point_twice(cuda_device):
    import torch

    w = workloads.config0()
    grid, s = _setup(w)
    # 11 temperatures: two integration groups (8 + 3), so the second group's
    # outputs land at an offset and the partial sums are reused between groups
    temps = np.array([1e-3, 1.0, 2.0, 4.0, 7.0, 10.0, 15.0, 20.0, 25.0, 30.0, 40.0])
    dev = f"cuda:{cuda_device}"
    with SimulationCUDA(w.dim, w.phi_steps, grid.info(), device=cuda_device) as sim:
        for coherent in (True, False):
            sim.InitSample(grid, s, coherent)
            for B in (20.0, 5.0):
                lifetimes, _ = sim.ComputeLifetimes(B)
                expected = sim.DeriveTemperatures(temps)
                d_lt = torch.from_numpy(lifetimes).to(dev)
                for call in range(2):
                    d_out = torch.full((2 * len(temps),), float("nan"), dtype=torch.float64, device=dev)
                    N.check(_noalloc(d_lt, w.dim, w.phi_steps, s, coherent, B, temps, d_out), None)
                    torch.cuda.synchronize()
                    _check_against(expected, d_out.cpu().numpy(), (coherent, B, call))


def test_noalloc_at_the_stated_maximum_phi_steps(cuda_device):
    """phi_steps = 1025 (4100 phases): the phase table fills the scratch array."""
    import torch

    w = workloads.config0()
    grid, s = _setup(w)
    dim, temps = 5, np.array([1.0, 10.0, 40.0])
    dev = f"cuda:{cuda_device}"
    with SimulationCUDA(dim, MAX_PHI_STEPS, grid.info(), device=cuda_device) as sim:
        for coherent in (True, False):
            sim.InitSample(grid, s, coherent)
            lifetimes, _ = sim.ComputeLifetimes(20.0)
            expected = sim.DeriveTemperatures(temps)
            d_lt = torch.from_numpy(lifetimes).to(dev)
            for call in range(2):
                d_out = torch.full((2 * len(temps),), float("nan"), dtype=torch.float64, device=dev)
                N.check(_noalloc(d_lt, dim, MAX_PHI_STEPS, s, coherent, 20.0, temps, d_out), None)
                torch.cuda.synchronize()
                _check_against(expected, d_out.cpu().numpy(), (coherent, call))


def test_noalloc_rejects_bad_arguments_before_enqueueing(cuda_device):
    import torch

    w = workloads.config0()
    _, s = _setup(w)
    dev = f"cuda:{cuda_device}"
    n = w.dim * w.dim * 4 * w.phi_steps
    d_lt = torch.zeros(n, dtype=torch.float64, device=dev)
    lib = N.cuda_lib()
    # incoherent sector, T = 0 in the second integration group: nothing of the
    # call (not even the first group) may have been enqueued
    temps = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0, 9.0, 0.0, 11.0])
    d_out = torch.full((2 * len(temps),), float("nan"), dtype=torch.float64, device=dev)
    assert _noalloc(d_lt, w.dim, w.phi_steps, s, False, 20.0, temps, d_out) == N.ES_ERR_BAD_ARG
    assert b"T > 0" in lib.es_last_error(None)
    torch.cuda.synchronize()
    assert torch.isnan(d_out).all()
    # no temperatures: success, nothing written
    d_out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    assert _noalloc(d_lt, w.dim, w.phi_steps, s, True, 20.0, np.zeros(0), d_out) == N.ES_OK
    torch.cuda.synchronize()
    assert torch.isnan(d_out).all()
    # beyond the fixed scratch
    assert _noalloc(d_lt, 3, MAX_PHI_STEPS + 2, s, True, 20.0, np.array([1.0]), d_out) == N.ES_ERR_BAD_ARG
    assert b"1025" in lib.es_last_error(None)
    # even sizes and a non-positive field
    assert _noalloc(d_lt, 4, w.phi_steps, s, True, 20.0, np.array([1.0]), d_out) == N.ES_ERR_BAD_ARG
    assert _noalloc(d_lt, w.dim, w.phi_steps, s, True, 0.0, np.array([1.0]), d_out) == N.ES_ERR_BAD_ARG
    torch.cuda.synchronize()
    assert torch.isnan(d_out).all()
