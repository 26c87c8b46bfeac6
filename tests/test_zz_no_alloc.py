"""es_derive_temperatures_noalloc: stages (b)+(c) for callers that cannot allocate.

Callers that own all device memory through their own pool, or that run where a
driver allocation is not allowed, pass the lifetimes and the output as device
pointers; the entry point's scratch is a fixed array inside the library. This
file checks, through the C ABI, that two calls in a row give the sigmas of the
allocating entry point (es_derive_temperatures) within the sigma tolerance of the
parity tests, for both sectors, and that the size limit is enforced. It is
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


def test_noalloc_matches_allocating_entry_point_twice(cuda_device):
    import torch

    w = workloads.config0()
    grid = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                          w.target_cell_population)
    s = make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                      w.impurity_radius, w.target_cell_population)
    temps = np.array([1e-3, 1.0, 10.0, 40.0])
    lib = N.cuda_lib()
    with SimulationCUDA(w.dim, w.phi_steps, grid.info(), device=cuda_device) as sim:
        for coherent in (True, False):
            sim.InitSample(grid, s, coherent)
            for B in (20.0, 5.0):
                lifetimes, _ = sim.ComputeLifetimes(B)
                expected = sim.DeriveTemperatures(temps)
                d_lt = torch.from_numpy(lifetimes).to(f"cuda:{cuda_device}")
                for call in range(2):
                    d_out = torch.full((2 * len(temps),), float("nan"), dtype=torch.float64,
                                       device=f"cuda:{cuda_device}")
                    st = lib.es_derive_temperatures_noalloc(C.c_void_p(d_lt.data_ptr()), w.dim, w.phi_steps,
                                                            C.byref(s), int(coherent), B, temps.ctypes.data,
                                                            len(temps), C.c_void_p(d_out.data_ptr()), None)
                    N.check(st, None)
                    torch.cuda.synchronize()
                    got = d_out.cpu().numpy()
                    for t, e in enumerate(expected):
                        assert abs(got[2 * t] - e.xx) <= SIGMA_RTOL * abs(e.xx), (coherent, B, call, t)
                        assert abs(got[2 * t + 1] - e.xy) <= SIGMA_RTOL * abs(e.xy), (coherent, B, call, t)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda_device):
    import torch

    s = make_settings(1e-12, 0.3, True, 1.68e5, 1e-6, 1e-7, 1e15, 2e-9, 3)
    d = torch.zeros(4, dtype=torch.float64, device=f"cuda:{cuda_device}")
    temps = np.array([1.0])
    st = N.cuda_lib().es_derive_temperatures_noalloc(C.c_void_p(d.data_ptr()), 3, 1027, C.byref(s), 1, 20.0,
                                                     temps.ctypes.data, 1, C.c_void_p(d.data_ptr()), None)
    assert st == 1
    assert b"1025" in N.cuda_lib().es_last_error(None)
