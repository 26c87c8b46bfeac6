"""elasticscattering_b200 - B200-native (sm_100a) backend for ElasticScattering's
real-space conductivity path: per-orbit impurity-hit lifetimes, Simpson
integration over phase angle, Simpson reduction over the start-position grid to
sigma_xx and sigma_xy.

The compute lives in libes_cuda.so (CUDA kernels + the C ABI of
include/es_cuda.h); the impurity field and the .config runner live in
libes_host.so (include/es_host.h). This package binds both and mirrors the
reference's Simulation/Grid interface (simulation.py).
"""
from .simulation import (DeviceGrid, EsError, Grid, GridInformation, IterationResult, SampleMetrics, Settings, Sigma,
                         SimulationCUDA, make_settings)

__all__ = ["DeviceGrid", "EsError", "Grid", "GridInformation", "IterationResult", "SampleMetrics", "Settings", "Sigma",
           "SimulationCUDA", "make_settings"]
