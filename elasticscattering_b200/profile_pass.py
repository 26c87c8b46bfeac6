"""One sector pass of a named workload, for profiling or timing a kernel.

    python -m elasticscattering_b200.profile_pass --workload config1 --field 20 --coherent 0 [--passes 1]
        [--variant V] [--time]
    python -m elasticscattering_b200.profile_pass --slice [--passes K]

Builds the workload's impurity field on the host, uploads it, and runs
`--passes` lifetime passes (stage a) followed by one integration (stages b, c),
then prints the pass metrics as JSON. Meant to run under
`ncu --clock-control none -k <kernel> -c 1` (the flag leaves the GPU clocks alone).
With --time, every pass is timed with CUDA events on the context stream and
each lifetime variant's lifetimes are compared bit for bit.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import Grid, SimulationCUDA, make_settings, workloads
from . import _native as N


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="config1", choices=sorted(workloads.WORKLOADS))
    ap.add_argument("--field", type=float, default=20.0)
    ap.add_argument("--coherent", type=int, default=0)
    ap.add_argument("--passes", type=int, default=1)
    ap.add_argument("--precision", type=int, default=None,
                    help="0 = plain FP64, 1 = FP32/FP64 split (default: FP64 per pass, split batched)")
    ap.add_argument("--variant", type=int, default=None, help="lifetime kernel variant (default: library default)")
    ap.add_argument("--time", action="store_true", help="time every variant with CUDA events")
    ap.add_argument("--compare-split", action="store_true", help="time plain FP64 against split precision")
    ap.add_argument("--batch", action="store_true",
                    help="run the pass through the batched kernel (one instance, fused integration)")
    ap.add_argument("--mode", type=int, default=N.ES_BATCH_PERSISTENT,
                    help="--batch: es_batch_mode (2 persistent, 3 single-pass kernels)")
    ap.add_argument("--slice", action="store_true",
                    help="the bench's step: the representative 3-sample slice of the 64-sample, 32-field sweep "
                         "(one 129^2, 257^2 and 513^2 sample; 192 passes) in one graph replay of the default "
                         "batch mode, --passes replays")
    ap.add_argument("--chunk-iters", type=int, default=32)
    ap.add_argument("--sweep-sample", type=int, default=None,
                    help="--batch: run sample K of the 64-sample batched sweep draw instead of --workload")
    ap.add_argument("--sweep-fields", type=int, default=2, help="--sweep-sample: fields uniformly spaced 1-40 T")
    ap.add_argument("--tcp", type=int, default=12, help="--sweep-sample: target cell population")
    a = ap.parse_args()
    if a.slice:
        batch_slice(a)
        return
    if a.compare_split:
        compare_split(a)
        return
    if a.batch and a.sweep_sample is not None:
        batch_sweep_sample(a)
        return
    if a.batch:
        batch_pass(a)
        return
    w = workloads.WORKLOADS[a.workload]()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    s = make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                      w.impurity_radius, w.target_cell_population)
    prec = N.ES_PRECISION_FP64 if a.precision is None else a.precision
    with SimulationCUDA(w.dim, w.phi_steps, g.info(), precision=prec) as sim:
        sim.InitSample(g, s, bool(a.coherent))
        if a.variant is not None:
            sim.set_tuning(lifetime_variant=a.variant)
        if a.time:
            import torch
            stream = torch.cuda.ExternalStream(sim.stream_handle())
            report = {}
            ref = None
            for variant in (0, 2, 6):
                sim.set_tuning(lifetime_variant=variant)
                ms = []
                for _ in range(a.passes + 1):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    N.check(N.cuda_lib().es_enqueue_lifetimes(sim.ctx, a.field), sim.ctx)
                    e1.record(stream)
                    sim.synchronize()
                    ms.append(e0.elapsed_time(e1))
                lt, m = sim.ComputeLifetimes(a.field)
                same = None if ref is None else bool(np.array_equal(ref.view(np.int64), lt.view(np.int64)))
                ref = lt if ref is None else ref
                report[f"variant{variant}"] = {"ms": [round(x, 3) for x in ms[1:]], "bitwise_equal_to_v0": same}
            print(json.dumps({"workload": w.name, "field": a.field, "coherent": a.coherent, "timing": report}))
            return
        for _ in range(a.passes):
            N.check(N.cuda_lib().es_enqueue_lifetimes(sim.ctx, a.field), sim.ctx)
        sim.synchronize()
        m = sim.read_metrics(reset=True)
        sig = sim.DeriveTemperatures(np.array(w.temperatures))
    print(json.dumps({"workload": w.name, "field": a.field, "coherent": a.coherent, "orbits": w.orbits_per_pass,
                      "metrics": m, "sigma": [(x.xx, x.xy) for x in sig]}))


def batch_pass(a) -> None:
    from .batch import BatchPass, BatchSweep
    w = workloads.WORKLOADS[a.workload]()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    s = make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                      w.impurity_radius, w.target_cell_population)
    prec = N.ES_PRECISION_SPLIT if a.precision is None else a.precision
    with BatchSweep(chunk_iters=a.chunk_iters, precision=prec, mode=a.mode) as b:
        gid = b.add_grid(g)
        b.set_passes([BatchPass(gid, w.dim, w.phi_steps, bool(a.coherent), w.region_size, g.info().cell_size,
                                a.field, s, list(w.temperatures))])
        ms = []
        for _ in range(a.passes):
            if a.time:
                import torch
                stream = torch.cuda.ExternalStream(b.stream_handle())
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                b.enqueue()
                e1.record(stream)
                out, m = b.collect()
                ms.append(round(e0.elapsed_time(e1), 3))
            else:
                out, m = b.run()
    print(json.dumps({"workload": w.name, "field": a.field, "coherent": a.coherent, "orbits": w.orbits_per_pass,
                      "batch": True, "ms": ms, "metrics": m[0], "sigma": out[0, :len(w.temperatures)].tolist()}))


def batch_sweep_sample(a) -> None:
    """One sample of the batched sweep (its drawn start grid and density), every
    field of --sweep-fields x both sectors x the sweep's temperatures, in one
    batched launch."""
    from .batch import BatchSweep, sweep_passes
    wl = workloads.config2(n_samples=64, n_fields=a.sweep_fields)
    smp = wl.samples[a.sweep_sample]
    g = Grid.from_seed(smp.seed, wl.region_size, wl.region_extends, smp.density, wl.impurity_radius, a.tcp)
    prec = N.ES_PRECISION_SPLIT if a.precision is None else a.precision
    with BatchSweep(chunk_iters=a.chunk_iters, precision=prec, mode=a.mode) as b:
        gid = b.add_grid(g)
        b.set_passes(sweep_passes(wl, {smp.index: gid}, {smp.index: g.info().cell_size}, samples=[smp]))
        ms = []
        for _ in range(a.passes):
            if a.time:
                import torch
                stream = torch.cuda.ExternalStream(b.stream_handle())
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                b.enqueue()
                e1.record(stream)
                out, m = b.collect()
                ms.append(round(e0.elapsed_time(e1), 3))
            else:
                out, m = b.run()
        orbits = b.total_orbits
    print(json.dumps({"workload": wl.name, "sample": a.sweep_sample, "dim": smp.dim, "density": smp.density,
                      "tcp": a.tcp, "fields": wl.fields, "orbits": orbits, "ms": ms,
                      "retraced_fp64": sum(x["retraced_fp64"] for x in m),
                      "impurities_tested": sum(x["impurities_tested"] for x in m),
                      "cells_passed": sum(x["cells_passed"] for x in m)}))


def batch_slice(a) -> None:
    """The bench's step (bench.py's default workload) with the library's default
    batch tuning and the reference's cell population: graph replays of the
    representative slice, each timed with CUDA events on the batch stream."""
    from .batch import BatchSweep, sweep_passes
    wl = workloads.representative_slice(workloads.config2(), 0)
    grids = {s.index: Grid.from_seed(s.seed, wl.region_size, wl.region_extends, s.density, wl.impurity_radius,
                                     wl.target_cell_population) for s in wl.samples}
    prec = N.ES_PRECISION_SPLIT if a.precision is None else a.precision
    with BatchSweep(precision=prec) as b:
        ids = {k: b.add_grid(g) for k, g in grids.items()}
        b.set_passes(sweep_passes(wl, ids, {k: g.info().cell_size for k, g in grids.items()}))
        import torch
        stream = torch.cuda.ExternalStream(b.stream_handle())
        ms = []
        for _ in range(a.passes):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.enqueue()
            e1.record(stream)
            out, m = b.collect()
            ms.append(round(e0.elapsed_time(e1), 3))
        orbits = b.total_orbits
    print(json.dumps({"workload": wl.name, "orbits": orbits, "passes": len(m), "ms": ms,
                      "retraced_fp64": sum(x["retraced_fp64"] for x in m),
                      "cells_passed": sum(x["cells_passed"] for x in m)}))


def compare_split(a) -> None:
    import torch
    w = workloads.WORKLOADS[a.workload]()
    g = Grid.from_seed(w.seed(0), w.region_size, w.region_extends, w.density, w.impurity_radius,
                       w.target_cell_population)
    s = make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends, w.density,
                      w.impurity_radius, w.target_cell_population)
    res = {}
    lts = {}
    for name, prec in (("fp64", N.ES_PRECISION_FP64), ("split", N.ES_PRECISION_SPLIT)):
        with SimulationCUDA(w.dim, w.phi_steps, g.info(), precision=prec) as sim:
            sim.InitSample(g, s, bool(a.coherent))
            stream = torch.cuda.ExternalStream(sim.stream_handle())
            ms = []
            for _ in range(a.passes + 1):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                N.check(N.cuda_lib().es_enqueue_lifetimes(sim.ctx, a.field), sim.ctx)
                e1.record(stream)
                sim.synchronize()
                ms.append(e0.elapsed_time(e1))
            sim.read_metrics(reset=True)
            lt, m = sim.ComputeLifetimes(a.field)
            lts[name] = lt
            res[name] = {"ms": [round(x, 3) for x in ms[1:]], "retraced": m["retraced_fp64"]}
    x, y = lts["fp64"], lts["split"]
    nz = (x != 0) & (y != 0)
    res["flips"] = int(((x == 0) != (y == 0)).sum())
    res["bit_identical"] = float((x.view(np.int64) == y.view(np.int64)).mean())
    res["max_rel"] = float((np.abs(x[nz] - y[nz]) / np.abs(x[nz])).max()) if nz.any() else 0.0
    print(json.dumps({"workload": w.name, "field": a.field, "coherent": a.coherent, "orbits": w.orbits_per_pass,
                      **res}))


if __name__ == "__main__":
    main()
