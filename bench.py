#!/usr/bin/env python
"""Benchmark of the real-space conductivity path on B200.

Workload (one step): the config-1 sweep -- 257 x 257 start positions x 516
phases (34.08 M orbits per sector pass), density 5e15 m^-2, impurity radius
2e-9 m, B in {1, 5, 10, 20, 40} T, both sectors (coherent and incoherent), the
"T = 0" row (coherent tau = 1e-12 s, incoherent at 1e-3 K). One step = 10
sector passes = 340.8 M orbit lifetimes, then the phase and position Simpson
integrals (5 sigma(B) points).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs its own impurity sample (sample k =
rank), so per-GPU work is fixed (weak scaling); the one collective is an FP64
gather of the sample sigmas after the timed region. Prints ONE JSON line on rank 0.

`--impl reference` times the reference's own CPU implementation (its
SimulationCPU/Grid/es code built from its sources into oracle/_ref) on this
host's cores, on a bounded row sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from elasticscattering_b200 import workloads  # noqa: E402

METRIC = "orbit lifetimes/sec (sigma(B) points/sec reported alongside)"
UNIT = "lifetimes/s"
# Algorithmic FP64 operations per orbit, from a static count of the reference
# source (sqrt/div/floor/asin/cos/sin/exp count 1): particle creation (45),
# start-cell InsideImpurity test (7 each), GetNextCell step (237), CirclesCross
# test (11), GetFirstCrossTime on a crossing impurity (95).
FLOP_MODEL = {"per_orbit": 45, "per_start_test": 7, "per_cell": 237, "per_impurity_test": 11, "per_crossing": 95}
L2_FLUSH_BYTES = 256 << 20


def lifetime_flops(m: dict, n_orbits: int) -> float:
    return (FLOP_MODEL["per_orbit"] * n_orbits + FLOP_MODEL["per_start_test"] * m["start_cell_tests"]
            + FLOP_MODEL["per_cell"] * m["cells_passed"] + FLOP_MODEL["per_impurity_test"] * m["impurities_tested"]
            + FLOP_MODEL["per_crossing"] * m["crossings_tested"])


# ---------------------------------------------------------------- CPU side ---

def _ref_worker(args):
    """One host process: the reference's own CPU code on rows [j0, j1) of every
    (field, sector) pass of the workload. Returns (orbits, seconds)."""
    wname, sample, j0, j1 = args
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as O
    w = workloads.WORKLOADS[wname]()
    lib = O.ref()
    g = lib.ref_grid_new_seed(w.seed(sample), w.region_size, w.region_extends, w.density, w.impurity_radius,
                              w.target_cell_population)
    orbits, secs = 0, 0.0
    for coh in (1, 0):
        sim = lib.ref_sim_new(g, w.dim, w.phi_steps, w.tau, w.alpha, int(w.clockwise), w.particle_speed,
                              w.region_size, w.region_extends)
        lib.ref_sim_init_sample(sim, coh)
        for B in w.fields:
            t0 = time.perf_counter()
            orbits += lib.ref_sim_lifetimes_rows(sim, float(B), j0, j1, None, None)
            secs += time.perf_counter() - t0
        lib.ref_sim_free(sim)
    lib.ref_grid_free(g)
    return orbits, secs


def reference_cpu_sample(wname: str, rows_per_proc: int, procs: int) -> dict:
    """Times the reference CPU path on `procs` processes over disjoint row ranges."""
    w = workloads.WORKLOADS[wname]()
    jobs = []
    for p in range(procs):
        j0 = (p * w.dim) // procs
        jobs.append((wname, 0, j0, min(j0 + rows_per_proc, w.dim)))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, jobs)
    orbits = sum(r[0] for r in res)
    secs = max(r[1] for r in res)
    return {"orbits": orbits, "seconds": secs, "rate": orbits / secs, "procs": procs,
            "sample": f"{wname}: start-position rows [{jobs[0][2]},+{rows_per_proc}) per process x {procs} processes, "
                      f"all {len(w.fields)} fields x 2 sectors, reference SimulationCPU code (oracle/_ref)"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ref_so = ROOT / "oracle" / "_ref" / "libes_ref.so"
    if not ref_so.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libes_ref.so was not built here"}))
        return
    w = workloads.WORKLOADS[args.workload]()
    procs = os.cpu_count() or 1
    rows = max(1, args.ref_rows)
    for _ in range(args.warmup):  # untimed; one row per process
        reference_cpu_sample(args.workload, 1, procs)
    steps = []
    for _ in range(args.steps):
        steps.append(reference_cpu_sample(args.workload, rows, procs))
    orbits = sum(s["orbits"] for s in steps)
    secs = sum(s["seconds"] for s in steps)
    rate = orbits / secs
    per_point = 2 * w.orbits_per_pass / rate
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded impurity field)",
        "impl": "reference",
        "config": {"workload": w.name, "dim": w.dim, "phi_steps": w.phi_steps, "fields": w.fields,
                   "temperatures": w.temperatures, "sample": steps[0]["sample"]},
        "sigma_points_per_sec": 1.0 / per_point, "sigma_points_note": "lifetime stage only, extrapolated from the row sample",
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": procs, "kind": "reference", "sample": steps[0]["sample"]},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------- GPU side ---

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ["uuid", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap"]

    def __init__(self, uuid: str):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={','.join(self.FIELDS)}",
                                          "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) == len(self.FIELDS):
                    rows.append(parts)
        except OSError:
            pass
        finally:
            if self.path:
                Path(self.path).unlink(missing_ok=True)
        mine = [r for r in rows if self.uuid and self.uuid in r[0]] or rows
        if not mine:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in mine if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in mine if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in mine for k in range(4) if r[4 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(mine)}


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    from elasticscattering_b200 import Grid, SimulationCUDA, make_settings
    from elasticscattering_b200 import _native as N

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    w = workloads.WORKLOADS[args.workload]()

    # CPU baseline first (rank 0, one GPU only), before the GPU is touched.
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and (ROOT / "oracle/_ref/libes_ref.so").exists():
        cpu = reference_cpu_sample(args.workload, args.ref_rows, os.cpu_count() or 1)

    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    torch.cuda.set_device(local)
    dev = local

    grid = Grid.from_seed(w.seed(rank), w.region_size, w.region_extends, w.density, w.impurity_radius,
                          w.target_cell_population)
    settings = make_settings(w.tau, w.alpha, w.clockwise, w.particle_speed, w.region_size, w.region_extends,
                             w.density, w.impurity_radius, w.target_cell_population)
    sims = {}
    for coh in (True, False):
        s = SimulationCUDA(w.dim, w.phi_steps, grid.info(), device=dev)
        s.InitSample(grid, settings, coh)
        sims[coh] = s
    streams = {coh: torch.cuda.ExternalStream(s.stream_handle()) for coh, s in sims.items()}
    temps = np.array(w.temperatures, dtype=np.float64)
    n_t = len(temps)
    n_pass = len(w.fields) * 2
    out = torch.zeros((n_pass, 2 * n_t), dtype=torch.float64, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    main = torch.cuda.current_stream()

    def step():
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        flush.fill_(rank + 1)  # evict L2 before the step (inputs are 32 MB)
        ev0.record(main)
        for st in streams.values():
            st.wait_event(ev0)
        k = 0
        for B in w.fields:
            for coh, sim in sims.items():
                sim.enqueue_sigmas(float(B), temps, out[k].data_ptr())
                k += 1
        for st in streams.values():
            e = torch.cuda.Event()
            e.record(st)
            main.wait_event(e)
        ev1.record(main)
        return ev0, ev1

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    for s in sims.values():
        s.synchronize()
        s.read_metrics(reset=True)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = sum(s.launch_count() for s in sims.values())
    uuid = ""
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    events = []
    with ClockSampler(uuid) as clocks:
        for _ in range(args.steps):
            events.append(step())
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = sum(s.launch_count() for s in sims.values()) - launches0
    for s in sims.values():
        s.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in events]
    total_ms = float(sum(step_ms))
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    orbits_per_step = n_pass * w.orbits_per_pass
    value = world * args.steps * orbits_per_step / (total_ms * 1e-3)
    points_per_sec = world * args.steps * len(w.fields) * n_t / (total_ms * 1e-3)

    # Stage (a) alone, one launch per (field, sector): kernel time + algorithmic FLOPs.
    lt_ms, lt_flops = 0.0, 0.0
    per_field = []
    for B in w.fields:
        for coh, sim in sims.items():
            sim.read_metrics(reset=True)
            flush.fill_(3)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(streams[coh])
            N.check(N.cuda_lib().es_enqueue_lifetimes(sim.ctx, float(B)), sim.ctx)
            e1.record(streams[coh])
            sim.synchronize()
            ms = e0.elapsed_time(e1)
            m = sim.read_metrics(reset=True)
            fl = lifetime_flops(m, w.orbits_per_pass)
            lt_ms += ms
            lt_flops += fl
            per_field.append({"B": B, "coherent": coh, "ms": round(ms, 4),
                              "tflops": round(fl / (ms * 1e-3) / 1e12, 3),
                              "cells_per_orbit": round(m["cells_passed"] / w.orbits_per_pass, 3),
                              "imps_per_orbit": round(m["impurities_tested"] / w.orbits_per_pass, 3)})
    peak = C.c_double(0.0)
    N.check(N.cuda_lib().es_probe_fp64_fma(dev, C.byref(peak)))
    achieved = lt_flops / (lt_ms * 1e-3) / 1e12

    # End to end through the public API: host buffers, grid H2D every step,
    # blocking ComputeSigmas per (field, sector), sigma + metrics read back.
    xy = grid.GetImpurities()
    idx = grid.GetIndex()
    pin_xy = torch.from_numpy(xy.ravel()).pin_memory()
    pin_idx = torch.from_numpy(idx).pin_memory()
    isx = grid.GetSettings()
    host_out = np.zeros(2 * n_t)
    h2d = 2 * (pin_xy.numel() * 8 + pin_idx.numel() * 4)
    d2h = n_pass * (2 * n_t * 8 + 9 * 8 + 4)
    e2e_s = []
    for it in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for coh, sim in sims.items():
            N.check(N.cuda_lib().es_upload_grid(sim.ctx, C.c_void_p(pin_xy.data_ptr()), len(xy),
                                                C.c_void_p(pin_idx.data_ptr()), C.byref(isx), 0), sim.ctx)
        for B in w.fields:
            for coh, sim in sims.items():
                m = N.Metrics()
                N.check(N.cuda_lib().es_compute_sigmas(sim.ctx, float(B), temps.ctypes.data, n_t,
                                                       host_out.ctypes.data, C.byref(m)), sim.ctx)
        t1 = time.perf_counter()
        if it >= args.warmup:
            e2e_s.append(t1 - t0)
    e2e_t = torch.tensor([sum(e2e_s)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps * orbits_per_step / float(e2e_t.item())

    # The one collective: gather every rank's sample sigmas (FinishResults averages them).
    sig = out.clone()
    if world > 1:
        gathered = [torch.zeros_like(sig) for _ in range(world)]
        dist.all_gather(gathered, sig)
        dist.destroy_process_group()

    if rank != 0:
        return
    clk = clocks.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded impurity field; reference Grid RNG; one sample per GPU)",
        "config": {"workload": w.name, "dim": w.dim, "phi_steps": w.phi_steps, "fields": w.fields,
                   "temperatures": w.temperatures, "sectors": 2, "orbits_per_step_per_gpu": orbits_per_step,
                   "precision": "fp64 plain (reference semantics)",
                   "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write)"},
        "sigma_points_per_sec": points_per_sec,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                     "frac": achieved / peak.value if peak.value else None, "traffic": profiled_traffic(),
                     "kernel": "lifetime_fp64_kernel",
                     "peak_source": "measured in this run (es_probe_fp64_fma: FP64 FMA chains on every SM)",
                     "flop_model": FLOP_MODEL, "per_launch": per_field},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if cpu:
        line["cpu_baseline"] = {"value": cpu["rate"], "unit": UNIT, "cores": cpu["procs"], "kind": "reference",
                                "sample": cpu["sample"]}
    print(json.dumps(line))


def profiled_traffic():
    """DRAM bytes per lifetime launch from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "lifetime_fp64_config1.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="config1", choices=sorted(workloads.WORKLOADS))
    ap.add_argument("--ref-rows", type=int, default=2, help="start-position rows per CPU process")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
