#!/usr/bin/env python
"""Benchmark of the real-space conductivity path on B200.

Workload (one step): the config-1 sweep -- 257 x 257 start positions x 516
phases (34.08 M orbits per sector pass), density 5e15 m^-2, impurity radius
2e-9 m, B in {1, 5, 10, 20, 40} T, both sectors (coherent and incoherent), the
"T = 0" row (coherent tau = 1e-12 s, incoherent at 1e-3 K). One step = 10
sector passes = 340.8 M orbit lifetimes, then the phase and position Simpson
integrals (5 sigma(B) points).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision split|fp64]

The headline `value` is the split-precision path (FP32 orbit stepping, FP64
winner times, guarded FP64 re-trace), whose lifetimes are compared with the
plain FP64 path every run (`split_vs_fp64`); the plain FP64 path is timed in
the same run and reported under `fp64_path`.

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
            "sample": f"{wname}: {rows_per_proc} start-position row(s) per process x {procs} processes "
                      f"(disjoint rows), all {len(w.fields)} fields x 2 sectors, reference SimulationCPU code "
                      f"(oracle/_ref)"}


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
        time.sleep(0.3)
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


class Sweep:
    """Both sector contexts of one precision, resident grid, device-timed steps."""

    def __init__(self, w, grid, settings, precision: int, device: int):
        import torch
        from elasticscattering_b200 import SimulationCUDA
        self.w = w
        self.sims = {}
        for coh in (True, False):
            s = SimulationCUDA(w.dim, w.phi_steps, grid.info(), device=device, precision=precision)
            s.InitSample(grid, settings, coh)
            self.sims[coh] = s
        self.streams = {coh: torch.cuda.ExternalStream(s.stream_handle()) for coh, s in self.sims.items()}
        self.temps = np.array(w.temperatures, dtype=np.float64)
        self.out = torch.zeros((len(w.fields) * 2, 2 * len(self.temps)), dtype=torch.float64, device="cuda")

    def step(self, flush, fill: int):
        """One sweep: every (field, sector) pass enqueued on the two context streams."""
        import torch
        main = torch.cuda.current_stream()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        flush.fill_(fill)  # evict L2 before the step (the grid is 37 MB)
        ev0.record(main)
        for st in self.streams.values():
            st.wait_event(ev0)
        k = 0
        for B in self.w.fields:
            for coh, sim in self.sims.items():
                sim.enqueue_sigmas(float(B), self.temps, self.out[k].data_ptr())
                k += 1
        for st in self.streams.values():
            e = torch.cuda.Event()
            e.record(st)
            main.wait_event(e)
        ev1.record(main)
        return ev0, ev1

    def launches(self) -> int:
        return sum(s.launch_count() for s in self.sims.values())

    def lifetime_kernel(self, flush, device: int) -> dict:
        """Stage (a) alone, one launch per (field, sector): time and algorithmic FLOPs."""
        import torch
        from elasticscattering_b200 import _native as N
        lt_ms, lt_flops, per, retraced = 0.0, 0.0, [], 0
        for B in self.w.fields:
            for coh, sim in self.sims.items():
                sim.read_metrics(reset=True)
                flush.fill_(3)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(self.streams[coh])
                N.check(N.cuda_lib().es_enqueue_lifetimes(sim.ctx, float(B)), sim.ctx)
                e1.record(self.streams[coh])
                sim.synchronize()
                ms = e0.elapsed_time(e1)
                m = sim.read_metrics(reset=True)
                fl = lifetime_flops(m, self.w.orbits_per_pass)
                lt_ms += ms
                lt_flops += fl
                retraced += m["retraced_fp64"]
                per.append({"B": B, "coherent": coh, "ms": round(ms, 4),
                            "alg_tflops": round(fl / (ms * 1e-3) / 1e12, 3),
                            "cells_per_orbit": round(m["cells_passed"] / self.w.orbits_per_pass, 3),
                            "imps_per_orbit": round(m["impurities_tested"] / self.w.orbits_per_pass, 3),
                            "retraced_fp64": m["retraced_fp64"]})
        return {"ms": lt_ms, "flops": lt_flops, "per_launch": per, "retraced_fp64": retraced}

    def close(self):
        for s in self.sims.values():
            s.close()


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    from elasticscattering_b200 import Grid, make_settings
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
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    n_t = len(w.temperatures)
    n_pass = len(w.fields) * 2
    orbits_per_step = n_pass * w.orbits_per_pass
    uuid = ""
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass

    precisions = {"split": N.ES_PRECISION_SPLIT, "fp64": N.ES_PRECISION_FP64}
    order = [args.precision] + [p for p in precisions if p != args.precision]
    res = {}
    lifetimes = {}
    for name in order:
        sw = Sweep(w, grid, settings, precisions[name], dev)
        for _ in range(args.warmup):
            sw.step(flush, rank + 1)
        torch.cuda.synchronize()
        for s in sw.sims.values():
            s.synchronize()
            s.read_metrics(reset=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = sw.launches()
        events = []
        with ClockSampler(uuid) as clocks:
            for _ in range(args.steps):
                events.append(sw.step(flush, rank + 1))
            torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        for s in sw.sims.values():
            s.synchronize()
        total_ms = float(sum(a.elapsed_time(b) for a, b in events))
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        r = {"total_ms": total_ms, "launches": sw.launches() - launches0, "clocks": clocks.summary(),
             "value": world * args.steps * orbits_per_step / (total_ms * 1e-3),
             "points_per_sec": world * args.steps * len(w.fields) * n_t / (total_ms * 1e-3),
             "sigma": sw.out.cpu().numpy().tolist()}
        lk = sw.lifetime_kernel(flush, dev)
        r["kernel"] = lk
        # one pass kept for the split-vs-fp64 comparison (B = 20 T, incoherent)
        lt, _ = sw.sims[False].ComputeLifetimes(20.0)
        lifetimes[name] = lt
        if name == args.precision:
            r["e2e"] = e2e_through_api(args, w, grid, sw, world, dist, N, torch)
        sw.close()
        res[name] = r

    peak64 = C.c_double(0.0)
    peak32 = C.c_double(0.0)
    N.check(N.cuda_lib().es_probe_fp64_fma(dev, C.byref(peak64)))
    N.check(N.cuda_lib().es_probe_fp32_fma(dev, C.byref(peak32)))
    a, b = lifetimes["fp64"], lifetimes["split"]
    nz = (a != 0) & (b != 0)
    split_vs = {"pass": "B=20 T incoherent", "orbits": int(a.size),
                "bit_identical_fraction": float((a.view(np.int64) == b.view(np.int64)).mean()),
                "hit_class_flips": int(((a == 0) != (b == 0)).sum()),
                "max_rel_lifetime_diff": float((np.abs(a[nz] - b[nz]) / np.abs(a[nz])).max()) if nz.any() else 0.0}
    sa, sb = np.array(res["fp64"]["sigma"]), np.array(res["split"]["sigma"])
    split_vs["max_rel_sigma_diff"] = float((np.abs(sa - sb) / np.maximum(np.abs(sa), 1e-300)).max())

    # The one collective: gather every rank's sample sigmas (FinishResults averages them).
    if world > 1:
        sig = torch.tensor(res[args.precision]["sigma"], dtype=torch.float64, device="cuda")
        gathered = [torch.zeros_like(sig) for _ in range(world)]
        dist.all_gather(gathered, sig)
        dist.destroy_process_group()
    if rank != 0:
        return

    def roofline(name, peak, bound, peak_src):
        k = res[name]["kernel"]
        achieved = k["flops"] / (k["ms"] * 1e-3) / 1e12
        return {"bound": bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None, "traffic": profiled_traffic(name),
                "kernel": "lifetime_split_kernel + lifetime_retrace_kernel" if name == "split" else "lifetime_fp64_kernel",
                "work": "algorithmic FP64-op count of the reference's TraceOrbit (flop_model) per launch",
                "peak_source": peak_src, "flop_model": FLOP_MODEL, "per_launch": k["per_launch"],
                "avg_launch_ms": k["ms"] / len(k["per_launch"]), "retraced_fp64": k["retraced_fp64"]}

    head = res[args.precision]
    other = "fp64" if args.precision == "split" else "split"
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 (split)" if args.precision == "split" else "f64",
        "data": "synthetic (seeded impurity field; reference Grid RNG; one sample per GPU)",
        "config": {"workload": w.name, "dim": w.dim, "phi_steps": w.phi_steps, "fields": w.fields,
                   "temperatures": w.temperatures, "sectors": 2, "orbits_per_step_per_gpu": orbits_per_step,
                   "precision": args.precision,
                   "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write)"},
        "sigma_points_per_sec": head["points_per_sec"],
        "roofline": roofline(args.precision, peak32.value if args.precision == "split" else peak64.value,
                             "fp32 pipe (bulk) + fp64" if args.precision == "split" else "fp64 pipe",
                             f"measured in this run (es_probe_{'fp32' if args.precision == 'split' else 'fp64'}_fma: "
                             f"FMA chains on every SM)"),
        "e2e": head["e2e"],
        "gpu_launches": head["launches"],
        "clocks": head["clocks"],
        f"{other}_path": {"value": res[other]["value"], "ms_per_step": res[other]["total_ms"] / args.steps,
                          "sigma_points_per_sec": res[other]["points_per_sec"], "gpu_launches": res[other]["launches"],
                          "clocks": res[other]["clocks"],
                          "roofline": roofline(other, peak64.value if other == "fp64" else peak32.value,
                                               "fp64 pipe" if other == "fp64" else "fp32 pipe (bulk) + fp64",
                                               "measured in this run (es_probe_*_fma)")},
        "split_vs_fp64": split_vs,
        "measured_peaks_tflops": {"fp64_fma": peak64.value, "fp32_fma": peak32.value},
    }
    if cpu:
        line["cpu_baseline"] = {"value": cpu["rate"], "unit": UNIT, "cores": cpu["procs"], "kind": "reference",
                                "sample": cpu["sample"]}
    print(json.dumps(line))


def e2e_through_api(args, w, grid, sw, world, dist, N, torch) -> dict:
    """The blocking public API per (field, sector): the grid uploaded from pinned
    host memory every step, sigma and metrics read back to the host."""
    xy = grid.GetImpurities()
    idx = grid.GetIndex()
    pin_xy = torch.from_numpy(xy.ravel()).pin_memory()
    pin_idx = torch.from_numpy(idx).pin_memory()
    isx = grid.GetSettings()
    temps = sw.temps
    n_t = len(temps)
    host_out = np.zeros(2 * n_t)
    n_pass = len(w.fields) * 2
    h2d = 2 * (pin_xy.numel() * 8 + pin_idx.numel() * 4)
    d2h = n_pass * (2 * n_t * 8 + C.sizeof(N.Metrics) + 4)
    times = []
    for it in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for coh, sim in sw.sims.items():
            N.check(N.cuda_lib().es_upload_grid(sim.ctx, C.c_void_p(pin_xy.data_ptr()), len(xy),
                                                C.c_void_p(pin_idx.data_ptr()), C.byref(isx), 0), sim.ctx)
        for B in w.fields:
            for coh, sim in sw.sims.items():
                m = N.Metrics()
                N.check(N.cuda_lib().es_compute_sigmas(sim.ctx, float(B), temps.ctypes.data, n_t,
                                                       host_out.ctypes.data, C.byref(m)), sim.ctx)
        t1 = time.perf_counter()
        if it >= args.warmup:
            times.append(t1 - t0)
    t = torch.tensor([sum(times)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    orbits_per_step = n_pass * w.orbits_per_pass
    return {"value": world * args.steps * orbits_per_step / float(t.item()), "unit": UNIT,
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}


def profiled_traffic(name: str):
    """DRAM bytes per lifetime launch from the committed ncu summary, if present."""
    p = ROOT / "profiles" / ("lifetime_split_config1.md" if name == "split" else "lifetime_fp64_config1.md")
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
    ap.add_argument("--precision", choices=["split", "fp64"], default="split")
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
