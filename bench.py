#!/usr/bin/env python
"""Benchmark of the real-space conductivity path on B200.

Default workload (--workload config2): the batched sigma(B) sweep -- 64
impurity samples x 32 fields uniformly spaced 1-40 T x T in {0, 10, 40} K, per
sample a start grid of 129^2, 257^2 or 513^2 positions and a density drawn
log-uniformly from 1e15-1e16 m^-2 (draw seed 12345), 516 phases, both sectors.
One step = one CUDA-graph replay of this GPU's slice of the sweep: one sample
of each start grid (the draw picks each with probability 1/3, so the slice is
three average samples), all 32 fields and 3 temperatures: 192 sector passes,
11.4 G orbit lifetimes, 288 sigma(B) points, on the FP32/FP64 split path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload config2|config1|...]

The line also carries: the same passes in FP64 (the split path's error per
result), the plain per-pass FP64 GPU path on the same passes (the stated
20x bar for the batched split path), stages (b)+(c) against HBM, the full 64-sample sweep timed once, the
config-1 sweep (257^2 x 516 orbits, 5 fields), the public API end to end, and
the reference's own CPU code on a bounded sample of the slice.

Under torchrun (N > 1) rank r runs the r-th slice (weak scaling; the full sweep
is split by LPT on estimated cost). Prints ONE JSON line on rank 0.

`--impl reference` times the reference's own CPU implementation (its
SimulationCPU/Grid/es code built from its sources into oracle/_ref) on this
host's cores, on a bounded row sample of the same slice.
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


def _ref_worker_pass(p: dict):
    """One host process: the reference's CPU code on rows [j0, j1) of the given
    (sample, field, sector) passes. Returns (orbits, seconds)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as O
    lib = O.ref()
    g = lib.ref_grid_new_seed(p["seed"], p["L"], p["ext"], p["density"], p["r"], p["tcp"])
    orbits, secs = 0, 0.0
    for coh in (1, 0):
        sim = lib.ref_sim_new(g, p["dim"], p["ppq"], p["tau"], p["alpha"], int(p["cw"]), p["speed"], p["L"], p["ext"])
        lib.ref_sim_init_sample(sim, coh)
        for B in p["fields"]:
            t0 = time.perf_counter()
            orbits += lib.ref_sim_lifetimes_rows(sim, float(B), p["j0"], p["j1"], None, None)
            secs += time.perf_counter() - t0
        lib.ref_sim_free(sim)
    lib.ref_grid_free(g)
    return orbits, secs


def reference_cpu_batched(wl, tcp_for, procs: int, rows: int = 2) -> dict:
    """The reference CPU path on a bounded sample of a batched sweep: process k
    takes start-position rows of sample k (mod the sample count) at the sweep's
    smallest, middle and largest field, both sectors -- `rows` rows of a 513^2
    sample, proportionally more of a smaller one, so every process does about the
    same number of orbits."""
    fields = sorted(wl.fields)
    pick = [fields[0], fields[len(fields) // 2], fields[-1]]
    big = max(s.dim for s in wl.samples)
    jobs = []
    for k in range(procs):
        s = wl.samples[k % len(wl.samples)]
        n = max(1, min(s.dim, round(rows * big / s.dim)))
        j0 = (k * 7919) % (s.dim - n + 1)
        jobs.append({"seed": s.seed, "L": wl.region_size, "ext": wl.region_extends, "density": s.density,
                     "r": wl.impurity_radius, "tcp": tcp_for(s.density), "dim": s.dim, "ppq": wl.phi_steps,
                     "tau": wl.tau, "alpha": wl.alpha, "cw": wl.clockwise, "speed": wl.particle_speed,
                     "fields": pick, "j0": j0, "j1": j0 + n})
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker_pass, jobs)
    orbits = sum(r[0] for r in res)
    secs = max(r[1] for r in res)
    return {"orbits": orbits, "seconds": secs, "rate": orbits / secs, "procs": procs,
            "sample": f"{wl.name}: {rows} start-position row(s) of a {big}^2 sample per process (proportionally "
                      f"more of smaller ones) x {procs} processes over the slice's samples, fields {pick} x 2 "
                      f"sectors, reference SimulationCPU code (oracle/_ref)"}


def run_reference_batched(args) -> None:
    """Reference arm of the batched sweep: its CPU code on bounded row samples of
    the same slice, at the reference's own target_cell_population."""
    wl = batch_workload(args, 0, 1)
    procs = os.cpu_count() or 1
    tcp = lambda d: wl.target_cell_population  # noqa: E731  (the reference's config value)
    for _ in range(args.warmup):
        reference_cpu_batched(wl, tcp, procs, 1)
    steps = [reference_cpu_batched(wl, tcp, procs, args.ref_rows) for _ in range(args.steps)]
    orbits = sum(s["orbits"] for s in steps)
    secs = sum(s["seconds"] for s in steps)
    rate = orbits / secs
    orbits_per_point = wl.orbits / max(1, wl.sigma_points)
    print(json.dumps({
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
        "data": "synthetic (seeded impurity fields; per-sample start grid and density drawn with seed 12345)",
        "config": {"workload": wl.name, "sample": steps[0]["sample"]},
        "sigma_points_per_sec": rate / orbits_per_point,
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": procs, "kind": "reference", "sample": steps[0]["sample"]},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ref_so = ROOT / "oracle" / "_ref" / "libes_ref.so"
    if not ref_so.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libes_ref.so was not built here"}))
        return
    if args.workload == "config2":
        run_reference_batched(args)
        return
    if args.workload == "config4":
        print(json.dumps({"impl": "reference", "unavailable": "config 4 is the learned surrogate, which has no "
                          "reference counterpart; the reference's CPU cost per sigma point is in the config-1 and "
                          "config-2 lines"}))
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
    check_field = 20.0 if 20.0 in w.fields else float(w.fields[-1])
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
        # one pass kept for the split-vs-fp64 comparison (B = 20 T where the sweep has it, incoherent)
        lt, _ = sw.sims[False].ComputeLifetimes(check_field)
        lifetimes[name] = lt
        if name == args.precision:
            r["e2e"] = e2e_through_api(args, w, grid, sw, world, dist, N, torch)
        sw.close()
        res[name] = r

    # The same sweep through the batched path: the 10 passes in one graph replay,
    # integration fused into the lifetime kernel, split precision.
    from elasticscattering_b200.batch import BatchPass, BatchSweep
    bsw = BatchSweep(dev, precision=N.ES_PRECISION_SPLIT)
    gid = bsw.add_grid(grid)
    bsw.set_passes([BatchPass(gid, w.dim, w.phi_steps, coh, w.region_size, grid.info().cell_size, float(B), settings,
                              list(w.temperatures)) for B in w.fields for coh in (True, False)])
    bstream = torch.cuda.ExternalStream(bsw.stream_handle())
    for _ in range(args.warmup):
        bsw.run(with_metrics=False)
    bms = []
    for _ in range(args.steps):
        flush.fill_(7)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(bstream)
        bsw.enqueue()
        e1.record(bstream)
        bout, _ = bsw.collect(with_metrics=False)
        bms.append(e0.elapsed_time(e1))
    bsw.close()
    b_sig = bout[:, :n_t, :].reshape(len(w.fields) * 2, 2 * n_t)
    f_sig = np.array(res["fp64"]["sigma"])
    batched = {"ms_per_step": float(np.mean(bms)), "value": orbits_per_step / (float(np.mean(bms)) * 1e-3),
               "sigma_points_per_sec": len(w.fields) * n_t / (float(np.mean(bms)) * 1e-3),
               "max_rel_sigma_vs_fp64": float((np.abs(b_sig - f_sig) / np.abs(f_sig)).max()),
               "note": "es_batch in its default mode (ES_BATCH_PASS_KERNELS: the single-pass kernels for each "
                       "pass in turn), one graph replay per step"}

    peak64 = C.c_double(0.0)
    peak32 = C.c_double(0.0)
    N.check(N.cuda_lib().es_probe_fp64_fma(dev, C.byref(peak64)))
    N.check(N.cuda_lib().es_probe_fp32_fma(dev, C.byref(peak32)))
    a, b = lifetimes["fp64"], lifetimes["split"]
    nz = (a != 0) & (b != 0)
    split_vs = {"pass": f"B={check_field:g} T incoherent", "orbits": int(a.size),
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
                "frac": achieved / peak if peak else None, "traffic": profiled_traffic(name, w.orbits_per_pass),
                "kernel": ("lifetime_split_kernel + lifetime_finish_kernel + lifetime_retrace_kernel" if name == "split"
                           else "lifetime_fp64_kernel"),
                "work": "algorithmic FP64-op count of the reference's TraceOrbit (flop_model) per launch",
                "peak_source": peak_src, "flop_model": FLOP_MODEL, "per_launch": k["per_launch"],
                "avg_launch_ms": k["ms"] / len(k["per_launch"]), "retraced_fp64": k["retraced_fp64"],
                "issue": profiled_issue(name)}

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
        "batched_path": batched,
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


def measured_peak(key: str, fallback: float, unit: str) -> tuple:
    """A peak from MEASURED_PEAKS.json (driver-written, measured on this pool's
    B200s), else the stated fallback measurement."""
    try:
        v = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())[key])
        return v, f"of measured (MEASURED_PEAKS.json {key})"
    except Exception:
        return fallback, f"of fallback ({fallback:g} {unit}; MEASURED_PEAKS.json absent)"


def batch_workload(args, rank: int, world: int):
    """The per-GPU slice of the 64-sample, 32-field sweep: by default the
    representative slice (one 129^2, one 257^2 and one 513^2 sample; rank r takes
    the r-th of each), with --samples N the first N samples per rank."""
    full = workloads.config2(n_fields=args.fields)
    if args.samples > 0:
        return workloads.shard_samples(workloads.config2(n_samples=max(64, args.samples * world), n_fields=args.fields),
                                       rank, world, args.samples)
    return workloads.representative_slice(full, rank)


def integrate_roofline(wl, s, tcp_for, dev, flush, torch, N) -> dict:
    """Stages (b)+(c) alone (es_enqueue_derive_temperatures on resident lifetimes),
    timed with CUDA events on the context stream, on the largest pass of the
    slice (513^2 x 516 orbits, 1.09 GB of FP64 lifetimes: larger than L2, and L2
    is flushed before every launch). Algorithmic bytes per launch: the 8-byte
    lifetimes read once (the partial sums are a few KB)."""
    from elasticscattering_b200 import Grid, SimulationCUDA, make_settings
    from elasticscattering_b200.batch import incoherent_temperature
    g = Grid.from_seed(s.seed, wl.region_size, wl.region_extends, s.density, wl.impurity_radius, tcp_for(s.density))
    st = make_settings(wl.tau, wl.alpha, wl.clockwise, wl.particle_speed, wl.region_size, wl.region_extends,
                       s.density, wl.impurity_radius, tcp_for(s.density))
    temps = np.array([incoherent_temperature(t) for t in wl.temperatures])
    B = float(wl.fields[len(wl.fields) // 2])
    peak, src = measured_peak("hbm_gbs", 6650.0, "GB/s")
    out = {}
    d_out = torch.zeros(2 * len(temps), dtype=torch.float64, device="cuda")
    for name, prec in (("split", N.ES_PRECISION_SPLIT), ("fp64", N.ES_PRECISION_FP64)):
        with SimulationCUDA(s.dim, wl.phi_steps, g.info(), device=dev, precision=prec) as sim:
            sim.InitSample(g, st, False)
            sim.ComputeLifetimes(B, copy=False)
            stream = torch.cuda.ExternalStream(sim.stream_handle())
            per = {}
            for nt in (1, len(temps)):
                ms = []
                for it in range(8):
                    flush.fill_(it)
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    sim.enqueue_derive_temperatures(temps[:nt], d_out.data_ptr())
                    e1.record(stream)
                    sim.synchronize()
                    if it >= 2:
                        ms.append(e0.elapsed_time(e1))
                per[nt] = float(np.mean(ms))
            n = sim.n_orbits
        bytes_alg = 8.0 * n
        achieved = bytes_alg / (per[1] * 1e-3) / 1e9
        out[name] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": src, "avg_launch_ms": per[1], "ms_at_all_temperatures": per[len(temps)],
                     "temperatures_at_once": len(temps),
                     "traffic": profiled_traffic(f"integrate_flat_{name}_config1.md", n),
                     "kernel": "integrate_flat_kernel + reduce_partials_kernel",
                     "work": f"{bytes_alg:.4g} algorithmic bytes per launch (8-byte lifetimes of one "
                             f"{s.dim}^2 x {4 * wl.phi_steps}-orbit pass, one temperature)"}
    return out


def run_batched(args) -> None:
    """The batched sweep (config 2): samples x fields x temperatures with per-sample
    start grids and densities, one graph replay per step, autotuned cell sizes and
    launch shape. A step is one graph replay of this GPU's slice of the sweep
    (default: one sample of each start grid, all 32 fields, T in {0, 10, 40} K,
    both sectors: 192 passes, 11.4 G orbits). Reports, besides the split path's
    throughput: the FP64 batch of the same passes (the per-result error), the
    plain per-pass FP64 GPU path on the same work (the stated 20x bar),
    stages (b)+(c) against HBM, the full 64-sample sweep timed once (split over
    the GPUs by LPT on estimated cost), the config-1 sweep, and the reference
    CPU code on a bounded sample of the slice."""
    import torch
    import torch.distributed as dist
    from concurrent.futures import ThreadPoolExecutor

    from elasticscattering_b200 import DeviceGrid, Grid, SimulationCUDA, autotune, make_settings
    from elasticscattering_b200 import _native as N
    from elasticscattering_b200.batch import (BatchSweep, finish_results, gather_sweep, incoherent_temperature,
                                              per_sample_sigmas, sweep_passes)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = local
    wl = batch_workload(args, rank, world)

    t_tune = time.perf_counter()
    tune = autotune.tune_sweep(wl, device=dev, cache=args.tune_cache, force=args.retune)
    tune_wall = time.perf_counter() - t_tune
    tcp_for = tune.tcp_for

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and (ROOT / "oracle/_ref/libes_ref.so").exists():
        cpu = reference_cpu_batched(wl, tcp_for, os.cpu_count() or 1, args.ref_rows)

    def build(s):
        return Grid.from_seed(s.seed, wl.region_size, wl.region_extends, s.density, wl.impurity_radius,
                              tcp_for(s.density))

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:
        grids = list(ex.map(build, wl.samples))
    grid_build_s = time.perf_counter() - t0
    cell = {s.index: g.info().cell_size for s, g in zip(wl.samples, grids)}
    uuid = ""
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    bs = BatchSweep(dev, precision=N.ES_PRECISION_SPLIT, **tune.shape)
    ids = {s.index: bs.add_grid(g) for s, g in zip(wl.samples, grids)}
    passes = sweep_passes(wl, ids, cell)
    bs.set_passes(passes)
    n_pass = len(passes)
    stream = torch.cuda.ExternalStream(bs.stream_handle())
    for _ in range(args.warmup):
        bs.run(with_metrics=False)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = bs.launch_count()
    ms = []
    with ClockSampler(uuid) as clocks:
        for it in range(args.steps):
            flush.fill_(it & 0xFF)  # evict L2 between steps
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            bs.enqueue()
            e1.record(stream)
            out_split, mets = bs.collect()
            ms.append(e0.elapsed_time(e1))
    graph_replays = bs.launch_count() - launches0
    total_ms = float(sum(ms))
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    step_ms = total_ms / args.steps
    orbits = bs.total_orbits
    nt = len(wl.temperatures)
    points = len(wl.samples) * len(wl.fields) * nt
    # counted from the recorded graph: per pass the orbit table, the lifetime walk,
    # the winners' FP64 finish (long-walk passes), the FP64 re-trace, integration
    # and reduction; or the persistent kernel and its FP64 re-trace
    kernels_per_replay = bs.graph_kernels()
    alg_flops = sum(lifetime_flops(m, 0) for m in mets) + FLOP_MODEL["per_orbit"] * orbits
    retraced = sum(m["retraced_fp64"] for m in mets)

    # the FP64 batch of the same passes: per-result error of the split path
    bs.set_tuning(precision=N.ES_PRECISION_FP64)
    bs.run(with_metrics=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    bs.enqueue()
    e1.record(stream)
    out_fp64, mets64 = bs.collect()
    fp64_batch_ms = e0.elapsed_time(e1)
    # the split walk with the FP64 integration: the FP64 batch's sigma bit for bit
    exact = None
    if tune.shape["mode"] == N.ES_BATCH_PASS_KERNELS:
        bs.set_tuning(precision=N.ES_PRECISION_SPLIT_EXACT)
        bs.run(with_metrics=False)
        flush.fill_(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bs.enqueue()
        e1.record(stream)
        out_exact, _ = bs.collect()
        exact_ms = e0.elapsed_time(e1)
        exact = {"ms_per_replay": exact_ms, "lifetimes_per_sec": bs.total_orbits / (exact_ms * 1e-3),
                 "sigma_points_per_sec": len(wl.samples) * len(wl.fields) * len(wl.temperatures) / (exact_ms * 1e-3),
                 "sigma_bit_identical_to_fp64_batch": bool(np.array_equal(out_exact, out_fp64)),
                 "fp64_batch_ms": fp64_batch_ms,
                 "note": "ES_PRECISION_SPLIT_EXACT: the split walk (lifetimes the FP64 walk's bit for bit) with the "
                         "FP64 integration, one replay of the same passes"}
    bs.close()
    a, b = out_split[:, :nt, :], out_fp64[:, :nt, :]
    rel = np.abs(a - b) / np.abs(b)
    # sigma(B) points: coherent + incoherent per (sample, field, temperature)
    pa, pb = a[0::2] + a[1::2], b[0::2] + b[1::2]
    prel = np.abs(pa - pb) / np.abs(pb)
    metrics_equal = all(x[k] == y[k] for x, y in zip(mets, mets64)
                        for k in ("cells_passed", "impurities_tested", "particles_inside_impurity",
                                  "particles_escaped", "particles_at_bound"))

    # the plain per-pass FP64 GPU path (one blocking ComputeSigmas per pass, the
    # reference's call pattern) on the same passes
    temps = [incoherent_temperature(x) for x in wl.temperatures]
    torch.cuda.synchronize()
    t_plain = time.perf_counter()
    worst_vs_plain = 0.0
    k = 0
    for s, g in zip(wl.samples, grids):
        st = next(p.settings for p in passes if p.grid == ids[s.index])
        sims = {coh: SimulationCUDA(s.dim, wl.phi_steps, g.info(), device=dev, precision=N.ES_PRECISION_FP64)
                for coh in (True, False)}
        for coh, sim in sims.items():
            sim.InitSample(g, st, coh)
        for B in wl.fields:
            for coh in (True, False):
                sig = sims[coh].ComputeSigmas(float(B), temps)
                for ti, sg in enumerate(sig):
                    for c, v in enumerate((sg.xx, sg.xy)):
                        worst_vs_plain = max(worst_vs_plain, abs(out_split[k, ti, c] - v) / abs(v))
                k += 1
        for sim in sims.values():
            sim.close()
    plain_s = time.perf_counter() - t_plain
    plain_pps = points / plain_s

    # stages (b)+(c) against HBM
    big = max(wl.samples, key=lambda x: x.dim)
    integ = integrate_roofline(wl, big, tcp_for, dev, flush, torch, N)

    # end to end through the public API with host buffers: each step copies the
    # host grids in, replays and reads sigma and metrics back
    e2e_steps = max(1, min(args.steps, 3))
    be = BatchSweep(dev, precision=N.ES_PRECISION_SPLIT, **tune.shape)
    e2e_times = []
    for it in range(e2e_steps + 1):
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t_e = time.perf_counter()
        be.clear()
        eid = {s.index: be.add_grid(g) for s, g in zip(wl.samples, grids)}
        be.set_passes(sweep_passes(wl, eid, cell))
        out_e2e, _ = be.run(with_metrics=True)
        if it > 0:  # the first call records the graph
            e2e_times.append(time.perf_counter() - t_e)
    be.close()
    e2e_t = torch.tensor([sum(e2e_times)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_s = float(e2e_t.item()) / e2e_steps
    h2d = sum(g.GetTotalImpurityCount() * 16 + g.GetCellsPerRow() ** 2 * 4 for g in grids)
    d2h = n_pass * (N.ES_BATCH_MAX_T * 2 * 8 + 10 * 8)

    # end to end from the sweep's seeds: every sample's grid built on the GPU
    # (bit-identical to the host Grid), then the same run and readback
    torch.cuda.synchronize()
    t_seed = time.perf_counter()
    bd = BatchSweep(dev, precision=N.ES_PRECISION_SPLIT, **tune.shape)
    did = {}
    for s in wl.samples:
        dg = DeviceGrid.from_seed(s.seed, wl.region_size, wl.region_extends, s.density, wl.impurity_radius,
                                  tcp_for(s.density), device=dev)
        did[s.index] = bd.add_grid(dg)
        dg.close()
    device_grid_s = time.perf_counter() - t_seed
    bd.set_passes(sweep_passes(wl, did, cell))
    out_seed, _ = bd.run(with_metrics=True)
    seed_s = time.perf_counter() - t_seed
    bd.close()
    seeds_match = bool(np.array_equal(out_seed, out_split))

    # the whole 64-sample sweep once, split over the GPUs by LPT on estimated cost
    full_sweep = None
    if not args.no_full_sweep:
        fw = workloads.lpt_shard(workloads.config2(n_fields=args.fields), rank, world)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t_full = time.perf_counter()
        bf = BatchSweep(dev, precision=N.ES_PRECISION_SPLIT, **tune.shape)
        fid, fcell = {}, {}
        for s in fw.samples:
            dg = DeviceGrid.from_seed(s.seed, fw.region_size, fw.region_extends, s.density, fw.impurity_radius,
                                      tcp_for(s.density), device=dev)
            fid[s.index] = bf.add_grid(dg)
            fcell[s.index] = dg.info().cell_size
            dg.close()
        fpasses = sweep_passes(fw, fid, fcell)
        bf.set_passes(fpasses)
        fstream = torch.cuda.ExternalStream(bf.stream_handle())
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(fstream)
        bf.enqueue()
        f1.record(fstream)
        fout, _ = bf.collect(with_metrics=False)
        full_wall = time.perf_counter() - t_full
        full_dev = f0.elapsed_time(f1) * 1e-3
        full_orbits = bf.total_orbits
        bf.close()
        # the one exchange: every rank's per-sample sigmas to every rank, then
        # FinishResults (sample means, delta_xx) in sample order
        local = per_sample_sigmas(fpasses, fout, {v: k for k, v in fid.items()}, len(fw.fields),
                                  len(fw.temperatures))
        fcoh, finc = gather_sweep(local, 64, dist if world > 1 else None)
        fin = finish_results(fcoh, finc)
        ft = torch.tensor([full_wall, full_dev], dtype=torch.float64, device="cuda")
        fo = torch.tensor([float(full_orbits)], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(ft, op=dist.ReduceOp.MAX)
            dist.all_reduce(fo, op=dist.ReduceOp.SUM)
        full_pts = 64 * len(fw.fields) * len(fw.temperatures)
        full_sweep = {"samples": 64, "fields": len(fw.fields), "temperatures_K": fw.temperatures,
                      "orbits": int(fo[0].item()), "partition": "LPT on estimated cost (workloads.lpt_shard)",
                      "scaling": "strong", "wall_s": float(ft[0].item()), "device_s": float(ft[1].item()),
                      "lifetimes_per_sec": float(fo[0].item()) / float(ft[1].item()),
                      "sigma_points_per_sec": full_pts / float(ft[1].item()),
                      "finish_results": {"rows": int(fin["delta_xx"].size),
                                         "delta_xx_median": float(np.median(fin["delta_xx"])),
                                         "sigma_xx_total_at_1T_0K": float(fin["coherent"][0, 0, 0]
                                                                          + fin["incoherent"][0, 0, 0])},
                      "note": "timed once outside the step loop; wall_s includes building every grid on the "
                              "GPU from its seed and recording the graph, device_s is the graph replay"}

    # the config-1 sweep (257^2 x 516, 5 fields, both sectors) on the per-pass split path
    c1 = None
    if not args.no_config1:
        w1 = workloads.config1()
        g1 = Grid.from_seed(w1.seed(rank), w1.region_size, w1.region_extends, w1.density, w1.impurity_radius,
                            w1.target_cell_population)
        s1 = make_settings(w1.tau, w1.alpha, w1.clockwise, w1.particle_speed, w1.region_size, w1.region_extends,
                           w1.density, w1.impurity_radius, w1.target_cell_population)
        sw1 = Sweep(w1, g1, s1, N.ES_PRECISION_SPLIT, dev)
        for _ in range(3):
            sw1.step(flush, 1)
        torch.cuda.synchronize()
        ev = [sw1.step(flush, 2) for _ in range(5)]
        torch.cuda.synchronize()
        c1_ms = float(sum(x.elapsed_time(y) for x, y in ev)) / 5
        sw1.close()
        c1 = {"workload": w1.name, "ms_per_step": c1_ms,
              "value": 2 * len(w1.fields) * w1.orbits_per_pass / (c1_ms * 1e-3), "unit": UNIT,
              "sigma_points_per_sec": len(w1.fields) * len(w1.temperatures) / (c1_ms * 1e-3),
              "note": "per-pass split path (es_enqueue_sigmas on two sector contexts), 10 passes per step, "
                      "L2 flushed before each step"}

    peak32 = C.c_double(0.0)
    N.check(N.cuda_lib().es_probe_fp32_fma(dev, C.byref(peak32)))
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    achieved = alg_flops / (step_ms * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": world * args.steps * orbits / (total_ms * 1e-3), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (split)",
        "data": "synthetic (seeded impurity fields; per-sample start grid and density drawn with seed 12345)",
        "config": {"workload": wl.name, "sweep": "config2: 64 samples x 32 fields (1-40 T) x T in {0, 10, 40} K",
                   "samples": [{"index": s.index, "dim": s.dim, "density": s.density} for s in wl.samples],
                   "fields": len(wl.fields), "temperatures_K": wl.temperatures, "passes": n_pass,
                   "orbits_per_step": orbits, "phi_steps": wl.phi_steps,
                   "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write)"},
        "sigma_points_per_sec": world * args.steps * points / (total_ms * 1e-3),
        "tuning": {"shape": tune.shape, "tcp_by_density_class": list(zip(tune.density_edges[:-1], tune.tcp)),
                   "tuner_seconds": round(tune.seconds, 1), "tuner_wall_this_run_s": round(tune_wall, 1)},
        "gpu_launches": graph_replays * kernels_per_replay,
        "graph_replays": graph_replays,
        "retraced_fp64": retraced,
        "clocks": clocks.summary(),
        "roofline": {"bound": "fp32 pipe", "achieved": achieved, "peak": peak32.value, "unit": "TFLOP/s",
                     "frac": achieved / peak32.value if peak32.value else None,
                     "peak_source": "measured FP32 FMA rate (es_probe_fp32_fma, in this run)",
                     "traffic": (profiled_traffic("split", orbits / n_pass)
                                 if tune.shape["mode"] == N.ES_BATCH_PASS_KERNELS
                                 else profiled_traffic("batch_kernel_config2.md")),
                     "kernel": "lifetime_split_kernel + lifetime_finish_kernel + lifetime_retrace_kernel (per pass, "
                               "in the graph)",
                     "work": "algorithmic FP64-op count of the reference's TraceOrbit (flop_model) over the "
                             "graph replay, divided by the replay's device time (the lifetime kernels are "
                             "~98% of it); traffic is per average pass",
                     "flop_model": FLOP_MODEL, "issue": profiled_issue("split")},
        "roofline_integrate": integ,
        "split_vs_fp64": {"results": int(rel.size), "max_rel": float(rel.max()), "median_rel": float(np.median(rel)),
                          "above_1e-6": int((rel > 1e-6).sum()), "sigma_points_max_rel": float(prel.max()),
                          "metrics_equal": metrics_equal, "fp64_batch_ms": fp64_batch_ms,
                          "per_instance_max_rel": [float(x) for x in rel.reshape(n_pass, -1).max(axis=1)]},
        "split_exact_batch": exact,
        "plain_fp64_path": {"passes": n_pass, "points": points, "seconds": plain_s, "points_per_sec": plain_pps,
                            "split_batch_points_per_sec": points / (step_ms * 1e-3),
                            "speedup_same_work": plain_s / (step_ms * 1e-3),
                            "max_rel_vs_plain_fp64": worst_vs_plain,
                            "note": "the same passes through es_compute_sigmas (blocking, FP64 contexts), "
                                    "against the timed split graph replay; the stated bar is 20x"},
        "full_sweep": full_sweep,
        "config1_sweep": c1,
        "host_grid_build_s": grid_build_s,
        "device_grid_build_s": device_grid_s,
        "e2e": {"value": world * orbits / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "seconds_per_step": e2e_s,
                "note": "BatchSweep with host grids each step: grid copies, graph record, replay, sigma and "
                        "metrics read back"},
        "e2e_from_seeds": {"value": orbits / seed_s, "unit": UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": d2h, "seconds": seed_s, "sigma_equal_to_host_grid_run": seeds_match,
                           "note": "grids built on the GPU from the sweep's seeds inside the timed region "
                                   "(DeviceGrid), graph record, run, readback"},
    }
    if cpu:
        line["cpu_baseline"] = {"value": cpu["rate"], "unit": UNIT, "cores": cpu["procs"], "kind": "reference",
                                "sample": cpu["sample"]}
    print(json.dumps(line))


def run_surrogate(args) -> None:
    """Config 4: the learned surrogate. Trains the 4-member ensemble on 20k
    simulator runs (the batched split path at the sweep's resolution, 129^2 starts
    x 516 phases; half of the draw over the full config-4 ranges, half with one
    coordinate in the sub-range where the error concentrated), then serves
    4096-query batches with fallback to the simulator where the members disagree
    by more than 1%, and compares latency and error with the simulator itself."""
    import torch

    from elasticscattering_b200 import surrogate as S

    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and int(os.environ.get("RANK", "0")) != 0:
        return  # replicas only: the surrogate is served from one GPU
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    res = S.Resolution()  # 129^2 x 516: the batched sweep's resolution
    sim = S.Simulator(res, device=dev)
    build_s = sim.prebuild(sim.levels)
    t0 = time.perf_counter()
    train_q = sim.snapped(S.training_queries(args.train_points, seed=1))
    train_s = sim(train_q)
    data_s = time.perf_counter() - t0
    ens = S.MLPEnsemble(4, dev)
    sur = S.Surrogate(ens, sim, tolerance=0.01)
    t0 = time.perf_counter()
    # Adam at 2e-3, halved after each quarter of the run.
    losses = sur.fit(train_q, train_s, steps=args.train_steps, batch=256, lr=2e-3, seed=0)
    train_s_time = time.perf_counter() - t0
    # fallback threshold: calibrated on held-out simulator answers so that the
    # network's own answers meet the 1% bar at the 95th percentile
    cal_q = sim.snapped(S.sample_queries(args.eval_queries * 2, seed=50))
    tol = sur.calibrate(cal_q, sim(cal_q), target=0.01, quantile=0.95)

    Q = 4096
    batches = [sim.snapped(S.sample_queries(Q, seed=100 + k)) for k in range(args.steps + args.warmup)]
    # the simulator on the same kind of batch: latency and the error reference
    eval_q = batches[-1][:args.eval_queries]
    t0 = time.perf_counter()
    truth = sim(eval_q)
    sim_s = time.perf_counter() - t0
    sim_ms_per_query = 1e3 * sim_s / len(eval_q)
    nn_only = (np.abs(S.untarget(eval_q, ens.predict(S.features(eval_q))[0]).mean(axis=0) - truth)
               / np.abs(truth)).max(axis=1)

    def serve(tolerance: float) -> dict:
        sur.tolerance = tolerance
        for k in range(args.warmup):
            sur.query(batches[k])
        net_ms, fb_frac, t_total = [], [], 0.0
        for k in range(args.warmup, args.warmup + args.steps):
            t0 = time.perf_counter()
            _, fb, _, tm = sur.query(batches[k])
            t_total += time.perf_counter() - t0
            net_ms.append(1e3 * tm["network_s"])
            fb_frac.append(float(fb.mean()))
        sig, fb, _, _ = sur.query(eval_q)
        err = (np.abs(sig - truth) / np.abs(truth)).max(axis=1)
        ans = ~fb
        med_fb = statistics.median(fb_frac)
        return {"spread_threshold": tolerance, "queries_per_sec": args.steps * Q / t_total,
                "ms_per_batch": 1e3 * t_total / args.steps,
                "network_ms_per_batch": statistics.median(net_ms),
                "fallback_fraction": med_fb,
                # per query: the network pass alone when it answers, else the simulator too
                "median_query_latency_ms": statistics.median(net_ms) if med_fb < 0.5 else None,
                "latency_gain_median": (sim_ms_per_query * Q) / statistics.median(net_ms) if med_fb < 0.5 else None,
                "error_all_p50": float(np.median(err)), "error_all_p95": float(np.quantile(err, 0.95)),
                "error_all_max": float(err.max()), "answered_by_network": int(ans.sum()),
                "error_network_answers_p95": float(np.quantile(err[ans], 0.95)) if ans.any() else None,
                "error_network_answers_max": float(err[ans].max()) if ans.any() else None}

    stated = serve(0.01)
    calibrated = serve(tol)

    # one query at a time: the network pass (features, copies, kernels, untarget)
    # against the simulator on that one query (its graph recorded and run for it)
    sur.tolerance = 0.01
    one_nn, one_sim = [], []
    for k in range(3):
        sur.query(eval_q[k:k + 1])
    for k in range(64):
        one_nn.append(1e3 * sur.query(eval_q[k:k + 1])[3]["network_s"])
    sim(eval_q[:1])
    for k in range(8):
        t0 = time.perf_counter()
        sim(eval_q[k:k + 1])
        one_sim.append(1e3 * (time.perf_counter() - t0))
    single = {"network_ms_median": statistics.median(one_nn), "simulator_ms_median": statistics.median(one_sim),
              "latency_gain_median": statistics.median(one_sim) / statistics.median(one_nn),
              "note": "a single query per call: the network pass alone (it answers at the stated spread) "
                      "against the simulator run for that query"}
    line = {
        "metric": "sigma queries/sec (surrogate with fallback)", "value": stated["queries_per_sec"],
        "unit": "queries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": stated["ms_per_batch"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 (hidden layers) + f32 head",
        "data": "synthetic: config-4 draws (B, density, tau log-uniform; T uniform), densities at the 16 grid levels",
        "config": {"workload": "config4-surrogate", "queries_per_batch": Q, "train_points": args.train_points,
                   "train_steps": args.train_steps,
                   "simulator": "batched split path, 129^2 starts x 516 phases (the sweep's resolution)",
                   "training_draw": "half over the config-4 ranges, half with B, tau or T in its hard sub-range",
                   "error_target": "1% at the 95th percentile of network answers, fallback at 1% member spread"},
        "operating_point_spread_1pct": stated,
        "operating_point_calibrated": calibrated,
        "single_query_latency": single,
        "simulator_latency_ms_per_query": sim_ms_per_query,
        "simulator_latency_ms_per_batch_extrapolated": sim_ms_per_query * Q,
        "network_only_error": {"queries": int(len(eval_q)), "p50": float(np.median(nn_only)),
                               "p95": float(np.quantile(nn_only, 0.95)), "max": float(nn_only.max())},
        "training": {"grid_build_s": build_s, "data_s": data_s, "train_s": train_s_time,
                     "final_loss": losses[-1]},
        "gpu_launches": ens.launch_count(),
        # the queries arrive as host arrays and the answers return to the host on every call
        "e2e": {"value": stated["queries_per_sec"], "unit": "queries/s", "h2d_bytes_per_step": Q * 5 * 4,
                "d2h_bytes_per_step": Q * (ens.n_nets * 2 + 2 + 2) * 4,
                "note": "Surrogate.query on host arrays: features in, member/mean/spread out, simulator fallback"},
        "roofline": mlp_roofline(Q, ens.n_nets, statistics.median([calibrated["network_ms_per_batch"],
                                                                    stated["network_ms_per_batch"]])),
    }
    ens.close()
    sim.close()
    print(json.dumps(line))


def mlp_roofline(q: int, n_nets: int, ms: float) -> dict:
    """The network pass of one serving batch against the measured dense BF16 rate:
    2 flops per multiply-add of the 5-256-256-256-256-2 layers, every member."""
    macs = 5 * 256 + 3 * 256 * 256 + 256 * 2
    flops = 2.0 * q * n_nets * macs
    peak, src = None, "MEASURED_PEAKS.json absent: fallback 1590 TFLOP/s"
    try:
        peak = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["bf16_tflops"])
        src = "MEASURED_PEAKS.json bf16_tflops (burst, cuBLAS bf16 GEMM)"
    except Exception:
        peak = 1590.0
    achieved = flops / (ms * 1e-3) / 1e12
    return {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": None,
            "kernel": "es_mlp_query's batched path: query_features_kernel, tc_gemm_kernel (tcgen05.mma, BF16 in, "
                      "FP32 accumulator in TMEM) for the 256 x 256 layers, gemm_kernel (mma.sync) for the 5 -> 256 "
                      "layer, head_forward_kernel (FP32), query_combine_kernel; timed host to host",
            "work": f"{flops:.3g} flops per {q}-query batch, {n_nets} members", "peak_source": src,
            "note": "latency-bound: a 4096 x 256 x 256 layer is 0.27 GFLOP, a few microseconds at peak"}


def profiled_issue(name: str):
    """The issue-slot view of a lifetime kernel from its committed ncu summary:
    the fraction of cycles a warp scheduler issued (smsp__issue_active) and the
    active lanes per issued instruction. These kernels are issue-bound, so their
    ceiling is the issue rate with 32 lanes per instruction, not an FMA pipe."""
    p = ROOT / "profiles" / ("lifetime_split_config1.md" if name == "split" else "lifetime_fp64_config1.md")
    if not p.exists():
        return None
    out = {}
    for line in p.read_text().splitlines():
        for key in ("issue_active_frac", "threads_per_instruction"):
            if line.startswith(key + ":"):
                try:
                    out[key] = float(line.split(":", 1)[1].strip())
                except ValueError:
                    pass
    if len(out) != 2:
        return None
    out["lane_frac"] = out["threads_per_instruction"] / 32.0
    out["source"] = f"ncu --set full summary, profiles/{p.name} (one 257^2 x 516-orbit pass, B = 20 T)"
    return out


def profiled_traffic(name: str, orbits: int | None = None):
    """DRAM bytes per launch from a committed ncu summary ("split", "fp64" or a
    file name under profiles/), if present. With `orbits`, a summary that states
    the orbits of its captured launch (`orbits_per_launch:`) is scaled to a launch
    of that many orbits (the lifetime kernels write 8 bytes per orbit and read
    little else)."""
    if name.endswith(".md"):
        p = ROOT / "profiles" / name
    else:
        p = ROOT / "profiles" / ("lifetime_split_config1.md" if name == "split" else "lifetime_fp64_config1.md")
    if not p.exists():
        return None
    fields = {}
    for line in p.read_text().splitlines():
        for key in ("traffic_bytes_per_launch", "orbits_per_launch"):
            if line.startswith(key + ":"):
                try:
                    fields[key] = float(line.split(":", 1)[1].strip())
                except ValueError:
                    pass
    traffic = fields.get("traffic_bytes_per_launch")
    if traffic is not None and orbits and fields.get("orbits_per_launch"):
        traffic *= orbits / fields["orbits_per_launch"]
    return traffic


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["split", "fp64"], default="split")
    ap.add_argument("--workload", default="config2", choices=sorted(workloads.WORKLOADS) + ["config2", "config4"])
    ap.add_argument("--train-points", type=int, default=20000, help="config4: simulator runs for training")
    ap.add_argument("--train-steps", type=int, default=36000, help="config4: Adam steps")
    ap.add_argument("--eval-queries", type=int, default=512, help="config4: queries checked against the simulator")
    ap.add_argument("--ref-rows", type=int, default=2, help="start-position rows per CPU process")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--samples", type=int, default=0,
                    help="config2: 0 = the representative slice (one sample of each start grid per GPU); "
                         "N > 0 = the first N samples per GPU")
    ap.add_argument("--fields", type=int, default=32, help="config2: fields uniformly spaced 1-40 T")
    ap.add_argument("--no-full-sweep", action="store_true", help="config2: skip the one timing of all 64 samples")
    ap.add_argument("--no-config1", action="store_true", help="config2: skip the config-1 sweep")
    ap.add_argument("--tune-cache", default=None, help="config2: autotuner cache file")
    ap.add_argument("--retune", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "config2":
        run_batched(args)
    elif args.workload == "config4":
        run_surrogate(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
