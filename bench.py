"""Benchmark of the per-timestep hot path on the PMB brittle-fracture
notched-plate impact (plate 0.2 x 0.1 x 0.009 m, dx = 0.2/800 ->
800 x 400 x 36 = 11.52 M particles, delta = 3.01 dx, two 0.05 m notches,
16.5 m/s impact strip held by a zero-force BC).

One bench step = one velocity-Verlet time step of the whole plate: bond
break test + PMB force over every directed bond, force BC, both half-step
updates. Metric: bond-updates/s = (directed neighbour entries, broken ones
included, since the kernel visits them) x steps / device time.

Default run: the mixed-precision path (FP32 bonds, FP64 state) is the
headline `value`; the plain FP64 path runs the same steps from the same
start and is reported beside it (`plain_fp64`, `mixed_vs_plain`), with the
per-field error of mixed vs FP64 (`mixed_error_vs_fp64`).

`other_workloads` (N = 1): short runs of the 1.2 M-particle variant of the
plate, the LPS fracture box (8.0 M particles), the Hertzian DEM packing
(4.0 M spheres) and the 41^3 PMB elastic wave, each mixed beside plain FP64
with the error between them.

`serving` (N = 1): the served stream of 512 independent PMB/LPS jobs
(particles log-uniform in [1e3, 2e6], 200-2000 steps) through the job
server (continuous batching, mixed precision, jobs of at most 32768
particles advanced in batch groups): capacity from a saturated pass, then
Poisson arrivals at 0.8 x capacity with p50/p99 job latency, the per-job
server (batch groups off) on the same saturated stream, and the same jobs
one at a time on the plain FP64 path under the same arrivals in real time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (torchrun, one rank per GPU): every rank advances its own plate
(independent specimens, no data-path collective; weak scaling); value is
all ranks' bond updates over the slowest rank's device time.
--impl reference: the CPU oracle (the reference's algorithm restated in
C++/OpenMP; the reference itself needs Kokkos + Cabana + MPI and cannot be
built here) on all host threads, rank 0 only, each step a bounded slab of
the same plate.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from cabanapd_b200 import problems as P  # noqa: E402

PLATE_CELLS = (800, 400, 36)
HORIZON_FACTOR = 3.01  # delta / dx of the plate
LPS_CELLS = (1000, 400, 20)   # LPS random-notch box, dx = 1e-4: 8.0 M particles
PLATE_1P2M_CELLS = (376, 188, 17)  # the ~1.2 M-particle variant of the plate
WAVE_CELLS = 41               # PMB elastic wave, 41^3 particles
DEM_DIMS = (200, 200, 100)    # Hertz packing: 4.0 M spheres
CPU_SLAB_X = 50  # bounded CPU sample: the first 50 x-columns of the plate


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_bond(name):
    """DRAM bytes per directed bond of a bond kernel from its committed ncu
    summary under profiles/, or None."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        for line in fh:
            if line.startswith("dram_bytes_per_bond:"):
                return float(line.split(":")[1])
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        """Start sampling every 50 ms and wait (up to 3 s) for the first
        sample, so that sampling covers the timed region that follows."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
            return
        t_end = time.perf_counter() + 3.0
        while not self.lines and time.perf_counter() < t_end and self.proc.poll() is None:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def stop(self, t0=None, t1=None):
        """Summary of the samples read in [t0, t1 + 0.1 s] (host clock; all
        samples when no window is given)."""
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, line in self.lines:
            if t0 is not None and not (t0 <= t <= t1 + 0.1):
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, value, device):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(pg, value, device):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg, device):
    if pg is None:
        return
    if device == "cpu":
        pg.barrier()
        return
    import torch
    pg.barrier(device_ids=[device])
    torch.cuda.synchronize(device)


def aggregate(pg, device, ms_local, bonds_local, steps):
    """Whole-job throughput: every rank's bond updates over the slowest
    rank's device time (max over ranks)."""
    ms = reduce_max(pg, ms_local, device)
    total = reduce_sum(pg, float(bonds_local), device)
    return total * steps / (ms / 1e3), ms, total


def visible_index(local):
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    ids = [c for c in cvd.split(",") if c.strip()]
    if ids and ids[min(local, len(ids) - 1)].strip().isdigit():
        return int(ids[min(local, len(ids) - 1)])
    return local


# ---------------------------------------------------------------------------
def cpu_sample_problem():
    prob = P.plate_impact(num_cells=PLATE_CELLS, steps=1, horizon_factor=HORIZON_FACTOR)
    nx, ny, nz = PLATE_CELLS
    ix = np.arange(prob["x"].shape[0]) % nx
    keep = ix < CPU_SLAB_X
    remap = -np.ones(keep.size, dtype=np.int64)
    remap[keep] = np.arange(int(keep.sum()))
    sub = dict(prob)
    for k in ("x", "vol", "rho", "nofail", "v0"):
        sub[k] = np.ascontiguousarray(prob[k][keep])
    sub["bcs"] = [(kind, c, remap[idx[keep[idx]]], vals) for kind, c, idx, vals in prob["bcs"]]
    return sub


def time_cpu_sample(target_seconds=15.0, max_steps=200):
    """Oracle on all host threads over the bounded slab; returns a dict."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    threads = os.cpu_count() or 1
    pyoracle.set_num_threads(threads)
    sub = cpu_sample_problem()
    s = pyoracle.OracleSystem(sub["params"])
    P.setup(s, sub)
    bonds = s.neighbor_stats()[1]
    t0 = time.perf_counter()
    s.run(1)
    t1 = time.perf_counter() - t0
    steps = int(max(1, min(max_steps, target_seconds / max(t1, 1e-6))))
    t0 = time.perf_counter()
    s.run(steps)
    dt = time.perf_counter() - t0
    return {"value": bonds * steps / dt, "unit": "bond-updates/s", "cores": threads,
            "kind": "port", "steps": steps, "seconds": dt, "bonds_per_step": bonds,
            "particles": s.n,
            "sample": (f"first {CPU_SLAB_X} of {PLATE_CELLS[0]} x-columns of the plate "
                       f"({s.n} particles, {bonds} bonds), {steps} timed steps after 1 "
                       f"warm-up step, CPU oracle (C++17/OpenMP port of the reference "
                       f"kernels), {threads} threads")}


def run_reference(args, world, rank):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    threads = os.cpu_count() or 1
    pyoracle.set_num_threads(threads)
    sub = cpu_sample_problem()
    s = pyoracle.OracleSystem(sub["params"])
    P.setup(s, sub)
    bonds = s.neighbor_stats()[1]
    s.run(args.warmup)
    t0 = time.perf_counter()
    s.run(args.steps)
    dt = time.perf_counter() - t0
    value = bonds * args.steps / dt
    sample = (f"each step: one time step of the first {CPU_SLAB_X} of {PLATE_CELLS[0]} "
              f"x-columns of the plate ({s.n} particles, {bonds} bonds); CPU oracle "
              f"(C++17/OpenMP restatement of the reference kernels; the reference "
              f"needs Kokkos/Cabana/MPI and is not buildable here), {threads} threads")
    line = {
        "impl": "reference", "metric": "bond-updates/s", "value": value,
        "unit": "bond-updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "pmb_fracture_notched_plate_impact",
                   "plate_cells": list(PLATE_CELLS), "sample_particles": s.n,
                   "sample_bonds": bonds},
        "cpu_baseline": {"value": value, "unit": "bond-updates/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "bond-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
PRECISION = {"exact": 0, "fp64": 1, "mixed": 2}
KERNEL = {"fp64": "k_pmb_stencil64<fracture> (lattice-stencil FP64 bond stage, fused step)",
          "mixed": "k_pmb_stencil32<fracture> (lattice-stencil FP32 bond stage, fused step)",
          "exact": "k_pd_force<PMB, fracture> (bit-exact)"}
PROFILE = {"fp64": "pmb_stencil64_plate.txt", "mixed": "pmb_stencil32_plate.txt",
           "exact": "pmb_force_exact_plate.txt"}


def timed_steps(sys_, stream, args, device, pg, sampler):
    """Warm-up, then exactly args.steps device-timed steps (CUDA events on
    the launching stream, barrier + synchronize on both sides)."""
    import torch
    sys_.step(args.warmup)
    sys_.synchronize()
    sys_.set_kernel_timing(True)
    launches0 = sys_.kernel_launches()
    barrier(pg, device)
    torch.cuda.synchronize(device)
    if sampler:
        sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    ev0.record(stream)
    sys_.step(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize(device)
    t1 = time.perf_counter()
    clocks = sampler.stop(t0, t1) if sampler else None
    barrier(pg, device)
    k_ms, k_n, k_bytes = sys_.kernel_time()
    sys_.set_kernel_timing(False)
    return {"ms": ev0.elapsed_time(ev1), "launches": sys_.kernel_launches() - launches0,
            "k_ms": k_ms, "k_n": k_n, "k_bytes": k_bytes, "clocks": clocks}


def roofline(prec, r, bonds):
    hbm, hbm_kind = peaks()
    avg_ms = r["k_ms"] / max(r["k_n"], 1)
    achieved = r["k_bytes"] / (avg_ms / 1e3) / 1e9
    tpb = traffic_per_bond(PROFILE[prec])
    return {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": hbm_kind, "kernel": KERNEL[prec],
            "kernel_ms_avg": avg_ms, "kernel_launches": r["k_n"],
            "algorithmic_bytes_per_launch": r["k_bytes"],
            "traffic": (tpb * bonds if tpb else None)}


def _time_system(s, stream, device, steps, warmup):
    import torch
    s.step(warmup)
    s.synchronize()
    s.set_kernel_timing(True)
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    s.step(steps)
    ev1.record(stream)
    torch.cuda.synchronize(device)
    k_ms, k_n, k_bytes = s.kernel_time()
    s.set_kernel_timing(False)
    return ev0.elapsed_time(ev1), k_ms / max(k_n, 1), k_bytes


def other_workload(name, steps):
    """(problem, precisions, kernel names, description) of another hot-path
    workload measured beside the headline plate."""
    mixed_pmb = "k_pmb_stencil32<fracture> (fused step)"
    fp64_pmb = "k_pmb_stencil64<fracture> (fused step)"
    if name == "lps":
        return (P.lps_random_notches(num_cells=LPS_CELLS, steps=steps), ["mixed", "fp64"],
                {"mixed": "k_lps_mtheta_lean + k_lps_force_lean<fracture> over lean warps, "
                          "k_lps_mtheta_mixed + k_lps_force_mixed over the rest (fused step)",
                 "fp64": "k_lps_m_theta_1pass + k_lps_force_pf<fracture> (fused step)"},
                {"workload": "lps_fracture_random_notches", "cells": list(LPS_CELLS)})
    if name == "plate_1p2m":
        return (P.plate_impact(num_cells=PLATE_1P2M_CELLS, steps=steps), ["mixed", "fp64"],
                {"mixed": mixed_pmb, "fp64": fp64_pmb},
                {"workload": "pmb_fracture_notched_plate_impact_1p2m",
                 "plate_cells": list(PLATE_1P2M_CELLS)})
    if name == "wave":
        return (P.elastic_wave_pmb(n=WAVE_CELLS, steps=steps), ["mixed", "fp64"],
                {"mixed": mixed_pmb.replace("fracture", "elastic"),
                 "fp64": fp64_pmb.replace("fracture", "elastic")},
                {"workload": "pmb_elastic_wave", "cells": [WAVE_CELLS] * 3})
    return (P.dem_packing(lattice_dims=DEM_DIMS, steps=steps), ["mixed", "fp64"],
            {"mixed": "k_hertz_force_mixed<per-particle radius> (FP64 overlap, FP32 force law)",
             "fp64": "k_hertz_force<per-particle radius>"},
            {"workload": "dem_hertz_packing", "lattice": list(DEM_DIMS), "rebuild_every": 10})


def check_mixed_error(workload, err):
    """A mixed-precision run that left finite values or the mixed bars far
    behind (relative error above 1e-3 in a field against FP64) has broken
    arithmetic: no throughput is reported for it."""
    bad = {k: v for k, v in err.items()
           if k in ("u", "v", "f", "theta") and not (np.isfinite(v) and v <= 1e-3)}
    if bad:
        raise SystemExit(f"{workload}: mixed precision departs from FP64: {bad}")


def measure_other(name, device, stream, steps, warmup):
    """A short measurement of another hot-path workload: the LPS fracture
    box (8.0 M particles), the 1.2 M-particle variant of the notched plate or
    the 41^3 PMB elastic wave, or the Hertzian DEM packing (4.0 M spheres,
    contact list rebuilt every 10 steps inside the timed steps), each mixed
    beside plain FP64 from the same start with the error of mixed vs FP64."""
    import cabanapd_b200
    prob, precs, kernel, wl = other_workload(name, steps)
    res, systems = {}, {}
    for prec in precs:
        s = cabanapd_b200.System(dict(prob["params"], device=device, precision=PRECISION[prec]))
        s.set_stream(stream.cuda_stream)
        P.setup(s, prob)
        _, bonds0 = s.neighbor_stats()
        ms, k_avg, k_bytes = _time_system(s, stream, device, steps, warmup)
        _, bonds1 = s.neighbor_stats()
        bonds = 0.5 * (bonds0 + bonds1) if name == "dem" else bonds0
        res[prec] = dict(precision=prec, ms_per_step=ms / steps,
                         value=bonds * steps / (ms / 1e3), kernel=kernel[prec],
                         kernel_ms_avg=k_avg)
        hbm, hbm_kind = peaks()
        rows = s.n - prob["n_frozen"]
        if name == "lps":
            # Both row passes of a step: the force pass's bytes (as the
            # library counts them) plus the weighted-volume / dilatation
            # pass (read x, u, vol, count, write m, theta and the two force
            # factors: 92 B per row; 4 B index + 1/8 B bond bit per bond),
            # over the whole step's time.
            step_bytes = k_bytes + 92.0 * rows + 4.125 * bonds0
            achieved = step_bytes / (ms / steps / 1e3) / 1e9
            res[prec]["roofline"] = {
                "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": hbm_kind,
                "algorithmic_bytes_per_step": step_bytes, "timed": "whole step"}
        elif name == "dem":
            achieved = k_bytes / (k_avg / 1e3) / 1e9
            res[prec]["roofline"] = {
                "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": hbm_kind,
                "algorithmic_bytes_per_launch": k_bytes,
                "timed": "contact kernel with the step epilogue"}
        if name == "dem":
            res[prec]["contact_rebuilds"] = s.contact_rebuilds()
            res[prec]["contacts"] = bonds
        systems[prec] = s
    head = precs[0]
    out = dict(wl, particles=systems[head].n, bonds=bonds, steps=steps, warmup=warmup,
               unit="bond-updates/s", **res[head])
    if name == "dem" and DEM_FULL_STEPS > warmup + steps:
        # The packing's mixed-vs-FP64 error over its full run (few pairs
        # overlap in the first steps, where both Hertz kernels skip them).
        for s in systems.values():
            s.step(DEM_FULL_STEPS - warmup - steps)
            s.synchronize()
        out_steps = DEM_FULL_STEPS
    else:
        out_steps = warmup + steps
    if "fp64" in res and head != "fp64":
        a, b = systems[head], systems["fp64"]
        err = {"after_steps": out_steps}
        fields = ("u", "v", "f", "theta") if name == "lps" else ("u", "v", "f")
        for fld in fields:
            x, y = a.get(fld), b.get(fld)
            err[fld] = float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
        if prob["params"].get("fracture"):
            err["damage_identical"] = bool(np.array_equal(a.get("phi"), b.get("phi")))
        if name == "dem":
            err["contact_rebuilds"] = [a.contact_rebuilds(), b.contact_rebuilds()]
            err["contacts"] = [a.neighbor_stats()[1], b.neighbor_stats()[1]]
        check_mixed_error(name, err)
        out["plain_fp64"] = res["fp64"]
        out["mixed_vs_plain"] = res["fp64"]["ms_per_step"] / res[head]["ms_per_step"]
        out["mixed_error_vs_fp64"] = err
    for s in systems.values():
        s.close()
    return out


def measure_batch(device, count=64, chunk=16, chunks=10, precision="mixed"):
    """Many small jobs (PMB / LPS, 1e3-3e4 particles) advanced as one batch
    (cpd_batch: one persistent-block launch per step for all of them, after
    the autotuner has timed its candidates) beside the same systems each
    replaying its own CUDA graph of `chunk` steps on its own stream (the
    per-job form). Host-timed over `chunks` chunks, synchronised."""
    import torch

    import cabanapd_b200
    jobs = P.served_jobs(count=count, n_range=(1e3, 3e4), steps_range=(4000, 4000), seed=77)

    def build():
        out = []
        for j in jobs:
            s = cabanapd_b200.System(dict(j["params"], device=device,
                                          precision=PRECISION[precision]))
            P.setup(s, j)
            out.append(s)
        return out

    systems = build()
    bonds = sum(s.neighbor_stats()[1] for s in systems)
    b = cabanapd_b200.Batch(systems, [4000] * count)
    ncand = len(b.tuning()[1])
    for _ in range(ncand):
        b.step(chunk)
        b.synchronize()
    b.step(chunk)
    b.synchronize()
    l0 = b.launches()
    t0 = time.perf_counter()
    for _ in range(chunks):
        b.step(chunk)
    b.synchronize()
    t_batch = time.perf_counter() - t0
    launches_batch = b.launches() - l0
    chosen, cands = b.tuning()
    b.close()
    for s in systems:
        s.close()

    systems = build()
    streams, graphs = [], []
    for s in systems:
        st = torch.cuda.Stream(device=device)
        s.set_stream(st.cuda_stream)
        s.step(chunk)
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=st):
            s.step(chunk)
        streams.append(st)
        graphs.append(g)
    for g, st in zip(graphs, streams):
        with torch.cuda.stream(st):
            g.replay()
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(chunks):
        for g, st in zip(graphs, streams):
            with torch.cuda.stream(st):
                g.replay()
    torch.cuda.synchronize(device)
    t_graphs = time.perf_counter() - t0
    del graphs
    for s in systems:
        s.close()
    work = bonds * chunk * chunks
    return {"workload": f"{count} independent jobs (PMB elastic cubes, PMB notched plates, "
                        "LPS random-notch boxes), particles log-uniform in [1000, 30000], "
                        "seed 77",
            "precision": precision, "bonds": bonds, "steps": chunk * chunks,
            "batched": {"bond_updates_per_s": work / t_batch, "s": t_batch,
                        "launches": launches_batch,
                        "tuner": {"chosen": chosen,
                                  "candidates": [{"blocks_per_sm": g, "order": o,
                                                  "bond_updates_per_s": t}
                                                 for g, o, t in cands]}},
            "per_system_graphs": {"bond_updates_per_s": work / t_graphs, "s": t_graphs},
            "batched_vs_per_system": t_graphs / t_batch,
            "timing": "host clock around synchronised chunks"}


E2E_JOBS = 3
OTHER_STEPS = {"lps": 20, "plate_1p2m": 100, "wave": 100, "dem": 50}
DEM_FULL_STEPS = 5000  # the packing's full run, for its mixed-vs-FP64 error


def run_gpu(args, world, rank, local, pg):
    import torch

    import cabanapd_b200
    device = local
    torch.cuda.set_device(device)
    prob = P.plate_impact(num_cells=PLATE_CELLS, steps=args.steps,
                          horizon_factor=HORIZON_FACTOR)
    stream = torch.cuda.Stream(device=device)
    precs = [args.precision] if args.precision != "mixed" or args.only else ["mixed", "fp64"]
    systems, res = {}, {}
    for prec in precs:
        sys_ = cabanapd_b200.System(dict(prob["params"], device=device,
                                         precision=PRECISION[prec]))
        sys_.set_stream(stream.cuda_stream)
        P.setup(sys_, prob)
        sampler = ClockSampler(visible_index(local)) if rank == 0 else None
        res[prec] = timed_steps(sys_, stream, args, device, pg, sampler)
        systems[prec] = sys_
    head = precs[0]
    _, bonds = systems[head].neighbor_stats()
    n = systems[head].n
    value, ms, total_bonds = aggregate(pg, device, res[head]["ms"], bonds, args.steps)
    particle_steps = reduce_sum(pg, float(n), device) * args.steps / (ms / 1e3)
    plain = None
    if "fp64" in res and head != "fp64":
        pv, pms, _ = aggregate(pg, device, res["fp64"]["ms"], bonds, args.steps)
        # Same start, same number of steps: error of the headline path vs FP64.
        a, b = systems[head], systems["fp64"]
        err = {}
        for fld in ("u", "v", "f"):
            x, y = a.get(fld), b.get(fld)
            err[fld] = float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
        wa, da = a.compute_energy()
        wb, db = b.compute_energy()
        err["strain_energy"] = abs(wa - wb) / abs(wb)
        err["damage_identical"] = bool(np.array_equal(a.get("phi"), b.get("phi")))
        err["total_damage"] = [da, db]
        check_mixed_error("plate", err)
        plain = {"value": pv, "ms_per_step": pms / args.steps,
                 "roofline": roofline("fp64", res["fp64"], bonds),
                 "gpu_launches": res["fp64"]["launches"]}
    for sys_ in systems.values():
        sys_.close()
    systems.clear()

    if args.skip_e2e:
        e2e_value, h2d, d2h, job_ms = None, None, None, None
    else:
        e2e_value, h2d, d2h, job_ms = run_e2e(args, prob, device, stream, pg, total_bonds, head)
    if rank != 0:
        return
    line = {
        "metric": "bond-updates/s", "value": value, "unit": "bond-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"mixed": "f32 bonds + f64 state", "fp64": "f64", "exact": "f64"}[head],
        "data": "synthetic",
        "config": {"workload": "pmb_fracture_notched_plate_impact",
                   "plate_cells": list(PLATE_CELLS), "horizon_over_dx": HORIZON_FACTOR,
                   "particles_per_gpu": n,
                   "bonds_per_gpu": bonds, "precision": head,
                   "l2": "inputs larger than L2 (neighbour list %.1f GB)" % (4 * bonds / 1e9),
                   "particle_steps_per_s": particle_steps},
        "roofline": roofline(head, res[head], bonds),
        "e2e": ({"value": e2e_value, "unit": "bond-updates/s",
                 "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                 "job": ("upload + neighbour build + prenotch + init + steps + "
                         "energy/damage read every 10 steps + download u"),
                 "jobs": len(job_ms), "job_ms": job_ms,
                 "statistic": "median over fresh systems"}
                if e2e_value is not None else None),
        "gpu_launches": res[head]["launches"],
        "clocks": res[head]["clocks"],
    }
    if plain is not None:
        line["plain_fp64"] = plain
        line["mixed_vs_plain"] = value / plain["value"]
        line["mixed_error_vs_fp64"] = err
    if world == 1 and not args.skip_others:
        line["other_workloads"] = [measure_other(w, device, stream, OTHER_STEPS[w], 3)
                                   for w in ("plate_1p2m", "lps", "dem", "wave")]
        line["small_jobs_batch"] = measure_batch(device)
    if world == 1 and not args.skip_serve:
        line["serving"] = run_serving(args, device)
    if world == 1 and not args.skip_cpu:
        line["cpu_baseline"] = time_cpu_sample()
        line["cpu_baseline"].pop("steps", None)
    print(json.dumps(line), flush=True)


def _percentile(values, q):
    v = sorted(values)
    if not v:
        return None
    k = (len(v) - 1) * q
    lo, hi = int(math.floor(k)), int(math.ceil(k))
    return v[lo] + (v[hi] - v[lo]) * (k - lo)


def _latency_summary(lat):
    return {"p50": _percentile(lat, 0.50), "p99": _percentile(lat, 0.99),
            "mean": sum(lat) / len(lat), "max": max(lat)}


def run_serving(args, device):
    """Served stream: independent PMB/LPS jobs through the job server
    (mixed precision). Passes over the same seeded jobs:
    1. saturated: all jobs submitted at t = 0 (batch groups on for jobs of
       at most --serve-batch particles); capacity = jobs / makespan;
    2. served: Poisson arrivals at 0.8 x capacity (seeded), latency =
       finish - arrival for every job;
    3. per-job server, saturated: the same server with batch groups off
       (every job on its own stream and graph), for comparison;
    4. one at a time, plain FP64, the same arrivals in real time: each job
       alone (set-up, steps, energy, u read back) once it has arrived and
       the previous one is done; latency = finish - arrival."""
    import cabanapd_b200
    n_lo, n_hi = args.serve_n
    jobs = P.served_jobs(count=args.serve_jobs, n_range=(n_lo, n_hi),
                         steps_range=tuple(args.serve_steps), seed=args.serve_seed)
    budget = int(args.serve_budget_gb * 1e9)

    def serve(arrivals, batch_max):
        srv = cabanapd_b200.Server(device=device, max_active=args.serve_active,
                                   steps_per_launch=args.serve_k, hbm_budget_bytes=budget,
                                   setup_threads=args.serve_setup_threads,
                                   batch_max_particles=batch_max)
        ids = []
        t0 = time.perf_counter()
        for prob, at in zip(jobs, arrivals):
            delay = at - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(prob, precision=PRECISION["mixed"]))
        srv.drain(timeout=7200)
        sts = [srv.status(i) for i in ids]
        stats = srv.stats()
        srv.close()
        failed = [i for i, st in zip(ids, sts) if st["state"] != cabanapd_b200.system.JOB_DONE]
        if failed:
            raise RuntimeError(f"serving: {len(failed)} jobs failed")
        first = min(st["submit_time"] for st in sts)
        span = max(st["finish_time"] for st in sts) - first
        bonds = sum(st["bonds"] * st["steps"] for st in sts)
        lat = [st["finish_time"] - st["submit_time"] for st in sts]
        wait = [st["start_time"] - st["submit_time"] for st in sts]
        setup = [st["ready_time"] - st["admit_time"] for st in sts]
        return {"makespan_s": span, "bond_updates": bonds,
                "throughput_bond_updates_per_s": bonds / span,
                "jobs_per_s": len(sts) / span, "latency_s": _latency_summary(lat),
                "queue_wait_s": _latency_summary(wait),
                "setup_s": dict(_latency_summary(setup), total=sum(setup)),
                "batched_jobs": sum(1 for j in jobs if batch_max > 0 and j["x"].shape[0] <= batch_max),
                "peak_resident_bytes": stats["peak_resident_bytes"],
                "gpu_launches": stats["kernel_launches"]}

    saturated = serve([0.0] * len(jobs), args.serve_batch)
    capacity = saturated["jobs_per_s"]
    rate = 0.8 * capacity
    rng = np.random.Generator(np.random.PCG64(args.serve_seed + 1))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(jobs))).tolist()
    served = serve(arrivals, args.serve_batch)
    per_job = None if args.serve_quick else serve([0.0] * len(jobs), 0)

    # One at a time on the plain FP64 path, the same arrivals in real time.
    lat, service, bonds_total = [], [], 0
    t0 = time.perf_counter()
    for prob, at in zip(jobs, arrivals):
        idle = at - (time.perf_counter() - t0)
        if idle > 0:
            time.sleep(idle)
        ts = time.perf_counter()
        s = cabanapd_b200.System(dict(prob["params"], device=device, precision=PRECISION["fp64"]))
        P.setup(s, prob)
        s.run(prob["num_steps"])
        s.compute_energy()
        s.get("u")
        tf = time.perf_counter()
        service.append(tf - ts)
        lat.append(tf - t0 - at)
        bonds_total += s.neighbor_stats()[1] * prob["num_steps"]
        s.close()
    span = time.perf_counter() - t0
    one_at_a_time = {"arrivals": "the served pass's Poisson arrivals, in real time",
                     "makespan_s": span, "service_time_sum_s": sum(service),
                     "throughput_bond_updates_per_s": bonds_total / span,
                     "latency_s": _latency_summary(lat)}
    kinds = {k: sum(1 for j in jobs if j["kind"] == k) for k in ("wave", "plate", "lps")}
    out = {
        "workload": (f"{len(jobs)} independent jobs: {kinds['wave']} PMB elastic-wave cubes, "
                     f"{kinds['plate']} PMB notched plates, {kinds['lps']} LPS random-notch "
                     f"boxes; particles log-uniform in [{n_lo:.0f}, {n_hi:.0f}], steps "
                     f"uniform in [{args.serve_steps[0]}, {args.serve_steps[1]}], seed "
                     f"{args.serve_seed}"),
        "precision": "mixed (FP32 bonds / FP64 state, PMB and LPS)",
        "server": {"max_active": args.serve_active, "steps_per_launch": args.serve_k,
                   "setup_threads": args.serve_setup_threads,
                   "batch_max_particles": args.serve_batch,
                   "cuda_graphs": True, "hbm_budget_bytes": budget},
        "capacity_jobs_per_s": capacity,
        "saturated": saturated,
        "arrival_rate_jobs_per_s": rate,
        "served": served,
        "one_at_a_time_fp64": one_at_a_time,
        "throughput_vs_one_at_a_time": (served["throughput_bond_updates_per_s"] /
                                        one_at_a_time["throughput_bond_updates_per_s"]),
    }
    if per_job is not None:
        out["per_job_server_saturated"] = per_job
        out["batched_vs_per_job_saturated"] = (saturated["throughput_bond_updates_per_s"] /
                                               per_job["throughput_bond_updates_per_s"])
    return out


def run_e2e(args, prob, device, stream, pg, total_bonds, prec):
    import torch

    import cabanapd_b200
    # End to end through the C ABI from pinned host buffers: upload, neighbour
    # build, pre-notch, BCs, init, K steps with energy/damage read back every
    # 10 steps, download of the displacement field.
    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.int32,
                        pin_memory=True)
        arr = t.numpy()
        arr[...] = a
        return arr

    hx, hvol, hrho = pinned(prob["x"]), pinned(prob["vol"]), pinned(prob["rho"])
    hnf = pinned(prob["nofail"].astype(np.int32))
    hv0 = pinned(prob["v0"])
    hu = pinned(np.zeros_like(prob["x"]))
    def one_job():
        torch.cuda.synchronize(device)
        barrier(pg, device)
        t0 = time.perf_counter()
        e2 = cabanapd_b200.System(dict(prob["params"], device=device, precision=PRECISION[prec]))
        e2.set_stream(stream.cuda_stream)
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        e2.set_particles(hx, hvol, hrho, hnf)
        e2.set_state(None, hv0)
        e2.build_neighbors()
        e2.prenotch(*prob["notches"])
        for kind, comp, idx, vals in prob["bcs"]:
            e2.add_bc(kind, idx, vals, component=comp)
        e2.init()
        done = 0
        reads = 0
        while done < args.steps:
            k = min(10, args.steps - done)
            e2.step_energy(k)  # k steps, then the output step's energy / damage totals
            done += k
            reads += 1
        e2.get("u", out=hu)
        s1.record(stream)
        torch.cuda.synchronize(device)
        wall = time.perf_counter() - t0
        ms = reduce_max(pg, max(s0.elapsed_time(s1), 1e3 * wall), device)
        e2.close()
        return ms, reads

    # The median of E2E_JOBS jobs, each from a fresh system.
    jobs = [one_job() for _ in range(E2E_JOBS)]
    e2e_ms = float(np.median([ms for ms, _ in jobs]))
    reads = jobs[0][1]
    h2d = (hx.nbytes + hvol.nbytes + hrho.nbytes + hnf.nbytes + hv0.nbytes) / args.steps
    d2h = (hu.nbytes + 16 * reads) / args.steps
    e2e_value = total_bonds * args.steps / (e2e_ms / 1e3)
    return e2e_value, h2d, d2h, [ms for ms, _ in jobs]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU baseline leg")
    ap.add_argument("--skip-e2e", action="store_true", help="omit the end-to-end leg")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "exact", "mixed"],
                    help="mixed (default): FP32 bonds / FP64 state, measured beside the "
                         "plain FP64 path; fp64: throughput FP64 only; exact: bit-exact")
    ap.add_argument("--only", action="store_true",
                    help="with mixed: skip the plain FP64 comparison run")
    ap.add_argument("--cells", default=None,
                    help="cells nx,ny,nz of the plate (or, with --only-other, of that "
                         "workload) for profiling on a smaller case")
    ap.add_argument("--horizon-factor", type=float, default=3.01,
                    help="delta / dx of the plate (for profiling the wide-table walk: 4)")
    ap.add_argument("--skip-serve", action="store_true", help="omit the served-stream leg")
    ap.add_argument("--skip-others", action="store_true",
                    help="omit the LPS-box and DEM-packing measurements")
    ap.add_argument("--only-other", choices=["lps", "dem", "plate_1p2m", "wave", "batch"],
                    default=None,
                    help="measure only that workload (for profiling) and print it")
    ap.add_argument("--serve-jobs", type=int, default=512, help="served stream: number of jobs")
    ap.add_argument("--serve-n", type=float, nargs=2, default=[1e3, 2e6],
                    help="served stream: particle-count range")
    ap.add_argument("--serve-batch", type=int, default=32768,
                    help="served stream: jobs of at most this many particles run in batch groups")
    ap.add_argument("--serve-quick", action="store_true",
                    help="served stream: omit the per-job-server comparison pass")
    ap.add_argument("--serve-steps", type=int, nargs=2, default=[200, 2000])
    ap.add_argument("--serve-seed", type=int, default=20261203)
    ap.add_argument("--serve-active", type=int, default=16)
    ap.add_argument("--serve-k", type=int, default=32, help="steps per CUDA-graph chunk")
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-setup-threads", type=int, default=4)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    global PLATE_CELLS, LPS_CELLS, DEM_DIMS, PLATE_1P2M_CELLS, WAVE_CELLS, HORIZON_FACTOR
    HORIZON_FACTOR = args.horizon_factor
    if args.cells:
        cells = tuple(int(c) for c in args.cells.split(","))
        if args.only_other == "lps":
            LPS_CELLS = cells
        elif args.only_other == "dem":
            DEM_DIMS = cells
        elif args.only_other == "plate_1p2m":
            PLATE_1P2M_CELLS = cells
        elif args.only_other == "wave":
            WAVE_CELLS = cells[0]
        else:
            PLATE_CELLS = cells
    world, rank, local, pg = (int(os.environ.get("WORLD_SIZE", "1")),
                              int(os.environ.get("RANK", "0")),
                              int(os.environ.get("LOCAL_RANK", "0")), None)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.only_other:
        import torch
        torch.cuda.set_device(local)
        stream = torch.cuda.Stream(device=local)
        if args.only_other == "batch":
            out = measure_batch(local, precision=args.precision)
        else:
            out = measure_other(args.only_other, local, stream, args.steps, args.warmup)
        print(json.dumps(out), flush=True)
        return
    world, rank, local, pg = dist_setup()
    try:
        run_gpu(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
