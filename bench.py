"""Benchmark of the Lagrange + ADI-remap step (MaHyCo) on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: Sedov point blast, 128^3 hex mesh on [0,1.2]^3 with 1% seeded node
jitter, one ideal gas (gamma 1.4), plain FP64.  A step is one cycle
(Lagrange phase + three directional remap sweeps + finalisation + dt
reduction) over the whole mesh.  Metric: cell-cycles/s (whole job).

`value` is timed with CUDA events on the context stream around K graph-replayed
cycles, state resident in HBM (working set ~2 GB > 126 MB L2, so no L2 flush is
needed).  `e2e` is the same metric through the reference-facing C ABI: from host
buffers (pinned), mhy_create + mhy_set_state + mhy_hydro_start_init, then K
cycles driven entry point by entry point with dt read back to the host every
cycle (the Arcane time loop reads it), then the final density, energy and
velocity read back.  N > 1 GPUs run independent replicas (weak scaling; the
path has no data exchange between independent meshes).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "arcane-benchs_b200"))

METRIC = "cell-cycles/s"
WORKLOADS = ("sedov", "two_material", "sphere_inclusion", "batched")


def make_case(args):
    """The workload's mesh and initial state (seeded, synthetic) and its name."""
    from mhy_b200 import gen
    tag = "fp64" if args.precision == "fp64" else "mixed"
    if args.workload == "sedov":
        c, name = gen.sedov(n=args.n), f"sedov-{args.n}^3-jitter1%-{tag}"
    elif args.workload == "two_material":
        c, name = gen.two_material(256, 128, 128), f"two-material-256x128x128-{tag}"
    else:
        c, name = gen.sphere_inclusion(384, 384, 192), f"sphere-inclusion-384x384x192-{tag}"
    c.options.precision = 0 if args.precision == "fp64" else 1
    return c, name


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=WORKLOADS, default="sedov",
                    help="sedov: Sedov 128^3 (the headline); two_material: 256x128x128, two gases; "
                         "sphere_inclusion: 384x384x192, two gases; batched: 64 Sod/Sedov instances of "
                         "32^3..96^3 advanced together (instances split across GPUs)")
    ap.add_argument("--n", type=int, default=128, help="Sedov mesh cells per direction")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="fp64: the reference's arithmetic bit for bit; mixed: FP32 remap evaluation, FP64 state")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default tuning (no autotuner trials)")
    ap.add_argument("--tune-lines", default=None,
                    help="set lines per block of the cell y, cell z, node y, node z sweeps (e.g. 16,16,8,8) instead "
                         "of autotuning (profiling runs: timings under a profiler mislead the autotuner)")
    ap.add_argument("--cpu-sample-cycles", type=int, default=5)
    return ap.parse_args()


# DRAM bytes (read + write) of one whole cycle, summed over its kernels, from
# one ncu capture of the 128^3 Sedov cycle (profiles/dram_traffic_sedov128_cycle.md).
# DRAM bytes of one cycle from ncu (dram__bytes_read.sum + dram__bytes_write.sum over the 10 kernels of the
# fourth cycle, cell y/z sweeps at 16 lines per block as the autotuner picks them)
TRAFFIC_PER_CYCLE = {("sedov", 128, "fp64"): 3465343744.0, ("sedov", 128, "mixed"): 2912002560.0}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or f[0] != self.gpu:
                continue
            try:
                sm.append(float(f[1])); smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() in ("active", "0x1", "1"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(case, cycles, wname):
    """The oracle (CPU restatement of the reference algorithm) on this host, all cores."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import mhy_oracle
    threads = os.cpu_count() or 1
    o = mhy_oracle.Oracle(case, pow_mode="libm", threads=threads)
    o.step(1)  # first cycle (page faults, thread start) not timed
    t0 = time.perf_counter()
    o.step(cycles)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": case.ncells * cycles / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{wname} (same mesh and state), cycles 2..{cycles + 1} after init, "
                      f"OpenMP {threads} threads, oracle built -O3 -ffp-contract=off"}


def run_reference(args):
    """--impl reference: the reference algorithm on the host cores (the reference
    itself needs the Arcane framework, absent here, so its CPU restatement runs)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import mhy_oracle
    threads = os.cpu_count() or 1
    if args.workload == "batched":
        return run_reference_batched(args, threads)
    case, wname = make_case(args)
    o = mhy_oracle.Oracle(case, pow_mode="libm", threads=threads)
    t0 = time.perf_counter()
    o.step(max(1, args.warmup))
    per = (time.perf_counter() - t0) / max(1, args.warmup)
    budget_s = 90.0
    k = max(1, min(args.steps, int(budget_s / max(per, 1e-6))))
    t0 = time.perf_counter()
    o.step(k)
    el = time.perf_counter() - t0
    val = case.ncells * k / el
    sample = (f"{wname}, {k} of {args.steps} requested cycles timed after {max(1, args.warmup)} warm-up "
              f"(bounded to ~{budget_s:.0f} s), OpenMP {threads} threads")
    line = {"metric": METRIC, "value": val, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
            "steps": k, "warmup": max(1, args.warmup), "ms_per_step": el / k * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wname, "cells": case.ncells, "nodes": case.nnodes},
            "cpu_baseline": {"value": val, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def apply_tuning(obj, args):
    """Autotune (default), a fixed --tune-lines setting, or nothing; returns
    the tuning for the JSON line."""
    import mhy_b200
    if args.tune_lines:
        t = mhy_b200.CTuning.default()
        for slot, w in zip((3, 4, 6, 7), (int(x) for x in args.tune_lines.split(","))):
            t.lines_per_block[slot] = w
        obj.set_tuning(t)
        d = obj.tuning().as_dict()
        d["set_by"] = "--tune-lines"
        return d
    if args.no_autotune:
        return None
    t = obj.autotune(2)                                 # trials on this state, restored; outside the timed region
    d = t.as_dict()
    d["cycle_ms_default"] = round(sum(t.ms_default), 3)
    d["cycle_ms_tuned"] = round(sum(t.ms_tuned), 3)
    return d


def conservation(t0, t1, cycles):
    """Drift of the conserved totals over the run: t0, t1 are lists of
    mhy_get_totals results (one per instance) before and after."""
    import math
    m0, m1 = math.fsum(t["mass"] for t in t0), math.fsum(t["mass"] for t in t1)
    e0, e1 = math.fsum(t["total_energy"] for t in t0), math.fsum(t["total_energy"] for t in t1)
    return {"mass_drift_rel": (m1 - m0) / m0, "total_energy_drift_rel": (e1 - e0) / e0, "cycles": cycles,
            "sum": "compensated TwoSum on the device (mhy_get_totals), fixed order"}


def mixed_accuracy(cases, densities, cycles, device, batched=False, totals=None):
    """Density L1 error of the mixed-precision run against the FP64 path on the
    same inputs and cycle count (the FP64 device path equals the oracle bit for
    bit, which the GPU parity tests check): sum |rho_mixed - rho_fp64| / sum |rho_fp64|;
    with totals (the mixed run's mhy_get_totals per instance), the relative
    difference of total mass and total energy from the FP64 run's."""
    import copy
    import math
    import numpy as np
    import mhy_b200
    ref_cases = []
    for c in cases:
        r = copy.copy(c)
        r.options = copy.copy(c.options)
        r.options.precision = 0
        ref_cases.append(r)
    if batched:
        b = mhy_b200.Batch(ref_cases, device=device)
        b.step(cycles)
        refs = [b.field(i, "density") for i in range(len(ref_cases))]
        ref_tot = [b.totals(i) for i in range(len(ref_cases))]
        b.close()
    else:
        g = mhy_b200.Context(ref_cases[0], device=device)
        g.step(cycles)
        refs = [g.field("density")]
        ref_tot = [g.totals()]
        g.close()
    num = math.fsum(float(np.abs(a - r).sum()) for a, r in zip(densities, refs))
    den = math.fsum(float(np.abs(r).sum()) for r in refs)
    out = {"density_l1_rel_vs_fp64": num / den, "cycles": cycles,
           "reference": "FP64 device path on the same inputs (bitwise equal to the CPU oracle)"}
    if totals is not None:
        for key, q in (("mass_rel_vs_fp64", "mass"), ("total_energy_rel_vs_fp64", "total_energy")):
            a = math.fsum(t[q] for t in totals)
            r = math.fsum(t[q] for t in ref_tot)
            out[key] = (a - r) / r
    return out


def run_reference_batched(args, threads):
    """--impl reference --workload batched: the instances advanced one after
    the other on the host cores by the oracle, a bounded sample: every
    instance in turn for two cycles until the time budget is spent."""
    import mhy_oracle
    from mhy_b200 import gen
    cases = gen.batched()
    budget_s, done, el, n_inst = 90.0, 0, 0.0, 0
    for c in cases:
        o = mhy_oracle.Oracle(c, pow_mode="libm", threads=threads)
        o.step(1)
        t0 = time.perf_counter()
        o.step(2)
        el += time.perf_counter() - t0
        done += 2 * c.ncells
        n_inst += 1
        o.close()
        if el > budget_s:
            break
    val = done / el
    sample = (f"{n_inst} of {len(cases)} instances, 2 cycles each after 1 untimed cycle "
              f"(bounded to ~{budget_s:.0f} s), OpenMP {threads} threads")
    line = {"metric": METRIC, "value": val, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
            "steps": 2, "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batched-64-sod-sedov-32..96^3-fp64", "instances": len(cases),
                       "cells": sum(c.ncells for c in cases)},
            "cpu_baseline": {"value": val, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours_batched(args):
    """The batched form: 64 independent uneven instances in one set of
    persistent launches per cycle, per-instance dt on the device.  With N GPUs
    the instance list is split by cell count (replicas.partition; strong
    scaling: the job is fixed)."""
    import numpy as np
    import torch
    import mhy_b200
    from mhy_b200 import gen, bytes_model, replicas

    world, rank, local = replicas.ranks()
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        replicas.init("nccl", device=dev)
    all_cases = gen.batched()
    for c in all_cases:
        c.options.precision = 0 if args.precision == "fp64" else 1
    mine = [all_cases[i] for i in replicas.partition([c.ncells for c in all_cases], world, rank)]
    cells = sum(c.ncells for c in mine)
    b = mhy_b200.Batch(mine, device=local)
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    tot0 = [b.totals(i) for i in range(len(mine))]
    tuning = apply_tuning(b, args)
    b.step(args.warmup)
    b.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        replicas.barrier()
        torch.cuda.synchronize()
        start.record(stream)
        b.step(args.steps)
        stop.record(stream)
        torch.cuda.synchronize()
        replicas.barrier()
    ms, value = replicas.aggregate(cells, args.steps, start.elapsed_time(stop), dev)
    status = max(b.status(i) for i in range(len(mine)))
    kpc = b.kernels_per_cycle()
    tot1 = [b.totals(i) for i in range(len(mine))]
    cons = conservation(tot0, tot1, args.warmup + args.steps)
    accuracy = None
    if args.precision == "mixed":
        accuracy = mixed_accuracy(mine, [b.field(i, "density") for i in range(len(mine))],
                                  args.warmup + args.steps, local, batched=True, totals=tot1)
    b.close()

    e2e = None
    if not args.no_e2e:
        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()
        hcases = [gen.Case(c.name, c.nx, c.ny, c.nz, pinned(c.coords), c.gamma, pinned(c.fracvol), pinned(c.density),
                           pinned(c.pressure), pinned(c.velocity), c.options, c.cycles) for c in mine]
        outs = [(pinned(np.zeros(c.ncells)), pinned(np.zeros(c.ncells)), pinned(np.zeros((c.nnodes, 3))))
                for c in mine]
        L = mhy_b200.load()
        replicas.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b2 = mhy_b200.Batch(hcases, device=local)
        apply_tuning(b2, args)                             # the cached choice for these mesh sizes
        for _ in range(args.steps):
            b2.step(1)
            b2.dt(0)                                   # D2H of a step result + sync, every cycle
        for i, (r, e, v) in enumerate(outs):
            for name, arr in (("density", r), ("internal_energy", e), ("velocity", v)):
                mhy_b200._check(L.mhy_batch_get_field(b2.h, i, mhy_b200.FIELDS[name],
                                                      arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes))
        el = time.perf_counter() - t0
        b2.close()
        el_ms, e2e_value = replicas.aggregate(cells, args.steps, el * 1e3, dev)
        h2d = sum(c.coords.nbytes + c.fracvol.nbytes + c.density.nbytes + c.pressure.nbytes + c.velocity.nbytes
                  for c in mine) / args.steps
        d2h = 16 + sum(r.nbytes + e.nbytes + v.nbytes for r, e, v in outs) / args.steps
        e2e = {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": round(h2d, 1),
               "d2h_bytes_per_step": round(d2h, 1),
               "path": "mhy_batch_create+set_state+hydro_start_init, per-cycle mhy_batch_step + mhy_batch_get_dt, "
                       "mhy_batch_get_field x3 per instance; wall clock, max over ranks"}

    b_cells = sum(c.ncells * bytes_model.bytes_per_cell_cycle(c.ncells, c.nnodes) for c in mine)
    peak, peak_kind = measured_peak()
    achieved = b_cells * args.steps / (ms / 1e3) / 1e9 / (world if world > 1 else 1)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": peak_kind,
                "kernel": f"one batched cycle graph ({kpc} persistent launches), algorithmic bytes "
                          f"{b_cells / cells:.1f} B/cell-cycle averaged over this GPU's instances"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(mine[1], args.cpu_sample_cycles, f"batch instance 1 ({mine[1].nx}^3 Sedov)")
    if rank == 0:
        total = sum(c.ncells for c in all_cases)
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"batched-64-sod-sedov-32..96^3-{'fp64' if args.precision == 'fp64' else 'mixed'}",
                           "instances": len(all_cases),
                           "cells": total, "cells_per_gpu": cells, "parallelism": f"instances split over {world}",
                           "l2": "working set > 126 MB L2 (no flush needed)", "tuning": tuning},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": kpc * args.steps,
                "clocks": clk.summary(), "device_status": status, "conservation": cons}
        if accuracy:
            line["accuracy"] = accuracy
            line["dtype"] = "f32 remap evaluation / f64 state"
        print(json.dumps(line), flush=True)
    replicas.finish()
    return 0


def run_ours(args):
    import numpy as np
    import torch
    import mhy_b200
    from mhy_b200 import gen, bytes_model, replicas

    world, rank, local = replicas.ranks()
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        replicas.init("nccl", device=dev)

    case, wname = make_case(args)
    ctx = mhy_b200.Context(case, device=local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
    kpc = ctx.kernels_per_cycle()
    tot0 = [ctx.totals()]
    tuning = apply_tuning(ctx, args)

    ctx.step(args.warmup)
    ctx.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        replicas.barrier()
        torch.cuda.synchronize()
        start.record(stream)
        ctx.step(args.steps)
        stop.record(stream)
        torch.cuda.synchronize()
        replicas.barrier()
    ms_local = start.elapsed_time(stop)
    ctx.synchronize()
    status = ctx.status()
    ms, value = replicas.aggregate(case.ncells, args.steps, ms_local, dev)
    tot1 = [ctx.totals()]
    cons = conservation(tot0, tot1, args.warmup + args.steps)
    accuracy = None
    if args.precision == "mixed":
        accuracy = mixed_accuracy([case], [ctx.field("density")], args.warmup + args.steps, local, totals=tot1)
    ctx.close()

    # end to end through the per-entry-point C ABI, host buffers in pinned memory
    e2e = None
    if not args.no_e2e:
        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()
        hcase = gen.Case(case.name, case.nx, case.ny, case.nz, pinned(case.coords), case.gamma,
                         pinned(case.fracvol), pinned(case.density), pinned(case.pressure), pinned(case.velocity),
                         case.options, case.cycles)
        out_rho = pinned(np.zeros(case.ncells)); out_e = pinned(np.zeros(case.ncells))
        out_v = pinned(np.zeros((case.nnodes, 3)))
        L = mhy_b200.load()
        replicas.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c2 = mhy_b200.Context(hcase, device=local)
        apply_tuning(c2, args)                             # the cached choice for this mesh size
        for _ in range(args.steps):
            c2.cycle_by_entry_points()
            c2.dt()                                   # D2H of the step's result (dt, 16 B) + sync
        for name, arr in (("density", out_rho), ("internal_energy", out_e), ("velocity", out_v)):
            mhy_b200._check(L.mhy_get_field(c2.h, mhy_b200.FIELDS[name], arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes))
        el_local = time.perf_counter() - t0
        c2.close()
        el_ms, e2e_value = replicas.aggregate(case.ncells, args.steps, el_local * 1e3, dev)
        h2d = (case.coords.nbytes + case.fracvol.nbytes + case.density.nbytes + case.pressure.nbytes
               + case.velocity.nbytes) / args.steps
        d2h = 16 + (out_rho.nbytes + out_e.nbytes + out_v.nbytes) / args.steps
        e2e = {"value": e2e_value, "unit": METRIC,
               "h2d_bytes_per_step": round(h2d, 1), "d2h_bytes_per_step": round(d2h, 1),
               "path": "mhy_create+mhy_set_state+mhy_hydro_start_init, per-cycle entry points + mhy_get_dt, "
                       "mhy_get_field x3; wall clock, max over ranks"}

    mixed_fraction = float(((case.fracvol > 0).sum(0) > 1).mean()) if case.nenv > 1 else 0.0
    b_alg = bytes_model.bytes_per_cell_cycle(case.ncells, case.nnodes, case.nenv, mixed_fraction)
    peak, peak_kind = measured_peak()
    per_gpu_cells_per_s = case.ncells * args.steps / (ms / 1e3)
    achieved = b_alg * per_gpu_cells_per_s / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": TRAFFIC_PER_CYCLE.get((args.workload, args.n, args.precision)),
                "algorithmic_bytes_per_launch": round(b_alg * case.ncells, 1),
                "kernel": f"one cycle graph ({kpc} kernels, launched as one unit), algorithmic bytes "
                          f"{b_alg:.1f} B/cell-cycle x {case.ncells} cells; traffic = DRAM bytes of one cycle (ncu)",
                "peak_kind": peak_kind}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(case, args.cpu_sample_cycles, wname)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": wname, "cells": case.ncells, "nodes": case.nnodes,
                           "environments": case.nenv,
                           "cells_per_gpu": case.ncells, "parallelism": f"replicas{world}",
                           "l2": "working set > 1 GB, far above the 126 MB L2 (no flush needed)",
                           "tuning": tuning},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": kpc * args.steps, "clocks": clk.summary(), "device_status": status,
                "conservation": cons}
        if accuracy:
            line["accuracy"] = accuracy
            line["dtype"] = "f32 remap evaluation / f64 state"
        print(json.dumps(line), flush=True)
    replicas.finish()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_ours_batched(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
