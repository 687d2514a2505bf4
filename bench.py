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
path has no data exchange between independent meshes); with --slabs the one
mesh is split along z over the N GPUs instead (strong scaling: ghost layers,
one NCCL dt all-reduce and one halo exchange per cycle).

Beside the timed number, the default line carries `parity` (a fresh context
stepped cycle by cycle against the CPU oracle with the C library's pow, over
the same cycles as the timed run when they are at most --parity-cycles:
relative L-inf of density, energy and velocity, dt-sequence difference, and
whether the timed run's fields equal that context's bit for bit),
`cpu_baseline` (the same oracle run's wall time on all host cores, plus one
cycle on one thread, with the CPU model) and `forms` (the mixed-precision
Sedov mesh and the 64-instance batched sweep in FP64 and mixed, same cycles,
with their ratios to this line and the mixed forms' errors).
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
    ap.add_argument("--parity-cycles", type=int, default=60,
                    help="cycles of the parity check against the libm-pow oracle (capped at warmup + steps; "
                         "0 = no parity check)")
    ap.add_argument("--slabs", action="store_true",
                    help="split the one mesh along z over the N GPUs (ghost layers, one dt all-reduce and one "
                         "halo exchange per cycle over NCCL; strong scaling) instead of N independent replicas")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the mixed-precision and batched figures of the default line")
    return ap.parse_args()


# DRAM bytes (read + write) of one whole cycle, summed over its kernels
# (dram__bytes_read.sum + dram__bytes_write.sum from one ncu capture of the
# 128^3 Sedov cycle), with the digest of the kernel sources they were measured
# on: after any change to those sources the figure is reported as stale (null).
TRAFFIC_PER_CYCLE = {("sedov", 128, "fp64"): (3460821504.0, "1fee7bc5e6c8a96c"),
                     ("sedov", 128, "mixed"): (2910358272.0, "1fee7bc5e6c8a96c")}
KERNEL_SOURCES = ("mhy_kernels.cuh", "mhy_device.cuh", "mhy_pow_third.h", "mhy_line.cuh", "mhy_lagrange.cuh",
                  "mhy_kernels.cu", "mhy_cycle.cu", "mhy_multi.cu")


def kernel_sources_digest():
    import hashlib
    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        h.update((ROOT / "arcane-benchs_b200" / "csrc" / name).read_bytes())
    return h.hexdigest()[:16]


def cycle_traffic(key):
    """(traffic bytes or None, note)."""
    entry = TRAFFIC_PER_CYCLE.get(key)
    if entry is None:
        return None, "no ncu capture of this workload"
    traffic, digest = entry
    if digest != kernel_sources_digest():
        return None, "stale: the kernel sources changed since the ncu capture"
    return traffic, f"ncu capture on kernel sources {digest}"


def cpu_info():
    model = None
    try:
        for line in pathlib.Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


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


def single_thread(o, case):
    """One more cycle of an oracle on one thread (the oracle's thread count is
    process-wide, so it is restored afterwards)."""
    import mhy_oracle
    threads = os.cpu_count() or 1
    mhy_oracle.lib().orc_set_threads(1)
    t0 = time.perf_counter()
    o.step(1)
    el = time.perf_counter() - t0
    mhy_oracle.lib().orc_set_threads(threads)
    return {"value": case.ncells / el, "unit": METRIC, "cores": 1, "cycles": 1,
            "sample": "one cycle after the all-core sample, 1 OpenMP thread"}


def cpu_baseline(case, cycles, wname):
    """The oracle (CPU restatement of the reference algorithm) on this host:
    all cores, then one thread."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import mhy_oracle
    threads = os.cpu_count() or 1
    o = mhy_oracle.Oracle(case, pow_mode="libm", threads=threads)
    o.step(1)  # first cycle (page faults, thread start) not timed
    t0 = time.perf_counter()
    o.step(cycles)
    dt = time.perf_counter() - t0
    one = single_thread(o, case)
    o.close()
    return {"value": case.ncells * cycles / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{wname} (same mesh and state), cycles 2..{cycles + 1} after init, "
                      f"OpenMP {threads} threads, oracle built -O3 -ffp-contract=off",
            "single_thread": one, **cpu_info()}


def oracle_leg(case, wname, cycles, device, timed=None, want_cpu=True):
    """Parity and CPU baseline from one run of the oracle with the C library's
    pow (the reference's V^(1/3.), MahycoModule.cc:1259) on all host cores.

    Parity: a fresh FP64 context on the GPU, stepped one cycle at a time with
    its dt read back each cycle, against the oracle over `cycles` cycles from
    the same initial state: relative L-inf of density, specific internal energy
    and node velocity, and the largest relative difference of the dt sequence.
    When `timed` (the timed run's final fields, after the same number of
    cycles) is given, the timed run is also compared with that context bit for
    bit.  CPU baseline: the oracle's own wall time for cycles 2..cycles, then
    one cycle on one thread."""
    import numpy as np
    import mhy_b200
    sys.path.insert(0, str(ROOT / "oracle"))
    import mhy_oracle
    threads = os.cpu_count() or 1
    g = mhy_b200.Context(case, device=device)
    dtg = [g.dt()[0]]
    for _ in range(cycles):
        g.step(1)
        dtg.append(g.dt()[0])
    g.synchronize()
    gf = {f: g.field(f) for f in ("density", "internal_energy", "velocity")}
    g.close()
    o = mhy_oracle.Oracle(case, pow_mode="libm", threads=threads)
    dto = [o.scalars()["dt"]]
    o.step(1)                                          # first cycle (page faults, thread start) not timed
    dto.append(o.scalars()["dt"])
    t0 = time.perf_counter()
    for _ in range(cycles - 1):
        o.step(1)
        dto.append(o.scalars()["dt"])
    el = time.perf_counter() - t0

    def rel_linf(a, b):
        s = float(np.max(np.abs(b)))
        return float(np.max(np.abs(a - b))) / (s if s > 0 else 1.0)

    dto, dtg = np.array(dto), np.array(dtg)
    errs = {f"{f}_rel_linf": rel_linf(gf[f], o.field(f)) for f in gf}
    dt_err = float(np.max(np.abs(dtg - dto) / dto))
    parity = {"cycles": cycles, **errs, "dt_sequence_max_rel": dt_err,
              "bar": {"fields_rel_linf": 1e-10, "dt_rel": 1e-12},
              "within_bar": bool(max(errs.values()) <= 1e-10 and dt_err <= 1e-12),
              "reference": f"CPU oracle with libm pow, OpenMP {threads} threads; GPU context stepped cycle by cycle"}
    if timed is not None:
        parity["timed_run_bitwise_equal"] = bool(all(np.array_equal(timed[f], gf[f]) for f in gf))
    cpu = None
    if want_cpu and cycles >= 2:
        cpu = {"value": case.ncells * (cycles - 1) / el, "unit": METRIC, "cores": threads, "kind": "port",
               "sample": f"{wname} (same mesh and state), cycles 2..{cycles} of the parity run, "
                         f"OpenMP {threads} threads, oracle built -O3 -ffp-contract=off",
               "single_thread": single_thread(o, case), **cpu_info()}
    o.close()
    return parity, cpu


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
            "cpu_baseline": {"value": val, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample,
                             **cpu_info()},
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
    timed_fields = {f: ctx.field(f) for f in ("density", "internal_energy", "velocity")}
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
                       "mhy_get_field x3; wall clock, max over ranks",
               "tuning": "the autotuner's in-process cache for this mesh size (filled by the device-timed run "
                         "above); a first-time caller pays the trials once"
                         + (f", {tuning['cycle_ms_default'] * 3 * (tuning.get('trials') or 0):.1f} ms of "
                            "device time here" if tuning and 'cycle_ms_default' in tuning else "")}

    mixed_fraction = float(((case.fracvol > 0).sum(0) > 1).mean()) if case.nenv > 1 else 0.0
    b_alg = bytes_model.bytes_per_cell_cycle(case.ncells, case.nnodes, case.nenv, mixed_fraction)
    peak, peak_kind = measured_peak()
    per_gpu_cells_per_s = case.ncells * args.steps / (ms / 1e3)
    achieved = b_alg * per_gpu_cells_per_s / 1e9
    traffic, traffic_note = cycle_traffic((args.workload, args.n, args.precision))
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": traffic, "traffic_note": traffic_note,
                "algorithmic_bytes_per_launch": round(b_alg * case.ncells, 1),
                "kernel": f"one cycle graph ({kpc} kernels, launched as one unit), algorithmic bytes "
                          f"{b_alg:.1f} B/cell-cycle x {case.ncells} cells; traffic = DRAM bytes of one cycle (ncu)",
                "peak_kind": peak_kind}

    cpu, parity = None, None
    total_cycles = args.warmup + args.steps
    pcycles = min(args.parity_cycles, total_cycles)
    if rank == 0 and world == 1 and args.precision == "fp64" and pcycles > 0:
        parity, cpu = oracle_leg(case, wname, pcycles, local, timed_fields if pcycles == total_cycles else None,
                                 want_cpu=not args.no_cpu_baseline)
    if cpu is None and rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(case, args.cpu_sample_cycles, wname)
    forms = None
    if (rank == 0 and world == 1 and not args.no_forms and args.workload == "sedov" and args.precision == "fp64"):
        forms = measure_forms(args, local, value, timed_fields["density"], tot1[0])

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
        if parity:
            line["parity"] = parity
        if forms:
            line["forms"] = forms
        if accuracy:
            line["accuracy"] = accuracy
            line["dtype"] = "f32 remap evaluation / f64 state"
        print(json.dumps(line), flush=True)
    replicas.finish()
    return 0


def timed_cycles(obj, args, device):
    """Warm-up, then args.steps cycles timed with CUDA events on the object's
    stream (a Context or a Batch); returns ms."""
    import torch
    stream = torch.cuda.ExternalStream(obj.stream(), device=torch.device("cuda", device))
    obj.step(args.warmup)
    obj.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    obj.step(args.steps)
    stop.record(stream)
    torch.cuda.synchronize()
    obj.synchronize()
    return start.elapsed_time(stop)


def measure_forms(args, device, plain_value, plain_density, plain_totals):
    """The two production forms beside the plain FP64 Sedov line, over the
    same warm-up and timed cycles: the mixed-precision Sedov mesh, and the
    64-instance batched sweep (32^3..96^3, one persistent launch per kernel
    per cycle) in FP64 and mixed.  Each gives its cell-cycles/s and its ratio
    to the plain line; the mixed forms add the density L1 error against the
    FP64 path on the same inputs (that path equals the oracle bit for bit) and
    the relative differences of total mass and total energy."""
    import math
    import numpy as np
    import mhy_b200
    from mhy_b200 import gen
    cycles = args.warmup + args.steps

    def l1(a_list, r_list):
        num = math.fsum(float(np.abs(a - r).sum()) for a, r in zip(a_list, r_list))
        den = math.fsum(float(np.abs(r).sum()) for r in r_list)
        return num / den

    def rel(a, r):
        return (a - r) / r

    out = {"cycles_timed": args.steps, "cycles_total": cycles, "plain_fp64_value": plain_value}
    # mixed-precision Sedov
    case = gen.sedov(n=args.n)
    case.options.precision = 1
    ctx = mhy_b200.Context(case, device=device)
    apply_tuning(ctx, args)
    ms = timed_cycles(ctx, args, device)
    val = case.ncells * args.steps / (ms / 1e3)
    tm = ctx.totals()
    out["mixed_sedov"] = {"workload": f"sedov-{args.n}^3-jitter1%-mixed", "value": val, "ms_per_step": ms / args.steps,
                          "vs_plain_fp64": val / plain_value,
                          "density_l1_rel_vs_fp64": l1([ctx.field("density")], [plain_density]),
                          "mass_rel_vs_fp64": rel(tm["mass"], plain_totals["mass"]),
                          "total_energy_rel_vs_fp64": rel(tm["total_energy"], plain_totals["total_energy"]),
                          "device_status": ctx.status()}
    ctx.close()
    # batched sweep, FP64 then mixed
    res = {}
    for prec in (0, 1):
        cases = gen.batched()
        for c in cases:
            c.options.precision = prec
        b = mhy_b200.Batch(cases, device=device)
        apply_tuning(b, args)
        ms = timed_cycles(b, args, device)
        cells = sum(c.ncells for c in cases)
        res[prec] = {"value": cells * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                     "density": [b.field(i, "density") for i in range(len(cases))],
                     "totals": [b.totals(i) for i in range(len(cases))],
                     "status": max(b.status(i) for i in range(len(cases)))}
        b.close()
    for prec, name in ((0, "batched_fp64"), (1, "batched_mixed")):
        r = res[prec]
        out[name] = {"workload": f"batched-64-sod-sedov-32..96^3-{'fp64' if prec == 0 else 'mixed'}",
                     "value": r["value"], "ms_per_step": r["ms_per_step"], "vs_plain_fp64": r["value"] / plain_value,
                     "device_status": r["status"]}
    f64, mx = res[0], res[1]
    out["batched_mixed"]["vs_batched_fp64"] = mx["value"] / f64["value"]
    out["batched_mixed"]["density_l1_rel_vs_fp64"] = l1(mx["density"], f64["density"])
    for key, q in (("mass_rel_vs_fp64", "mass"), ("total_energy_rel_vs_fp64", "total_energy")):
        a = math.fsum(t[q] for t in mx["totals"])
        r = math.fsum(t[q] for t in f64["totals"])
        out["batched_mixed"][key] = rel(a, r)
    out["target"] = "mixed batched >= 1.6x the plain FP64 path at density L1 <= 1e-5"
    return out


def run_ours_slabs(args):
    """--slabs: the workload's mesh split along z over the N GPUs
    (mhy_b200/slabs.py).  Each rank advances its slab plus ghost layers; per
    cycle one NCCL all-reduce (min) of the dt bit patterns and one halo
    exchange (send/recv of the neighbours' boundary layers), both ordered on
    the context's stream.  value = the whole mesh's cell-cycles/s (owned cells
    only; the ghost layers' recomputation is overhead), max time over ranks."""
    import torch
    from mhy_b200 import bytes_model, replicas, slabs

    world, rank, local = replicas.ranks()
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        replicas.init("nccl", device=dev)
    case, wname = make_case(args)
    lay = slabs.layout(case.nz, world)
    rk = slabs.SlabRank(case, lay, rank, lambda c: slabs.GpuEngine(c, local))
    ctx = rk.eng.ctx
    tuning = apply_tuning(ctx, args)
    kpc = ctx.kernels_per_cycle() + 1                     # + the dt finish from the combined minimum
    slabs.run_distributed(rk, args.warmup)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        replicas.barrier()
        torch.cuda.synchronize()
        start.record(rk.eng.stream)
        slabs.run_distributed(rk, args.steps)
        stop.record(rk.eng.stream)
        torch.cuda.synchronize()
        replicas.barrier()
    owned_cells = rk.s.own * case.nx * case.ny
    ms, value = replicas.aggregate(owned_cells, args.steps, start.elapsed_time(stop), dev)
    status = ctx.status()
    b_alg = bytes_model.bytes_per_cell_cycle(case.ncells, case.nnodes)
    peak, peak_kind = measured_peak()
    achieved = b_alg * value / 1e9 / world
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32 remap evaluation / f64 state",
                "data": "synthetic",
                "config": {"workload": f"{wname}-slabs{world}", "cells": case.ncells, "nodes": case.nnodes,
                           "parallelism": f"z-slabs over {world} GPUs, {slabs.GHOST} ghost layers a side",
                           "slab_layers": [s.own for s in lay],
                           "l2": "working set > 126 MB L2 (no flush needed)", "tuning": tuning},
                "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": peak_kind,
                             "kernel": "one slab cycle per GPU (graph) + dt finish; algorithmic bytes of the owned "
                                       f"cells, {b_alg:.1f} B/cell-cycle"},
                "cpu_baseline": None, "e2e": None, "gpu_launches": kpc * args.steps, "clocks": clk.summary(),
                "device_status": status}
        print(json.dumps(line), flush=True)
    rk.eng.close()
    replicas.finish()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.slabs:
        return run_ours_slabs(args)
    if args.workload == "batched":
        return run_ours_batched(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
