#!/usr/bin/env python
"""AMOEBA energy+gradient throughput on the 24,000-atom water box (one B200 per rank).

One step = one full energy + gradient evaluation (vdW + PME multipoles + mutual
polarization solved by PCG to 1e-6 D RMS + torques) of 8,000 AMOEBA waters in a
62.08 A cube, PME 64^3 order 5, 7 A real space, 9 A vdW.  The system does not
shard (a 24k-atom PME evaluation is latency-bound on one GPU), so N GPUs run N
independent replicas: value = N * steps / (max over ranks of the timed seconds).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision both|fp64|mixed]

By default both forms run; the headline value is the mixed-precision form and the
plain FP64 form is reported beside it under "fp64".  A batch of 512 small systems
(96-3,000 atoms each) is timed beside it under "batch" (one-graph batch vs a loop of
single-system launches; --batch-systems 0 skips it).
  python bench.py --impl reference ...   # the CPU FP64 restatement on the host cores
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from forcefieldx_b200.system import (PRECISION_FP64, PRECISION_MIXED, WATER_24K,  # noqa: E402
                                     water_box, water_params)

METRIC = "AMOEBA energy+gradient evals/s, 24k-atom water box"
UNIT = "evals/s"
WORKLOAD = ("AMOEBA water, 8,000 molecules (24,000 atoms), 62.08 A cubic P1 box, seeded jittered lattice; "
            "PME 64^3 order 5, ewald-alpha 0.545, 7 A real space, 9 A buffered-14-7 vdW, 2 A list buffer; "
            "mutual polarization, PCG to 1e-6 D RMS")


def build_system():
    s = water_box(WATER_24K["n_side"], WATER_24K["edge"])
    return s


def build_params(precision: int):
    return water_params(WATER_24K["edge"], pme_grid=WATER_24K["grid"], precision=precision)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# Algorithmic work of one launch of a stage's dominant kernel, frozen in BASELINE.md: the
# compulsory HBM bytes of a pass (every per-atom input read once, every output written
# once; neighbour lists are derived data and not counted) and the FLOPs of the pair
# arithmetic, per undirected pair.
BYTES_PER_ATOM = {"ind_field": 150.0, "precond": 150.0, "real_energy": 240.0, "vdw": 80.0}
FLOPS_PER_PAIR = {"ind_field": 110.0, "precond": 110.0, "real_energy": 900.0, "vdw": 70.0}


def algorithmic_work(stage: str, n: int, pairs_half: int, vdw_pairs: int):
    """(compulsory bytes, FLOPs) of one launch of the stage's dominant kernel."""
    pairs = vdw_pairs if stage == "vdw" else pairs_half
    return BYTES_PER_ATOM[stage] * n, FLOPS_PER_PAIR[stage] * pairs


def fma_peak_tflops(fp64: bool):
    """FMA-pipe throughput of this GPU measured by libffxpeak.so (best of five launches)."""
    import ctypes
    path = os.path.join(ROOT, "forcefieldx_b200", "libffxpeak.so")
    lib = ctypes.CDLL(path)
    lib.ffxpeak_fma_tflops.restype = ctypes.c_int
    lib.ffxpeak_fma_tflops.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    tf = ctypes.c_double(0.0)
    if lib.ffxpeak_fma_tflops(1 if fp64 else 0, ctypes.byref(tf), None) != 0:
        raise RuntimeError("FMA peak microkernel failed")
    return tf.value


def measure(args, precision, system, dist, world, local):
    """Device-resident timing of one precision form, plus the end-to-end host-buffer run."""
    import torch
    from forcefieldx_b200.energy import ForceFieldEnergy
    from forcefieldx_b200 import cabi

    mixed = precision == PRECISION_MIXED
    params = build_params(precision)
    n = system.n_atoms
    ffe = ForceFieldEnergy(system, params)
    stream = torch.cuda.ExternalStream(ffe.stream)
    d_xyz = torch.tensor(system.xyz, dtype=torch.float64, device="cuda")
    d_grad = torch.empty_like(d_xyz)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > 126 MB L2

    for _ in range(args.warmup):
        ffe.energy_device(d_xyz.data_ptr(), d_grad.data_ptr())
    torch.cuda.synchronize()
    scf = ffe.count("scf_iter")
    pairs_half = ffe.count("permanent") - n
    terms = [float(t) for t in ffe.terms]

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms = 0.0
    launches = 0
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.steps):
        flush.zero_()                       # evict L2 between steps (untimed)
        torch.cuda.synchronize()
        start.record(stream)
        ffe.energy_device(d_xyz.data_ptr(), d_grad.data_ptr())
        end.record(stream)
        end.synchronize()
        total_ms += start.elapsed_time(end)
        launches += ffe.launch_count()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    # Stage breakdown from a separate, untimed pass: stage timing brackets every stage
    # with events and therefore runs the kernels as direct launches, not as the graph.
    ffe.lib.ffxg_set_timing(ffe._h, 1)
    for _ in range(args.steps):
        flush.zero_()
        ffe.energy_device(d_xyz.data_ptr(), d_grad.data_ptr())
    torch.cuda.synchronize()
    stage_ms = np.zeros(len(cabi.STAGE_NAMES))
    stage_n = np.zeros(len(cabi.STAGE_NAMES), dtype=np.int64)
    ffe.lib.ffxg_get_timings(ffe._h, stage_ms.ctypes.data_as(cabi._D), stage_n.ctypes.data_as(cabi._L), 12)
    ffe.lib.ffxg_set_timing(ffe._h, 0)
    t_max = total_ms
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    value = world * args.steps / (t_max / 1000.0)

    # Dominant pair stage and its roofline: compulsory bytes and algorithmic FLOPs of one
    # launch over the stage's measured average launch time (the kernel alone on the stream),
    # against the measured HBM copy bandwidth and the measured FMA-pipe throughput.
    kernel_stages = ["vdw", "ind_field", "real_energy"]
    per_stage = {cabi.STAGE_NAMES[i]: {"ms_total": float(stage_ms[i]), "launches": int(stage_n[i])}
                 for i in range(12)}
    dom = max(kernel_stages, key=lambda st: per_stage[st]["ms_total"])
    avg_ms = per_stage[dom]["ms_total"] / max(1, per_stage[dom]["launches"])
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    bytes_alg, flops_alg = algorithmic_work(dom, n, pairs_half, ffe.count("vdw"))
    achieved = bytes_alg / (avg_ms * 1e-3) / 1e9
    fp_peak = fma_peak_tflops(fp64=not mixed)
    fp_achieved = flops_alg / (avg_ms * 1e-3) / 1e12

    # End to end through the public API with host buffers (H2D coordinates, D2H gradient).
    x_host = np.ascontiguousarray(system.xyz)
    g_host = np.zeros_like(x_host)
    ffe.energy_and_gradient(x_host, g_host)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_steps = max(3, args.steps // 2)
    for _ in range(e2e_steps):
        ffe.energy_and_gradient(x_host, g_host)
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(n * 3 * 8),
           "d2h_bytes_per_step": int(n * 3 * 8 + 8 * cabi.N_TERMS + 8 * cabi.N_COUNTS),
           "api": "ffxg_energy_and_gradient (host xyz in, host gradient out)"}
    ffe.close()
    del flush
    return {
        "value": value, "ms_per_step": t_max / args.steps, "pcg_iterations": scf, "terms": terms,
        "launches": int(launches), "clocks": clocks, "e2e": e2e,
        "stages_ms_per_step": {k: v["ms_total"] / args.steps for k, v in per_stage.items()},
        "stages_note": "direct launches with per-stage events (the timed steps replay one CUDA graph)",
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None,
                     "kernel_stage": dom, "algorithmic_bytes_per_launch": bytes_alg,
                     "bytes_rule": f"{BYTES_PER_ATOM[dom]:.0f} B per atom per pass (compulsory HBM bytes)",
                     "avg_launch_ms": avg_ms, "peak_source": peak_src,
                     "fp_pipe": {"achieved": fp_achieved, "peak": fp_peak, "unit": "TFLOP/s",
                                 "frac": fp_achieved / fp_peak, "pipe": "FP64 FMA" if not mixed else "FP32 FMA",
                                 "flops_per_launch": flops_alg,
                                 "flops_rule": f"{FLOPS_PER_PAIR[dom]:.0f} FLOPs per undirected pair",
                                 "peak_source": "measured: FMA microkernel (libffxpeak.so) in this run"},
                     "note": "the stage's kernel timed alone on its stream with CUDA events (direct launches); "
                             "traffic: DRAM bytes come from separate ncu captures, not from this run"},
    }


def measure_md(args, system, dist, world, aspc=False):
    """Config 2's dynamics: ``--md-steps`` velocity-Verlet steps of 2 fs with SETTLE rigid
    waters on the device (ffxg_md_run: positions and velocities stay on the GPU, every step
    replays the evaluation graph, the neighbour list is rebuilt whenever an atom has moved
    more than half the buffer), mixed form, velocities drawn at 300 K.  Timed on the host
    clock around the one call, host copies included; ns/day is measured, not extrapolated.
    aspc: with the `scf-predictor ASPC` key (the solve starts from the extrapolation of the
    last six solutions; the reference's default, and the headline's, is no predictor)."""
    import math
    import torch
    from forcefieldx_b200.energy import ForceFieldEnergy
    n = system.n_atoms
    kcal, kb = 418.4, 0.0019872041
    mass = np.where(np.arange(n) % 3 == 0, 15.999, 1.008)
    roh, theta = 0.9572, math.radians(104.52)
    rng = np.random.default_rng(300)
    vel = rng.normal(size=(n, 3)) * np.sqrt(kb * 300.0 * kcal / mass)[:, None]
    with ForceFieldEnergy(system, build_params(PRECISION_MIXED)) as ffe:
        ffe.md_setup(mass, np.arange(n).reshape(-1, 3), roh, 2.0 * roh * math.sin(theta / 2.0))
        if aspc:
            ffe.set_scf_predictor(True)
        x, v, _, _ = ffe.md_run(system.xyz, vel, 0.002, 20)          # warm-up: graphs captured
        if dist:
            dist.barrier()
        builds0 = ffe.list_builds()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x, v, _, _ = ffe.md_run(x, v, 0.002, args.md_steps)
        dt = time.perf_counter() - t0
        builds = ffe.list_builds() - builds0
        if dist:
            t = torch.tensor([dt], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
    return {"steps": args.md_steps, "dt_fs": 2.0, "precision": "mixed", "seconds": dt,
            "ns_per_day": world * args.md_steps * 2e-6 / dt * 86400.0, "steps_per_s": world * args.md_steps / dt,
            "list_builds": int(builds), "scf_predictor": "ASPC" if aspc else "none",
            "method": "ffxg_md_run: velocity Verlet + SETTLE on the device, 300 K start, host clock around the call"}


def run_mine(args):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    system = build_system()
    n = system.n_atoms
    forms = {"fp64": PRECISION_FP64, "mixed": PRECISION_MIXED}
    order = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    runs = {name: measure(args, forms[name], system, dist, world, local) for name in order}
    head_name = order[-1]
    head = runs[head_name]

    md = None
    if args.md_steps > 0:
        md = measure_md(args, system, dist, world)
        md["with_aspc_predictor"] = measure_md(args, system, dist, world, aspc=True)

    batch = None
    if args.batch_systems > 0:
        try:
            batch = measure_batch(args, dist, world, rank)
        except Exception as exc:     # the headline stands without it
            batch = {"error": repr(exc)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(system, build_params(PRECISION_FP64), samples=args.cpu_samples)

    dtype = "f64" if head_name == "fp64" else "mixed: f32 pair/mesh/FFT math, f64 + 64-bit fixed-point accumulation"
    result = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded AMOEBA water box)",
        "config": {"workload": WORKLOAD, "atoms": n, "precision": head_name,
                   "pcg_iterations": head["pcg_iterations"], "energy_kcal_mol": head["terms"][9],
                   "parallelism": f"replicas x{world}", "l2": "flushed between steps (256 MB write, untimed)",
                   "ns_per_day_2fs_from_evals": head["value"] / world * 2e-6 * 86400},
        "roofline": head["roofline"],
        "stages_ms_per_step": head["stages_ms_per_step"],
        "e2e": head["e2e"], "gpu_launches": head["launches"], "clocks": head["clocks"],
    }
    if "fp64" in runs and head_name != "fp64":
        f = runs["fp64"]
        ref_terms = np.array(f["terms"])
        result["fp64"] = {"value": f["value"], "ms_per_step": f["ms_per_step"], "e2e": f["e2e"]["value"],
                          "pcg_iterations": f["pcg_iterations"], "roofline_frac": f["roofline"]["frac"],
                          "stages_ms_per_step": f["stages_ms_per_step"], "clocks": f["clocks"],
                          "gpu_launches": f["launches"]}
        result["mixed_over_fp64"] = head["value"] / f["value"]
        result["mixed_energy_error_vs_fp64_gpu"] = {
            "total_rel": abs(head["terms"][9] - f["terms"][9]) / abs(f["terms"][9]),
            "terms_abs": [abs(a - b) for a, b in zip(head["terms"], ref_terms)]}
    if md:
        result["md"] = md
    if batch:
        result["batch"] = batch
    if cpu:
        result["cpu_baseline"] = cpu
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


def measure_batch(args, dist, world, rank):
    """Many small systems: ``--batch-systems`` water boxes of 96-3,000 atoms (uniform in
    multiples of 3, 29.915 A^3 per molecule, PME grid per system at <= 1.2 A rounded up to
    2,3,5-smooth), mixed precision, energy + gradient of all of them per step through
    BatchEnergy (host coordinates in, host gradients out).  Systems are split over ranks by
    the longest-processing-time rule; one all-reduce gathers the per-system energies.  The
    stage-by-stage graph (the default, with its autotuned number of groups), the graph of
    per-system branches and the loop of single-system launches are timed."""
    import torch
    from forcefieldx_b200.batch import BatchEnergy, batch_workload, partition_lpt, torch_all_reduce
    nsys = args.batch_systems
    w = batch_workload(n_systems=nsys, seed=2026)
    parts = partition_lpt([s.n_atoms for s, _ in w], world)
    mine = parts[rank]
    reduce_sum = torch_all_reduce() if dist else (lambda a: a)
    out = {"systems": nsys, "atoms": int(sum(s.n_atoms for s, _ in w)), "steps": args.batch_steps,
           "metric": "energy+gradient systems/s (e2e: host coordinates in, host gradients out)"}
    with BatchEnergy([w[j][0] for j in mine], [w[j][1] for j in mine]) as b:
        for mode in ("graph", "branches", "loop"):
            b.set_mode(mode)
            for _ in range(3):
                b.energy_and_gradient()
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            for _ in range(args.batch_steps):
                e, _ = b.energy_and_gradient()
            dt = time.perf_counter() - t0
            if dist:
                t = torch.tensor([dt], dtype=torch.float64, device="cuda")
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                dt = float(t.item())
            out[mode] = {"systems_per_s": nsys * args.batch_steps / dt, "ms_per_batch": 1e3 * dt / args.batch_steps}
            if mode == "graph":
                groups, times = b.tuning()
                out[mode]["stages"] = b.stages()
                out[mode]["tuning"] = {"groups": groups, "device_ms_per_batch_by_groups": times}
        table = np.zeros(nsys)
        table[mine] = b.terms[:, 9]
        table = reduce_sum(table)
        out["pcg_iterations_mean"] = float(np.mean(b.counts[:, 2]))
        out["graph_over_loop"] = out["graph"]["systems_per_s"] / out["loop"]["systems_per_s"]
        out["energy_sum_kcal_mol"] = float(np.sum(table))
    return out


def cpu_baseline(system, params, samples=2):
    """The CPU FP64 restatement (oracle) on all host cores: a bounded sample of evaluations."""
    from oracle import binding as ob
    cores = os.cpu_count() or 1
    ob.energy(system, params, nthreads=cores)  # warm-up (page-in, thread pool)
    t0 = time.perf_counter()
    for _ in range(samples):
        ob.energy(system, params, nthreads=cores)
    dt = time.perf_counter() - t0
    return {"value": samples / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{samples} full energy+gradient evaluations of the 24k-atom box after 1 warm-up"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import binding as ob
    system = build_system()
    params = build_params(PRECISION_FP64)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        ob.energy(system, params, nthreads=cores)
    steps = args.steps
    t0 = time.perf_counter()
    for _ in range(steps):
        ob.energy(system, params, nthreads=cores)
    dt = time.perf_counter() - t0
    value = steps / dt
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded AMOEBA water box)",
        "config": {"workload": WORKLOAD, "atoms": system.n_atoms, "precision": "fp64"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{steps} full evaluations after {args.warmup} warm-up (Java reference unavailable: no JDK)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_lambda(args):
    """Electrostatic + vdW lambda evaluations of the 24k box (a 30-atom soft subset, OST:
    three evaluations per call plus the vacuum sub-system), timed on the device per call
    through the public API with host buffers: one JSON line per precision form."""
    import torch
    from forcefieldx_b200.energy import ForceFieldEnergy
    from forcefieldx_b200.system import Alchemy
    torch.cuda.set_device(0)
    system = build_system()
    n = system.n_atoms
    soft = np.zeros(n, dtype=np.int32)
    soft[:30] = 1
    alch = Alchemy(soft=soft, molecule=np.arange(n) // 3, elec=True)
    out = {"workload": WORKLOAD + "; elec-lambdaterm on 30 soft atoms (10 waters)", "lambda": {}}
    for name, prec in (("mixed", PRECISION_MIXED), ("fp64", PRECISION_FP64)):
        with ForceFieldEnergy(system, build_params(prec)) as ffe:
            ffe.set_alchemy(alch)
            res = {}
            for lam in args.lambda_values:
                ffe.set_lambda(lam)
                for _ in range(args.warmup):
                    ffe.energy_and_gradient(system.xyz)
                t0 = time.perf_counter()
                for _ in range(args.steps):
                    e, _ = ffe.energy_and_gradient(system.xyz)
                dt = (time.perf_counter() - t0) / args.steps
                d1, _, _ = ffe.get_dEdL()
                res[str(lam)] = {"evals_per_s": 1.0 / dt, "ms_per_eval": 1e3 * dt, "energy": e, "dEdL": d1,
                                 "pcg_iterations": int(ffe.count("scf_iter"))}
            out["lambda"][name] = res
    print(json.dumps(out))


def run_accuracy(args):
    """Mixed form vs FP64 on frames of a 300 K trajectory of the 24k box.

    The trajectory is run on the device (velocity Verlet + SETTLE, 2 fs, FP64 forces,
    velocity rescaling to 300 K every 10 steps after a hot lattice start); every 10th step
    after equilibration is a frame.  Each frame is evaluated in both forms; the FP64 form
    is itself checked against the CPU oracle on the first and last frames.  Prints one JSON
    line with per-term absolute and relative errors and the force RMS error."""
    import math
    from forcefieldx_b200.energy import ForceFieldEnergy
    from oracle import binding as ob

    system = build_system()
    n = system.n_atoms
    kcal, kb = 418.4, 0.0019872041
    mass = np.where(np.arange(n) % 3 == 0, 15.999, 1.008)
    settle = np.arange(n).reshape(-1, 3)
    roh, theta = 0.9572, math.radians(104.52)
    rhh = 2.0 * roh * math.sin(theta / 2.0)
    dof = 2.0 * n                     # 9 - 3 constraints per water
    rng = np.random.default_rng(300)
    vel = rng.normal(size=(n, 3)) * np.sqrt(kb * 300.0 * kcal / mass)[:, None]
    x = system.xyz.copy()
    frames = []
    with ForceFieldEnergy(system, build_params(PRECISION_FP64)) as md:
        md.md_setup(mass, settle, roh, rhh)
        for chunk in range(args.accuracy_equil // 10 + 10 * args.accuracy_frames // 10):
            x, vel, ep, ek = md.md_run(x, vel, 0.002, 10)
            temp = 2.0 * ek[-1] / (dof * kb)
            vel *= math.sqrt(300.0 / temp)
            if chunk >= args.accuracy_equil // 10:
                frames.append(x.copy())
    frames = frames[:args.accuracy_frames]
    f64 = ForceFieldEnergy(system, build_params(PRECISION_FP64))
    mix = ForceFieldEnergy(system, build_params(PRECISION_MIXED))
    err_terms, rel_total, grad_rms, pins = [], [], [], []
    for k, xf in enumerate(frames):
        _, g64 = f64.energy_and_gradient(xf)
        t64 = f64.terms.copy()
        _, gm = mix.energy_and_gradient(xf)
        tm = mix.terms.copy()
        err_terms.append(np.abs(tm - t64))
        rel_total.append(abs(tm[9] - t64[9]) / abs(t64[9]))
        grad_rms.append(float(np.sqrt(np.mean((gm - g64) ** 2))))
        if k in (0, len(frames) - 1):
            ref = ob.energy(system, build_params(PRECISION_FP64), xyz=xf)
            pins.append({"frame": k, "fp64_vs_oracle_total_rel": abs(t64[9] - ref["terms"][9]) / abs(ref["terms"][9]),
                         "fp64_vs_oracle_grad_rms": float(np.sqrt(np.mean((g64 - ref["grad"]) ** 2))),
                         "mixed_vs_oracle_total_rel": abs(tm[9] - ref["terms"][9]) / abs(ref["terms"][9]),
                         "mixed_vs_oracle_grad_rms": float(np.sqrt(np.mean((gm - ref["grad"]) ** 2)))})
    f64.close()
    mix.close()
    et = np.array(err_terms)
    names = ["vdw", "permanent", "polarization", "perm_real", "perm_self", "perm_recip", "pol_real", "pol_self",
             "pol_recip", "total"]
    print(json.dumps({
        "metric": "mixed-precision error vs FP64, 24k-atom water box, frames of a 300 K trajectory",
        "frames": len(frames), "trajectory": "2 fs velocity Verlet + SETTLE on the device, FP64 forces, rescaled "
                                             "to 300 K every 10 steps, frame every 10 steps after equilibration",
        "term_abs_error_max": dict(zip(names, et.max(0).tolist())),
        "term_abs_error_mean": dict(zip(names, et.mean(0).tolist())),
        "total_rel_error_max": float(max(rel_total)), "total_rel_error_mean": float(np.mean(rel_total)),
        "grad_rms_error_max": float(max(grad_rms)), "grad_rms_error_mean": float(np.mean(grad_rms)),
        "oracle_pins": pins}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--cpu-samples", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-systems", type=int, default=512,
                    help="also time a batch of this many small systems (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=5)
    ap.add_argument("--md-steps", type=int, default=1000,
                    help="also time this many 2 fs MD steps on the device (0: skip)")
    ap.add_argument("--lambda-values", type=float, nargs="*", default=None,
                    help="instead of the headline, time electrostatic lambda evaluations at these lambdas")
    ap.add_argument("--accuracy-frames", type=int, default=0,
                    help="instead of timing, report the mixed form's error on this many trajectory frames")
    ap.add_argument("--accuracy-equil", type=int, default=200, help="equilibration steps before the first frame")
    args = ap.parse_args()
    if args.accuracy_frames > 0:
        run_accuracy(args)
        return
    if args.lambda_values:
        run_lambda(args)
        return
    if args.warmup < 3 and args.impl == "mine":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_mine(args)


if __name__ == "__main__":
    main()
