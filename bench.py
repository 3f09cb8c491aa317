#!/usr/bin/env python
"""Benchmark: NUC3d RHS + TVD-RK3 time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one box per GPU): decaying isotropic turbulence on a periodic 256^3
box, seeded solenoidal velocity with E(k) ~ k^4 exp(-2 (k/4)^2), M = 1,
turbulent Mach 0.3, Reynolds number set for Re_lambda = 100; Navier-Stokes,
Lax-Friedrichs split, WENO5-Z reconstruction, CD6 viscous terms, TVD-RK3 at
CFL 0.5.  One "step" is one TVD-RK3 step (3 RHS evaluations) of every box.
The metric is cell-updates/s (cells x steps / s) over the whole job.

* ``value``: FP64 path, state resident in HBM, device-timed with CUDA events
  (max over ranks), the median of --repeats timed regions of exactly --steps
  steps each.  The state (671 MB per box) is larger than the 126 MB L2, so
  no flush is needed between steps.  ``clocks``: NVML samples every 10 ms
  over the timed regions.
* ``e2e``: the same metric through the C ABI with host buffers: each step
  uploads a state from pinned host memory, advances it one step and
  downloads the result to pinned host memory.  Three contexts on three
  streams take the steps in turn (nuc3d_set/get_state_host_async), so the
  copies overlap the steps; ``e2e.serial`` is the synchronous time loop
  through host memory (nuc3d_set_state_host, nuc3d_step with dt/residual,
  nuc3d_get_state_host).
* ``mixed``: the FP32-bulk / FP64-state form on the same workload, with its
  per-field relative L2 distance to the FP64 path after 100 steps.
* ``roofline``: the dominant kernel (inviscid WENO sweep), algorithmic FP64
  flops per launch over its event-timed average launch duration, against the
  FP64 FMA rate measured in the same run (nuc3d_probe_peak).
* ``long_horizon``: FP64 and mixed advanced 2000 steps from the same state,
  TKE, dissipation and spectrum compared over the run.
* ``config3``: forced HIT at 384^3, turbulent Mach 0.6, band forcing at a
  fixed injection rate, hccs and CRWENO5, FP64 and mixed (CFL 0.4).
* ``ensemble`` / ``served``: the batched 64-box ensemble and the served
  request stream (continuous batching vs a serial FP64 queue, with the same
  mix run as one batch as its ceiling).
* ``cpu_baseline``: the reference's own code (oracle/_ref) on host cores.

With --gpus N > 1 (torchrun), every rank advances its own box (independent
replicas, no data-path collective); timing is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "nuc3d-cartisian_b200" / "python"))

METRIC = "cell-updates/s at 256^3 (decaying HIT, WENO5-Z, N-S, TVD-RK3)"
UNIT = "cell-updates/s"
NX = 256
SEED = 0
K_PEAK = 4.0
MACH_T = 0.3
RE_LAMBDA = 100.0
CFL = 0.5
# Algorithmic FP64 flops (add/mul/div/sqrt = 1, FMA = 2) per cell, counted
# from the kernels' formulas: one directional sweep = 5 equations x
# (2 WENO5-Z faces of 76 flops + F^+ + F^- add + difference 2) + LF split 33.
FLOPS_INV_Z = 5 * (2 * 76 + 1 + 2) + 33
FLOPS_INV_JS = 5 * (2 * 68 + 1 + 2) + 33
FLOPS_PRIM = 20  # con2prim + eigenvalues, done by the x sweep while staging
FLOPS_PER_CELL_STAGE = 3 * FLOPS_INV_Z + FLOPS_PRIM + 156 + 111  # + viscous flux, update
# algorithmic flops of the average sweep launch (x, y, z; x carries con2prim)
FLOPS_INV_LAUNCH = FLOPS_INV_Z + FLOPS_PRIM / 3
STATE_BYTES_PER_CELL_UPDATE = 320  # compulsory FP64 state traffic of 3 RK stages
# DRAM bytes (read + write) per launch of the FP64 WENO5-Z sweep at 256^3,
# mean of x, y, z: the ncu capture at 128^3 in
# profiles/k_inviscid_weno5z_fp64_128.md (212.0, 269.4, 281.8 MB; the x sweep
# reads the state only and writes the primitives as well as its RHS) scaled
# by the cell count (x8); the traffic of a sweep is proportional to the cells
# it covers (whole lines, no halo growth with size along the other axes).
INV_TRAFFIC_BYTES = 8 * (212.03072e6 + 269.391872e6 + 281.837568e6) / 3
INV_TRAFFIC_NOTE = "ncu dram__bytes_read+write of the 128^3 capture x8 (cells), mean of x/y/z"


def hbm_peak_gbs():
    """Measured copy bandwidth of this pool's B200s (MEASURED_PEAKS.json)."""
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def config_dict(n_gpus, reynolds):
    return {
        "workload": f"decaying isotropic turbulence {NX}^3 periodic box, seeded solenoidal "
                    f"E(k)~k^4 exp(-2(k/{K_PEAK:g})^2), M=1, Mt={MACH_T}, Re_lambda={RE_LAMBDA:g}; "
                    "Navier-Stokes, LF split, WENO5-Z, CD6 viscous, TVD-RK3 CFL 0.5",
        "cells_per_box": NX ** 3,
        "boxes_per_gpu": 1,
        "reynolds": reynolds,
        "parallelism": f"replicas x{n_gpus} (one box per GPU, no collective)",
        "l2_flush": (f"not needed: {40 * NX ** 3 / 1e6:.0f} MB FP64 state per box > 126 MB L2"
                     if 40 * NX ** 3 > 126e6 else "state smaller than L2 (profiling size only)"),
        "timing": "median of the repeats, each exactly `steps` steps between barriers",
    }


# ------------------------------------------------------------- CPU side ----
def _cpu_worker(args):
    """One reference (or oracle) box of the bounded sample, timed."""
    kind, n, steps, warm, reynolds = args
    # the reference prints its MPI topology on stdout; keep the bench's
    # stdout to the one JSON line
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "nuc3d-cartisian_b200" / "python"))
    import numpy as np
    import oracle_ctypes as oc
    from nuc3d_b200.initial import hit_field
    import nuc3d_b200 as nb
    desc = nb.BoxDesc(n, n, n, mach=1.0)
    q = hit_field(desc, seed=SEED, k_peak=K_PEAK, mach_t=MACH_T)
    box = oc.Box(n, n, n, scheme=(oc.WENO5Z,) * 3, mach=1.0, reynolds=reynolds)
    eng = oc.Reference() if kind == "reference" else oc.Oracle()
    if warm:
        q, _, _ = eng.run_steps(box, CFL, warm, q)
    t0 = time.perf_counter()
    eng.run_steps(box, CFL, steps, q)
    return time.perf_counter() - t0


def cpu_sample(n, steps, warm, reynolds, workers):
    """Run `workers` independent boxes concurrently (spawned processes, one
    per core: the reference is one MPI rank per core and this machine has no
    MPI).  Returns (cell-updates/s, wall seconds, kind)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_ctypes as oc
    kind = "reference" if oc.Reference.available() else "port"
    if kind == "port":
        oc.build_oracle()
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(workers) as pool:
        times = pool.map(_cpu_worker, [(kind, n, steps, warm, reynolds)] * workers)
    wall = time.perf_counter() - t0
    slowest = max(times)
    return workers * n ** 3 * steps / slowest, slowest, kind


# ------------------------------------------------------------ clocks -------
_REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
            ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))


class ClockSampler:
    """SM clock, power and throttle reasons of one GPU sampled while a timed
    region runs (read only: NVML queries, every 10 ms, on a thread; nvidia-smi
    at 200 ms where NVML is unavailable).  The GPU is matched by PCI bus id,
    so CUDA_VISIBLE_DEVICES does not shift it."""

    def __init__(self, dev_index):
        import threading
        self.samples = []  # (sm_mhz, power_w, reasons bitmask)
        self.smax = None
        self.proc = None
        self.path = None
        self._stop = threading.Event()
        self._thread = None
        self.source = "nvml"
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(dev_index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            try:
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except pynvml.NVMLError:
                h = pynvml.nvmlDeviceGetHandleByIndex(dev_index)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

            def run():
                while not self._stop.is_set():
                    try:
                        self.samples.append((
                            float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)),
                            pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0,
                            int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))))
                    except pynvml.NVMLError:
                        pass
                    self._stop.wait(0.01)
            self._thread = threading.Thread(target=run, daemon=True)
            self._thread.start()
        except Exception:
            self._start_smi(dev_index)

    def _start_smi(self, gpu_index):
        self.source = "nvidia-smi"
        fields = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                  "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                  "clocks_event_reasons.sw_power_cap")
        self.path = Path(tempfile.mkstemp(prefix="clocks_", suffix=".csv")[1])
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={fields}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            for line in self.path.read_text().splitlines():
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 7:
                    continue
                try:
                    sm, self.smax, pw = float(parts[0]), float(parts[1]), float(parts[2])
                except ValueError:
                    continue
                mask = sum(bit for (nm, bit), v in zip(_REASONS[:4], parts[3:7])
                           if v.lower() == "active")
                self.samples.append((sm, pw, mask))
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm = [a for a, _, _ in self.samples]
        pw = [b for _, b, _ in self.samples]
        reasons = sorted({nm for _, _, m in self.samples for nm, bit in _REASONS if m & bit})
        counts = {nm: sum(1 for _, _, m in self.samples if m & bit) for nm, bit in _REASONS}
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                "sm_mhz_min": min(sm) if sm else None,
                "power_w_median": statistics.median(pw) if pw else None,
                "samples": len(sm), "source": self.source, "reasons": reasons,
                "reason_samples": {k: v for k, v in counts.items() if v}}


# ------------------------------------------------------------ GPU arm ------
def run_b200(args, rank, world, local_rank):
    import numpy as np
    import torch
    import nuc3d_b200 as nb
    from nuc3d_b200.replicas import RankInfo, Replicas, whole_job_rate

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    reps = Replicas(RankInfo(rank, world, local_rank), backend="nccl", timeout_s=120.0, device=dev)

    desc = nb.BoxDesc(NX, NX, NX, mach=1.0, scheme=(nb.WENO5Z,) * 3)
    q, reynolds = nb.hit_field(desc, seed=SEED + rank, k_peak=K_PEAK, mach_t=MACH_T,
                               re_lambda=RE_LAMBDA)
    desc = nb.BoxDesc(NX, NX, NX, mach=1.0, scheme=(nb.WENO5Z,) * 3, reynolds=reynolds)
    cells = desc.cells
    pinned = [torch.from_numpy(a).pin_memory() for a in q]
    host_q = [p.numpy() for p in pinned]

    stream = torch.cuda.current_stream(dev)

    def barrier():
        reps.barrier(lambda: torch.cuda.synchronize(dev))

    max_over_ranks = reps.max

    def timed_steps(solver, k):
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.step(k, CFL, stats=False)
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1)

    def timed_repeats(solver, k, repeats):
        """`repeats` timed regions of exactly k steps each (barrier + device
        sync on both sides, CUDA events on the launching stream); the max
        over ranks of each."""
        return [max_over_ranks(timed_steps(solver, k)) for _ in range(repeats)]

    peak64 = nb.probe_peak(nb.FP64)
    peak32 = nb.probe_peak(nb.MIXED)

    # ---- FP64, resident state: the headline value
    s64 = nb.Solver(desc, stream=stream)
    s64.set_state(host_q)
    s64.step(args.warmup, CFL, stats=False)
    s64.sync()
    clocks = ClockSampler(local_rank)
    launches0 = s64.launch_count()
    reps_ms = timed_repeats(s64, args.steps, args.repeats)
    launches = (s64.launch_count() - launches0) // args.repeats
    clock_info = clocks.stop()
    s64.sync()
    ms_max = statistics.median(reps_ms)
    ms_per_step = ms_max / args.steps
    value = whole_job_rate(cells, world, ms_per_step * 1e-3)
    timing = {"repeats": args.repeats, "steps_per_repeat": args.steps,
              "ms_per_step_each": [m / args.steps for m in reps_ms],
              "value_from": "median repeat", "timed_s_total": sum(reps_ms) / 1e3}

    tuning64 = s64.tuning()
    # ---- per-kernel event timing (separate short pass, same workload)
    s64.profile(True)
    s64.step(2, CFL, stats=False)
    prof = s64.profile_read(reset=True)
    s64.profile(False)
    inv_ms = sum(prof[k][0] for k in ("inv_x", "inv_y", "inv_z"))
    inv_n = sum(prof[k][1] for k in ("inv_x", "inv_y", "inv_z"))
    total_ms = sum(v[0] for v in prof.values())
    inv_avg_ms = inv_ms / max(inv_n, 1)
    achieved = FLOPS_INV_LAUNCH * cells / (inv_avg_ms * 1e-3) / 1e12
    roofline = {
        "bound": "fp64",
        "kernel": "k_inviscid<WENO5-Z, FP64> (directional sweep, x/y/z; x also recovers the primitives)",
        "achieved": achieved,
        "peak": peak64,
        "unit": "TFLOP/s",
        "frac": achieved / peak64,
        "peak_source": "FP64 FMA rate measured in this run (nuc3d_probe_peak)",
        "traffic": INV_TRAFFIC_BYTES,
        "traffic_source": INV_TRAFFIC_NOTE,
        "traffic_gbs": INV_TRAFFIC_BYTES / (inv_avg_ms * 1e-3) / 1e9,
        "flops_per_launch": FLOPS_INV_LAUNCH * cells,
        "avg_launch_ms": inv_avg_ms,
        "share_of_step": inv_ms / total_ms if total_ms else None,
        "kernel_ms_per_step": {k: v[0] / 2 for k, v in prof.items()},
        "autotuned_sweep_variant": tuning64,
        "step_fp64_tflops": FLOPS_PER_CELL_STAGE * 3 * cells / (ms_per_step * 1e-3) / 1e12,
        "hbm_state_frac": STATE_BYTES_PER_CELL_UPDATE * cells / (ms_per_step * 1e-3) / 1e9
                          / hbm_peak_gbs()[0],
        "hbm_peak_gbs": hbm_peak_gbs()[0],
        "hbm_peak_source": hbm_peak_gbs()[1],
    }

    # ---- e2e through the C ABI with host buffers
    # (a) serial: a time loop through host memory -- each step uploads the
    # state from pinned memory, advances it one step with dt/residual read
    # back, and downloads the result, which is the next step's input
    e2e_serial_steps = max(1, min(args.steps, 5))
    ser_q = [torch.from_numpy(p.copy()).pin_memory().numpy() for p in host_q]  # pinned
    s64.set_state(ser_q)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_serial_steps):
        s64.set_state(ser_q)               # H2D of the step's input state (pinned)
        s64.step(1, CFL, stats=True)       # dt and residual read back
        s64.get_state(ser_q)               # D2H of the step's result state
    barrier()
    e2e_serial_s = max_over_ranks(time.perf_counter() - t0)
    # (b) pipelined: every step advances a host-resident input state (the
    # benchmark field, pinned) one step and returns the result to pinned host
    # memory through nb.StepPipeline: three solver contexts on three streams
    # take the steps in turn, their host transfers in the device's copy lanes
    # (one upload and one download at a time, each with the whole host link),
    # so one context's upload, another's step and a third's download overlap
    n_pipe = 3
    pipe = nb.StepPipeline(desc, depth=n_pipe, cfl=CFL, device=dev)
    pipe.warm_up(host_q, args.warmup)  # graph capture, autotuning
    outs = [[torch.empty(desc.shape, dtype=torch.float64).pin_memory().numpy()
             for _ in range(5)] for _ in range(n_pipe)]
    # (30 steps by default: the pipeline's fill and drain, about one step's
    # upload + compute + download, spread over enough steps)
    e2e_steps = n_pipe * max(2, min(max(args.steps, 30), 60) // n_pipe)
    barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        pipe.submit(host_q, outs[i % n_pipe])   # H2D, one step, D2H
    pipe.drain()
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = world * cells * e2e_steps / e2e_s
    # every pipelined result is one step of the input: the same bits as a
    # single step taken on its own
    s64.set_state(host_q)
    s64.step(1, CFL, stats=False)
    one = s64.get_state()
    e2e_checked = all(np.array_equal(a, b) for out_i in outs for a, b in zip(out_i, one))
    pipe.close()
    del pipe
    # resident variant: state stays on the device, dt/residual read each step
    s64.set_state(host_q)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_serial_steps):
        s64.step(1, CFL, stats=True)
    barrier()
    res_s = max_over_ranks(time.perf_counter() - t0)
    s64.close()

    # ---- mixed precision form
    mixed = None
    if not args.skip_mixed:
        dm = nb.BoxDesc(**{**desc.__dict__, "precision": nb.MIXED})
        sm = nb.Solver(dm, stream=stream)
        sm.set_state(q)
        sm.step(args.warmup, CFL, stats=False)
        sm.sync()
        ms_m = statistics.median(timed_repeats(sm, args.steps, args.repeats))
        tuning32 = sm.tuning()
        sm.profile(True)
        sm.step(2, CFL, stats=False)
        prof_m = sm.profile_read(reset=True)
        sm.profile(False)
        sm.close()
        # accuracy: 100 steps from the same state, both precisions, with the
        # device statistics (FP64 reductions) logged every 25 steps
        nacc = args.accuracy_steps
        logs = {}
        finals = {}
        spectra = {}
        for name, d in (("fp64", desc), ("mixed", dm)):
            with nb.Solver(d, stream=stream) as a:
                a.set_state(q)
                log = [a.stats()]
                done = 0
                while done < nacc:
                    k = min(25, nacc - done)
                    a.step(k, CFL, stats=False)
                    done += k
                    log.append(a.stats())
                logs[name] = log
                finals[name] = a.get_state()
                spectra[name] = a.spectra()
        r64, r32 = finals["fp64"], finals["mixed"]
        errs = [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(r32, r64)]
        ke = [logs["mixed"][-1]["kinetic"], logs["fp64"][-1]["kinetic"]]

        def max_rel(key):
            return max(abs(m[key] - f[key]) / abs(f[key])
                       for m, f in zip(logs["mixed"], logs["fp64"]))
        mixed = {
            "value": world * cells / (ms_m / args.steps * 1e-3),
            "ms_per_step": ms_m / args.steps,
            "speedup_vs_fp64": ms_per_step / (ms_m / args.steps),
            "dtype": "fp32 bulk / fp64 state",
            "rel_l2_vs_fp64": max(errs),
            "rel_l2_per_field": errs,
            "tke_rel_diff": abs(ke[0] - ke[1]) / ke[1],
            "tke_max_rel_diff_over_run": max_rel("kinetic"),
            "dissipation_max_rel_diff_over_run": max_rel("dissipation"),
            "stats_every_steps": 25,
            # kinetic-energy spectrum (postproc::solveFFT "kin") after the run,
            # shells holding at least 1e-10 of the energy
            "spectrum_kin_max_rel_diff": spectrum_diff(spectra["mixed"][0], spectra["fp64"][0]),
            "spectrum_kin_fp64": [float(v) for v in spectra["fp64"][0]],
            "fp64_stats": {k: [round(v[k], 10) for v in logs["fp64"]]
                           for k in ("kinetic", "dissipation", "enstrophy", "re_lambda", "mach_t")},
            "accuracy_steps": nacc,
            "peak_fp32_tflops": peak32,
            "kernel_ms_per_step": {k: v[0] / 2 for k, v in prof_m.items()},
            "autotuned_sweep_variant": tuning32,
        }

    # The per-GPU characterisations (scheme timings, the 2000-step statistics
    # leg, the 384^3 configuration, the served stream) are the same on every
    # rank: a run on N > 1 GPUs measures the replicas' headline, mixed and
    # ensemble rates only, so that it holds the N GPUs for about as long as
    # the timed work needs.
    per_gpu_only = ["schemes", "long_horizon", "config3", "served"] if world > 1 else []
    if world > 1:
        args.skip_schemes = args.skip_long = args.skip_config3 = True
    schemes = None if args.skip_schemes else run_schemes(args, desc, q, stream, timed_steps,
                                                         max_over_ranks)
    long_horizon = None if (args.skip_long or args.skip_mixed) else run_long_horizon(
        args, desc, q, stream)
    config3 = None if args.skip_config3 else run_config3(args, stream)
    ensemble = None if args.skip_ensemble else run_ensemble(args, stream, barrier, max_over_ranks,
                                                            world, rank)
    served = None if (args.skip_serve or world > 1) else run_served(args)

    if rank != 0:
        reps.close()
        return None
    cpu = None
    if args.cpu_result is not None:
        cpu = args.cpu_result
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded HIT field; no dataset)",
        "config": config_dict(world, reynolds),
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": 5 * 8 * cells, "d2h_bytes_per_step": 5 * 8 * cells,
                "steps": e2e_steps,
                "how": f"C ABI through nb.StepPipeline, host buffers: each step uploads a pinned "
                       f"host state, advances it one TVD-RK3 step and downloads the result; "
                       f"{n_pipe} contexts on {n_pipe} streams take the steps in turn, their "
                       f"transfers in the device's copy lanes (one per direction at a time), "
                       f"so uploads, steps and downloads overlap",
                "results_equal_single_step": e2e_checked,
                "serial": {"value": world * cells * e2e_serial_steps / e2e_serial_s, "unit": UNIT,
                           "how": "one context, synchronous copies, the result of each step "
                                  "uploaded as the next step's input (a time loop through "
                                  "host memory), dt/residual read back",
                           "h2d_bytes_per_step": 5 * 8 * cells,
                           "d2h_bytes_per_step": 5 * 8 * cells + 16,
                           "steps": e2e_serial_steps},
                "resident": {"value": world * cells * e2e_serial_steps / res_s, "unit": UNIT,
                             "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 16}},
        "gpu_launches": launches,
        "timing": timing,
        "roofline": roofline,
        "clocks": clock_info,
        "mixed": mixed,
        "schemes": schemes,
        "long_horizon": long_horizon,
        "config3": config3,
        "ensemble": ensemble,
        "served": served,
        "cpu_baseline": cpu,
    }
    if per_gpu_only:
        line["legs_run_at_one_gpu_only"] = per_gpu_only
    reps.close()
    return line


def spectrum_diff(a, b):
    """Max relative difference over the shells of spectrum b that hold at
    least 1e-10 of its total."""
    import numpy as np
    on = b > 1e-10 * b.sum()
    return float(np.max(np.abs(a[on] - b[on]) / b[on]))


# -------------------------------------------------------- long horizon -----
LONG_KEYS = ("kinetic", "dissipation", "enstrophy", "re_lambda", "mach_t", "u_rms")


def run_long_horizon(args, desc, q, stream):
    """The 256^3 decaying HIT advanced --long-steps steps in FP64 and in mixed
    precision from the same state, with the device statistics (FP64
    reductions, postproc::solveQ) every --long-every steps and the
    kinetic-energy spectrum (postproc::solveFFT) at the middle and the end:
    how far the mixed form's TKE, dissipation and spectrum move from the
    FP64 path's over the run."""
    import numpy as np
    import torch
    import nuc3d_b200 as nb
    nsteps, every = args.long_steps, args.long_every
    logs, spectra, dev_ms, times = {}, {}, {}, {}
    for name, prec in (("fp64", nb.FP64), ("mixed", nb.MIXED)):
        d = nb.BoxDesc(**{**desc.__dict__, "precision": prec})
        with nb.Solver(d, stream=stream) as a:
            a.set_state(q)
            log, spec, ms = [a.stats()], {}, 0.0
            done = 0
            while done < nsteps:
                k = min(every, nsteps - done)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                a.step(k, CFL, stats=False)
                e1.record(stream)
                a.sync()
                ms += e0.elapsed_time(e1)
                done += k
                log.append(a.stats())
                if done == nsteps // 2 or done == nsteps:
                    spec[done] = a.spectra()[0]
            logs[name], spectra[name], dev_ms[name], times[name] = log, spec, ms, a.time()
    rel = {key: [abs(m[key] - f[key]) / abs(f[key]) for m, f in zip(logs["mixed"], logs["fp64"])]
           for key in LONG_KEYS}

    def first_over(key, bar=0.005):
        for i, v in enumerate(rel[key]):
            if v > bar:
                return i * every
        return None
    ke0 = logs["fp64"][0]
    tau = ke0["eddy_turnover"]
    return {
        "workload": f"{desc.nx}^3 decaying HIT (the headline field), WENO5-Z, CFL {CFL}, "
                    f"{nsteps} steps FP64 and mixed from the same state",
        "steps": nsteps, "stats_every_steps": every,
        "sim_time": times["fp64"],
        "eddy_turnover_time_initial": tau,
        "eddy_turnovers": times["fp64"] / tau if tau else None,
        "ms_per_step": {k: v / nsteps for k, v in dev_ms.items()},
        "cell_updates_per_s": {k: desc.cells * nsteps / (v * 1e-3) for k, v in dev_ms.items()},
        "tke_max_rel_diff": max(rel["kinetic"]),
        "dissipation_max_rel_diff": max(rel["dissipation"]),
        "max_rel_diff": {k: max(v) for k, v in rel.items()},
        "first_step_over_0.5pct": {k: first_over(k) for k in ("kinetic", "dissipation")},
        "spectrum_kin_max_rel_diff": {str(k): spectrum_diff(spectra["mixed"][k], spectra["fp64"][k])
                                      for k in spectra["fp64"]},
        "tke_decay": logs["fp64"][-1]["kinetic"] / ke0["kinetic"],
        "fp64_series": {k: [round(v[k], 10) for v in logs["fp64"]] for k in LONG_KEYS},
        "mixed_series": {k: [round(v[k], 10) for v in logs["mixed"]] for k in ("kinetic", "dissipation")},
        "spectrum_kin_fp64_end": [float(v) for v in spectra["fp64"][nsteps]],
    }


# ------------------------------------------------------------- config 3 ----
def run_config3(args, stream):
    """Forced isotropic turbulence with shocklets: --c3-n^3 (384) periodic
    box, seeded solenoidal field of the headline's spectrum at turbulent Mach
    0.6 (M 1, Re from Re_lambda 100), the band forcing on 0 < |k| <= 2 at a
    fixed injection rate equal to the initial dissipation rate, CFL 0.4.
    hccs (the reference's hybrid compact-WENO switch, CRWENO5 rows with linear
    compact rows where smooth) and plain CRWENO5, FP64 and mixed: device-timed
    steps, the mixed form's per-field relative L2 from FP64 after --c3-steps
    steps, and the mixed hccs run continued to --c3-long steps, checked finite
    every 100."""
    import numpy as np
    import torch
    import nuc3d_b200 as nb
    n = args.c3_n
    cfl = 0.4
    init = {"kind": "hit", "seed": 0, "k_peak": K_PEAK, "mach_t": 0.6, "re_lambda": RE_LAMBDA}
    with nb.Solver(nb.BoxDesc(n, n, n, mach=1.0), stream=stream) as s0:
        info = s0.init_state(init)
        st0 = s0.stats()
    rate = st0["dissipation"]
    out = {"workload": f"forced HIT {n}^3, Mt 0.6, M 1, Re_lambda {RE_LAMBDA:g} (Re "
                       f"{info['reynolds']:.6g}), band forcing 0<|k|<=2 at injection rate "
                       f"{rate:.6g} (the initial dissipation rate), CFL {cfl}",
           "cells": n ** 3, "reynolds": info["reynolds"], "injection_rate": rate,
           "initial": {k: st0[k] for k in ("kinetic", "dissipation", "mach_t", "re_lambda")}}
    for sname, sch, long_mixed in (("hccs", nb.HCCS, True), ("crweno5", nb.CRWENO5, False)):
        row, finals = {}, {}
        for pname, prec in (("fp64", nb.FP64), ("mixed", nb.MIXED)):
            d = nb.BoxDesc(n, n, n, mach=1.0, scheme=(sch,) * 3, precision=prec,
                           forcing=nb.FORCING_BAND, forcing_amp=rate, forcing_k=2.0)
            with nb.Solver(d, stream=stream) as s:
                s.init_state(init)
                s.step(args.warmup, cfl, stats=False)
                s.sync()
                k = max(3, min(args.steps, 10))
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                s.step(k, cfl, stats=False)
                e1.record(stream)
                s.sync()
                ms = e0.elapsed_time(e1) / k
                s.step(max(0, args.c3_steps - args.warmup - k), cfl, stats=False)
                s.sync()
                finals[pname] = s.get_state()
                st = s.stats()
                r = {"ms_per_step": ms, "cell_updates_per_s": n ** 3 / (ms * 1e-3),
                     "kinetic": st["kinetic"], "dissipation": st["dissipation"],
                     "mach_t": st["mach_t"],
                     "finite": bool(all(np.isfinite(a).all() for a in finals[pname]))}
                if prec == nb.MIXED and long_mixed:
                    done, ok, kes = args.c3_steps, True, []
                    while done < args.c3_long:
                        try:
                            s.step(min(100, args.c3_long - done), cfl, stats=False)
                            s.sync()
                        except nb.Nuc3dError as e:
                            ok = False
                            r["error"] = f"after {done} steps: {e}"
                            break
                        done = min(done + 100, args.c3_long)
                        kes.append(s.stats()["kinetic"])
                    r["long_steps"] = done
                    r["long_finite"] = ok
                    r["long_kinetic_every_100"] = kes
            row[pname] = r
        errs = [float(np.linalg.norm(a - b) / np.linalg.norm(b))
                for a, b in zip(finals["mixed"], finals["fp64"])]
        del finals
        row["rel_l2_vs_fp64_per_field"] = errs
        row["rel_l2_vs_fp64"] = max(errs)
        row["compared_after_steps"] = args.c3_steps
        row["mixed_speedup"] = row["fp64"]["ms_per_step"] / row["mixed"]["ms_per_step"]
        out[sname] = row
    return out


# ------------------------------------------------------------- schemes -----
def run_schemes(args, desc, q, stream, timed_steps, max_over_ranks):
    """Every reconstruction on the same 256^3 field, FP64 and mixed: ms per
    step and the directional sweeps' share (WENO5-Z FP64 is the headline
    above; this places the other Method.in schemes beside it)."""
    import nuc3d_b200 as nb
    k = max(3, min(args.steps, 10))
    out = {"steps": k, "workload": f"{desc.nx}^3 HIT, CFL {CFL}"}
    for name, sch in (("weno5js", nb.WENO5JS), ("weno5z", nb.WENO5Z), ("crweno5", nb.CRWENO5),
                      ("weno7js", nb.WENO7JS)):
        row = {}
        for pname, prec in (("fp64", nb.FP64), ("mixed", nb.MIXED)):
            d = nb.BoxDesc(**{**desc.__dict__, "scheme": (sch,) * 3, "precision": prec})
            with nb.Solver(d, stream=stream) as s:
                s.set_state(q)
                s.step(args.warmup, CFL, stats=False)
                s.sync()
                ms = max_over_ranks(timed_steps(s, k)) / k
                s.profile(True)
                s.step(1, CFL, stats=False)
                prof = s.profile_read(reset=True)
                s.profile(False)
            sweep = sum(prof[x][0] for x in ("inv_x", "inv_y", "inv_z"))
            row[pname] = {"ms_per_step": ms, "cell_updates_per_s": desc.cells / (ms * 1e-3),
                          "sweep_ms_per_step": sweep,
                          "sweep_share": sweep / max(sum(v[0] for v in prof.values()), 1e-12)}
        row["mixed_speedup"] = row["fp64"]["ms_per_step"] / row["mixed"]["ms_per_step"]
        out[name] = row
    return out


# ------------------------------------------------------------ ensemble -----
def ensemble_boxes(nboxes, seed0):
    """The batched-ensemble workload: box edges drawn from {32,48,64,96,128},
    turbulent Mach U[0.1,0.5], Re_lambda U[40,120], WENO5-JS or WENO5-Z per
    box, seeded HIT initial states generated on the device (box b uses seed
    seed0 + b).  Returns (desc, init) pairs."""
    import numpy as np
    import nuc3d_b200 as nb
    rng = np.random.default_rng(2024 + seed0)
    out = []
    for b in range(nboxes):
        n = int(rng.choice([32, 48, 64, 96, 128]))
        mt = float(rng.uniform(0.1, 0.5))
        rl = float(rng.uniform(40.0, 120.0))
        scheme = nb.WENO5JS if rng.uniform() < 0.5 else nb.WENO5Z
        d = nb.BoxDesc(n, n, n, mach=1.0, scheme=(scheme,) * 3)
        out.append((d, {"kind": "hit", "seed": seed0 + b, "k_peak": K_PEAK, "mach_t": mt,
                        "re_lambda": rl}))
    return out


def run_ensemble(args, stream, barrier, max_over_ranks, world, rank):
    import torch
    import nuc3d_b200 as nb
    boxes = ensemble_boxes(args.ensemble_boxes, 64 * rank)
    cells = sum(d.cells for d, _ in boxes)
    res = {"boxes_per_gpu": len(boxes), "cells_per_gpu": cells,
           "edges": sorted({d.nx for d, _ in boxes}),
           "workload": "batched ensemble: 64 periodic HIT boxes, edges {32,48,64,96,128}, "
                       "Mt U[0.1,0.5], Re_lambda U[40,120], WENO5-JS/Z per box, one launch per "
                       "kernel class for all boxes, step replayed as a CUDA graph"}
    for name, prec in (("mixed", nb.MIXED), ("fp64", nb.FP64)):
        with nb.Batch(prec, stream=stream) as B:
            ids = [B.add(d) for d, _ in boxes]
            for i, (_, init) in zip(ids, boxes):
                B.init_state(i, init)
            B.step(args.warmup)
            B.sync()
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            l0 = B.launch_count()
            e0.record(stream)
            B.step(args.steps)
            e1.record(stream)
            barrier()
            ms = max_over_ranks(e0.elapsed_time(e1))
            B.sync()
            res[name] = {"value": world * cells * args.steps / (ms * 1e-3), "unit": UNIT,
                         "ms_per_step": ms / args.steps,
                         "launches_per_step": (B.launch_count() - l0) / args.steps}
    res["mixed_speedup_vs_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
    return res


# ------------------------------------------------------------- serving -----
def served_requests(nreq, seed, rate):
    """The served stream: Poisson arrivals (mean `rate` per second), box edge
    log-uniform in [32, 192], steps log-uniform in [50, 1000], turbulent Mach
    U[0.1, 0.6], Re_lambda U[40, 120], scheme WENO5-JS / WENO5-Z / CRWENO5,
    seeded HIT initial state generated on the device."""
    import numpy as np
    import nuc3d_b200 as nb
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, nreq))
    t -= t[0]
    out = []
    for i in range(nreq):
        n = int(round(math.exp(rng.uniform(math.log(32), math.log(192)))))
        steps = int(round(math.exp(rng.uniform(math.log(50), math.log(1000)))))
        mt = float(rng.uniform(0.1, 0.6))
        rl = float(rng.uniform(40.0, 120.0))
        scheme = (nb.WENO5JS, nb.WENO5Z, nb.CRWENO5)[int(rng.integers(3))]
        d = nb.BoxDesc(n, n, n, mach=1.0, scheme=(scheme,) * 3)
        out.append((float(t[i]), d, steps,
                    {"kind": "hit", "seed": seed * 1000 + i, "k_peak": K_PEAK, "mach_t": mt,
                     "re_lambda": rl}))
    return out


def run_stream(reqs, precision, max_resident, budget_bytes, burst=False):
    """Submits the requests at their arrival times (burst: all at once) to a
    fresh server and collects every result (final state copied to the host)
    on a second thread.  Latency = completion - submission on the server's
    clock."""
    import threading
    import nuc3d_b200 as nb
    srv = nb.Server(precision=precision, budget_bytes=budget_bytes, max_resident=max_resident)
    results = []
    submitted = threading.Semaphore(0)

    def collect():
        for _ in reqs:
            submitted.acquire()  # a solve is outstanding
            r = srv.wait()
            r.pop("state", None)
            results.append(r)

    th = threading.Thread(target=collect)
    th.start()
    t0 = time.perf_counter()
    for ta, d, steps, init in reqs:
        delay = 0.0 if burst else t0 + ta - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        srv.submit(d, steps, CFL, init=init, want_state=True)
        submitted.release()
    th.join()
    st = srv.stats()
    srv.close()
    ok = [r for r in results if r["status"] == nb.OK]
    lat = sorted(r["t_done"] - r["t_submit"] for r in ok)
    span = max(r["t_done"] for r in results) - min(r["t_submit"] for r in results)
    pct = lambda q: lat[min(len(lat) - 1, int(math.ceil(q * len(lat))) - 1)] if lat else None  # noqa: E731
    return {
        "solves_per_s": len(ok) / span,
        "p50_latency_s": pct(0.50),
        "p99_latency_s": pct(0.99),
        "mean_queue_s": sum(r["t_admit"] - r["t_submit"] for r in ok) / max(len(ok), 1),
        "cell_updates_per_s": st["cell_updates"] / span,
        "span_s": span,
        "completed": len(ok),
        "failed": len(results) - len(ok),
        "peak_resident": st["peak_resident"],
        "peak_resident_gb": st["peak_resident_bytes"] / 1e9,
        "chunks": st["chunks"],
        "batch_steps": st["batch_steps"],
        "steps_per_chunk": st["batch_steps"] / max(st["chunks"], 1),
        "graph_captures": st["graph_captures"],
        "busy_s": st["busy_s"],
        "busy_frac": st["busy_s"] / span,
        "kernel_launches": st["launches"],
    }


def run_served(args):
    import nuc3d_b200 as nb
    reqs = served_requests(args.serve_requests, 5, args.serve_rate)
    budget = int(150e9)
    work = sum(d.cells * steps for _, d, steps, _ in reqs)
    res = {
        "workload": f"served stream: {len(reqs)} solves, Poisson arrivals at {args.serve_rate:g}/s, "
                    "box edge log-uniform 32-192, 50-1000 steps (log-uniform), Mt U[0.1,0.6], "
                    "Re_lambda U[40,120], scheme WENO5-JS/WENO5-Z/CRWENO5, seeded HIT on device, "
                    "final state copied to the host; HBM budget 150 GB",
        "requests": len(reqs),
        "cell_updates_requested": work,
        "schemes": {k: sum(1 for _, d, _, _ in reqs if d.scheme[0] == v)
                    for k, v in (("weno5js", nb.WENO5JS), ("weno5z", nb.WENO5Z),
                                 ("crweno5", nb.CRWENO5))},
        "mixed_continuous": run_stream(reqs, nb.MIXED, 256, budget),
        "fp64_serial": run_stream(reqs, nb.FP64, 1, budget),
        # the same 32 solves submitted at once: the whole mix runs as one
        # batch from the start, the ceiling of the continuous stream
        "mixed_one_batch": run_stream(reqs, nb.MIXED, 256, budget, burst=True),
    }
    res["solves_per_s_ratio"] = (res["mixed_continuous"]["solves_per_s"]
                                 / res["fp64_serial"]["solves_per_s"])
    res["continuous_vs_one_batch"] = (res["mixed_continuous"]["cell_updates_per_s"]
                                      / res["mixed_one_batch"]["cell_updates_per_s"])
    return res


# ------------------------------------------------------- reference arm -----
def run_reference(args, rank, world):
    if rank != 0:
        return None
    import nuc3d_b200 as nb
    n = args.cpu_n
    desc = nb.BoxDesc(n, n, n, mach=1.0)
    _, reynolds = nb.hit_field(desc, seed=SEED, k_peak=K_PEAK, mach_t=MACH_T, re_lambda=RE_LAMBDA)
    workers = args.cpu_workers or min(os.cpu_count() or 1, 64)
    value, wall, kind = cpu_sample(n, args.steps, args.warmup, reynolds, workers)
    sample = (f"{workers} concurrent {n}^3 boxes (one per core, the reference's single-rank "
              f"code), {args.warmup}+{args.steps} steps each, same physics and scheme")
    cfg = config_dict(world, reynolds)
    cfg["reference_sample"] = sample
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded HIT field)",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    global NX, METRIC
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--n", type=int, default=NX, help="box edge (default 256; smaller only for profiling)")
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--skip-mixed", action="store_true")
    ap.add_argument("--skip-ensemble", action="store_true")
    ap.add_argument("--skip-schemes", action="store_true")
    ap.add_argument("--ensemble-boxes", type=int, default=64)
    ap.add_argument("--accuracy-steps", type=int, default=100)
    ap.add_argument("--repeats", type=int, default=5,
                    help="timed regions of --steps steps each; value from the median")
    ap.add_argument("--skip-long", action="store_true")
    ap.add_argument("--long-steps", type=int, default=2000)
    ap.add_argument("--long-every", type=int, default=100)
    ap.add_argument("--skip-config3", action="store_true")
    ap.add_argument("--c3-n", type=int, default=384)
    ap.add_argument("--c3-steps", type=int, default=100, help="steps compared FP64 vs mixed")
    ap.add_argument("--c3-long", type=int, default=500, help="mixed steps checked for finiteness")
    ap.add_argument("--skip-serve", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=32)
    ap.add_argument("--serve-rate", type=float, default=20.0, help="mean arrivals per second")
    ap.add_argument("--cpu-n", type=int, default=48, help="box edge of the CPU sample")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--cpu-workers", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.repeats < 1:
        ap.error("--repeats must be >= 1")
    NX = args.n
    METRIC = METRIC.replace("256^3", f"{NX}^3")
    from nuc3d_b200.replicas import rank_info
    ri = rank_info(default_world=args.gpus)
    rank, world, local_rank = ri.rank, ri.world, ri.local_rank

    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    args.cpu_result = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # before any CUDA call: the CPU pool is spawned from a clean process
        import nuc3d_b200 as nb
        d = nb.BoxDesc(args.cpu_n, args.cpu_n, args.cpu_n, mach=1.0)
        _, re_cpu = nb.hit_field(d, seed=SEED, k_peak=K_PEAK, mach_t=MACH_T, re_lambda=RE_LAMBDA)
        workers = args.cpu_workers or min(os.cpu_count() or 1, 64)
        v, wall, kind = cpu_sample(args.cpu_n, args.cpu_steps, 0, re_cpu, workers)
        args.cpu_result = {
            "value": v, "unit": UNIT, "cores": workers, "kind": kind,
            "sample": f"{workers} concurrent {args.cpu_n}^3 HIT boxes (one per core), "
                      f"{args.cpu_steps} TVD-RK3 steps each, WENO5-Z N-S, {wall:.1f} s",
        }
    line = run_b200(args, rank, world, local_rank)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
