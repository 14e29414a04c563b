"""Benchmark of the OSCARS radiation hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl product|reference] [--compute fp64|mixed]

Workload (one "step"): single-electron flux on a 201 x 201 XY rectangle, 10 mm x 10 mm at z = 30 m,
at the first harmonic E1 = 458.9458 eV of a 41-period planar undulator (B0 = 0.5 T, 50 mm period),
3 GeV electron, 20001-point FP64 RK4 trajectory, adaptive level ladder (precision 0.01).  Inputs
are seeded synthetic stand-ins for the reference's example workloads.  Metric: Gsamples/s, one
sample = one (observer, energy, trajectory point) term of the radiation sum, counted as
2^(L+1)-1 per entry for stop level L.

``value``  flux integral with trajectory and observers resident in HBM (level samples rebuilt
           every step); CUDA events per step on the launching stream, L2 flushed between steps.
``e2e``    the same job through the C ABI (osc_flux) with pinned host buffers: observers copied
           in, level samples rebuilt, kernels, flux and levels copied out, every step; the
           trajectory is computed once before the loop, as in the reference arm's step.
           ``e2e.with_new_trajectory`` also draws a new particle every step (host RK4 + spline +
           trajectory upload inside the timing).
Under torchrun each rank runs its own job (energy E1 * (1 + 1e-3 rank)): no collective on the data
path, weak scaling; the reported time is the max over ranks.  The 10k-particle EPU beam is then run
split over the ranks (``epu_beam_10k_sharded``: particles round-robin, one NCCL all_reduce of the
partial fluxes, strong scaling).

``batched`` (single GPU) adds the two batched workloads: a 10k-particle EPU beam (101 x 101 flux)
and 512 uneven undulator jobs, each timed on the device (every chunk of jobs from its first to its
last kernel, device RK4 and splines included) and end to end through the public API, beside the
FP64 reference method on a subset of the same particles / jobs and the mixed-vs-FP64 error at a
fixed level.  ``tuning`` adds the differentiable field-tuning workload (gradient of a flux loss with
respect to 82 half-period undulator amplitudes) in grad/s.  ``--only beam|uneven|tuning`` runs one
of them alone.

``--impl reference`` times the reference's own CPU implementation (oracle/_ref, built from the
reference sources by oracle/Makefile; the CPU restatement in oracle/ when that build is absent)
on all host cores, on the same workload and metric.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import math
import os
import re
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("flux-integral Gsamples/s (obs×E×traj), mixed vs FP64 GPU at ≤1e-4 rel; grad/s")
E1 = 458.9458
GRID = 201
WORKLOAD = ("flux 201x201 XY rectangle 10mm x 10mm at z=30m, E=E1=458.9458 eV; planar undulator "
            "B0=0.5T lambda=50mm 41 periods; 3 GeV electron; 20001-point RK4; adaptive levels (precision 0.01)")
FLOP_PER_SAMPLE = 83  # algorithmic work per sample of the frequency-domain integrand


def _profiled_traffic():
    """DRAM bytes (read + write) per launch of each profiled kernel variant, from the ncu summaries
    under profiles/ (lines 'traffic per launch (dram read + write), <kernel>: <bytes> B')."""
    out = {}
    pat = re.compile(r"^traffic per launch \(dram read \+ write\), (\S+): (\d+) B")
    pdir = os.path.join(ROOT, "profiles")
    for fn in sorted(os.listdir(pdir)) if os.path.isdir(pdir) else []:
        if fn.endswith(".md"):
            for line in open(os.path.join(pdir, fn)):
                mt = pat.match(line.strip())
                if mt:
                    out[mt.group(1)] = int(mt.group(2))
    return out


def setup(o):
    o.add_bfield_undulator(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41, phase=-math.pi / 2)
    o.set_particle_beam(type="electron", energy_GeV=3, x0=[0, 0, 0], d0=[0, 0, 1], current=0.5)
    o.set_ctstartstop(-1.5, 1.5)
    o.set_npoints_trajectory(20001)


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons read through NVML every 20 ms while the timed
    region runs (the same counters `nvidia-smi --query-gpu=clocks.sm,clocks_event_reasons.*`
    reports).  Read-only: no setting of the GPU is touched."""
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._thr = None
        self.error = None

    def _run(self):
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            while not self._stop.is_set():
                self.samples.append((N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM),
                                     N.nvmlDeviceGetCurrentClocksEventReasons(h)))
                time.sleep(0.02)
        except Exception as e:  # no NVML: report it, the number itself is unaffected
            self.error = repr(e)

    def __enter__(self):
        self._thr = threading.Thread(target=self._run, daemon=True)
        self._thr.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._thr.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no NVML samples: %s" % self.error]}
        sm = sorted(c for c, _ in self.samples)
        reasons = sorted({name for _, r in self.samples for bit, name in self.REASONS.items() if r & bit})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples)}


def _quiet_import_reference():
    """Import the reference build with its start-up banner kept off stdout (the JSON line is ours)."""
    from oracle.oracle import reference_module
    sys.stdout.flush()
    saved = os.dup(1)
    try:
        os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
        return reference_module()
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)


def _cpu_flux_rows(o, kind, cores, nrows):
    """Flux on the central `nrows` rows of the 201 x 201 grid (same point spacing); returns
    (seconds, samples) with samples counted from the CPU path's own stop levels."""
    import numpy as np
    w1 = 0.01 * (nrows - 1) / (GRID - 1)
    kw = dict(energy_eV=E1, npoints=[nrows, GRID], width=[w1 if nrows > 1 else 1e-9, 0.01], translation=[0, 0, 30])
    if kind == "reference":
        kw["nthreads"] = cores
    t0 = time.perf_counter()
    o.calculate_flux_rectangle(**kw)
    dt = time.perf_counter() - t0
    lev = np.array([v for _, v in o.calculate_flux_rectangle(**dict(kw, quantity="level"))])
    return dt, float(np.sum(2.0 ** (lev + 1) - 1))


def _cpu_impl():
    from oracle.oracle import OracleSR
    S = _quiet_import_reference()
    cores = os.cpu_count() or 1
    if S is not None:
        return "reference", cores, S.sr(nthreads=cores, gpu=0)
    return "port", 1, OracleSR()


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def _cpu_flux_timed(o, kind, cores, nrows, passes):
    """`passes` timed passes of the flux on the central `nrows` rows; (list of seconds, samples per
    pass) with samples counted once from the CPU path's own stop levels (untimed)."""
    import numpy as np
    w1 = 0.01 * (nrows - 1) / (GRID - 1)
    kw = dict(energy_eV=E1, npoints=[nrows, GRID], width=[w1 if nrows > 1 else 1e-9, 0.01], translation=[0, 0, 30])
    if kind == "reference":
        kw["nthreads"] = cores
    times = []
    for _ in range(passes):
        t0 = time.perf_counter()
        o.calculate_flux_rectangle(**kw)
        times.append(time.perf_counter() - t0)
    lev = np.array([v for _, v in o.calculate_flux_rectangle(**dict(kw, quantity="level"))])
    return times, float(np.sum(2.0 ** (lev + 1) - 1))


def reference_arm(args):
    """The reference's own CPU implementation on all host threads (rank 0 only): every step is the
    whole 201 x 201 flux of the product arm's workload, same metric and config."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    kind, cores, o = _cpu_impl()
    setup(o)
    o.calculate_trajectory()
    if args.warmup > 0:
        _cpu_flux_timed(o, kind, cores, GRID, 1)
    times, samples = _cpu_flux_timed(o, kind, cores, GRID, args.steps)
    total = sum(times)
    value = samples * args.steps / total / 1e9
    desc = "full 201 x 201 grid per step, %d steps, %d threads, %s" % (args.steps, cores, _cpu_model())
    line = {"metric": METRIC, "value": value, "unit": "Gsamples/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": product_config(1), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "Gsamples/s", "cores": cores, "kind": kind, "sample": desc,
                             "cpu_model": _cpu_model()},
            "e2e": {"value": value, "unit": "Gsamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def product_config(world):
    return {"workload": WORKLOAD, "compute": "mixed", "l2": "flushed between steps (256 MB write)",
            "parallelism": "independent job per rank" if world > 1 else "single GPU"}


def cpu_baseline_leg():
    """The reference CPU path on the headline workload: all host threads over the whole 201 x 201
    grid (one pass), and one thread over the central rows that take about 5 s."""
    kind, cores, o = _cpu_impl()
    setup(o)
    o.calculate_trajectory()
    t_all, s_all = _cpu_flux_timed(o, kind, cores, GRID, 1)
    out = {"value": s_all / t_all[0] / 1e9, "unit": "Gsamples/s", "cores": cores, "kind": kind,
           "sample": "whole 201 x 201 grid, one pass, %.2f s" % t_all[0], "cpu_model": _cpu_model()}
    if kind == "reference":
        t5, _ = _cpu_flux_timed(o, kind, 1, 5, 1)
        rows = int(max(5, min(GRID, 5.0 / max(t5[0] / 5, 1e-6))))
        rows -= (rows + 1) % 2  # odd: the row set stays centred on the axis
        t1, s1 = _cpu_flux_timed(o, kind, 1, rows, 1)
        out["value_1thread"] = s1 / t1[0] / 1e9
        out["sample_1thread"] = "central %d of 201 rows x 201 columns, one pass, %.2f s, 1 thread" % (rows, t1[0])
    return out


def _time_device_steps(ctx, step, stream, flush, steps, warmup, local):
    """Per-step CUDA events on the launching stream, L2 flushed before every step (outside the
    events), the library's own per-launch profiling off.  Returns (per-step ms list, samples per step,
    launches per step, clocks)."""
    import ctypes
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    sm, ln = ctypes.c_longlong(), ctypes.c_longlong()
    ctx.call("osc_last_stats", ctypes.byref(sm), ctypes.byref(ln))  # the job is identical every step
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with ClockSampler(local) as clk:
        time.sleep(0.1)
        for i in range(steps):
            flush.zero_()
            evs[i][0].record(stream)
            step()
            evs[i][1].record(stream)
        torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs], sm.value, ln.value, clk.summary()


def _kernel_time(ctx, step, flush, steps):
    """Summed device time [ms] and count of the sample-sum kernel launches over `steps` steps, from the
    library's per-launch CUDA events (a separate pass: those events are off while `value` is timed)."""
    import ctypes
    import torch
    ctx.call("osc_set_profiling", 1)
    ctx.call("osc_get_profile", None, None, None, 1)
    for _ in range(steps):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    kms, kl = ctypes.c_double(), ctypes.c_longlong()
    ctx.call("osc_get_profile", ctypes.byref(kms), ctypes.byref(kl), None, 1)
    ctx.call("osc_set_profiling", 0)
    return kms.value, kl.value


def _long_run(step, stream, flush, min_s=1.0):
    """Steps repeated (L2 flushed before each, outside the events) until the timed total reaches
    min_s seconds: (steps, total ms)."""
    import torch
    total, n = 0.0, 0
    while total < 1e3 * min_s:
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(200)]
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            step()
            b.record(stream)
        torch.cuda.synchronize()
        total += sum(a.elapsed_time(b) for a, b in evs)
        n += len(evs)
    return n, total


PD_WORKLOAD = ("power density on the flux headline's 201x201 XY rectangle (10mm x 10mm at z=30m), same undulator, "
               "beam and trajectory; adaptive levels (precision 0.01); device-resident observers and outputs, level "
               "samples rebuilt every step")


def power_density_leg(ctx, d_obs, n, stream, flush, steps, warmup, local):
    """Power density on the headline grid (config 1), FP64 and mixed, timed like the flux headline;
    the mixed / FP64 peak-normalised difference at the fixed level 12."""
    import ctypes
    import numpy as np
    import torch
    from oscars_b200._lib import RadOpts
    dev = d_obs.device
    sptr = ctypes.c_void_p(stream.cuda_stream)
    d_lvl = torch.zeros(n, dtype=torch.int32, device=dev)
    out, arrays = {}, {}
    for m in ("fp64", "mixed"):
        def opts(**kw):
            o = RadOpts(precision=kw.get("precision", 0.01), max_level=kw.get("max_level", -2), max_level_extended=0,
                        nparticles=0, quantity=0, precision_mode=1 if m == "mixed" else 0)
            o.horizontal[:] = [1, 0, 0]
            o.propagation[:] = [0, 0, 1]
            return o
        o = opts()
        d_out = torch.zeros(n, dtype=torch.float64, device=dev)

        def step(o=o, d_out=d_out):
            ctx.call("osc_drop_level_cache")
            ctx.call("osc_power_density_device", ctypes.c_void_p(d_obs.data_ptr()), None, n, 0, ctypes.byref(o),
                     ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_lvl.data_ptr()), sptr)
        per, sps, lps, clocks = _time_device_steps(ctx, step, stream, flush, steps, warmup, local)
        ms = sum(per)
        out[m] = {"value": sps * steps / (ms * 1e-3) / 1e9, "unit": "Gsamples/s", "ms_per_step": ms / steps,
                  "samples_per_step": sps, "gpu_launches_per_step": lps, "clocks": clocks}
        of = opts(precision=0.0, max_level=12)
        ctx.call("osc_power_density_device", ctypes.c_void_p(d_obs.data_ptr()), None, n, 0, ctypes.byref(of),
                 ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_lvl.data_ptr()), sptr)
        torch.cuda.synchronize(dev)
        arrays[m] = d_out.cpu().numpy().copy()
    err = float(np.max(np.abs(arrays["mixed"] - arrays["fp64"])) / np.max(np.abs(arrays["fp64"])))
    return {"workload": PD_WORKLOAD, "steps": steps, "warmup": warmup, "fp64": out["fp64"], "mixed": out["mixed"],
            "mixed_over_fp64": out["mixed"]["value"] / out["fp64"]["value"],
            "mixed_vs_fp64_peak_rel_err": {"value": err, "fixed_level": 12}}


def power_density_only(steps, warmup):
    """The power-density leg alone on GPU 0 (for profiler runs)."""
    import torch
    from oscars_b200.sr import sr
    s = sr(gpu=1, device=0)
    setup(s)
    s.calculate_trajectory()
    xyz = s._rectangle([GRID, GRID], "XY", [0.01, 0.01], None, None, [0, 0, 30], 0, False)[0]
    dev = torch.device("cuda", 0)
    d_obs = torch.tensor(xyz, dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    torch.cuda.synchronize(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    return power_density_leg(s._ctx, d_obs, GRID * GRID, stream, flush, steps, warmup, 0)


def product_arm(args):
    import ctypes
    import numpy as np
    import torch
    import torch.distributed as dist
    from oscars_b200 import _lib
    from oscars_b200._lib import RadOpts
    from oscars_b200.sr import sr

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    energy = E1 * (1 + 1e-3 * rank)
    s = sr(gpu=1, device=local)
    setup(s)
    s.calculate_trajectory()
    ctx = s._ctx
    if args.variant >= 0:  # a fixed kernel variant (profiler runs: no autotuning under the profiler)
        ctx.call("osc_set_variant", 2 if args.compute == "mixed" else 0, args.variant)
    xyz, nrm, x12 = s._rectangle([GRID, GRID], "XY", [0.01, 0.01], None, None, [0, 0, 30], 0, False)
    n = GRID * GRID
    modes = ["fp64", "mixed"] if args.compute == "mixed" else ["fp64"]
    opts = {}
    for m in modes:
        o = RadOpts(precision=0.01, max_level=-2, max_level_extended=0, nparticles=0, quantity=0,
                    precision_mode=1 if m == "mixed" else 0)
        o.horizontal[:] = [1, 0, 0]
        o.propagation[:] = [0, 0, 1]
        opts[m] = o
    dev = torch.device("cuda", local)
    d_obs = torch.tensor(xyz, dtype=torch.float64, device=dev)
    d_out = {m: torch.zeros(n, dtype=torch.float64, device=dev) for m in modes}
    d_lvl = torch.zeros(n, dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    # one dedicated stream: the library's kernels, the L2 flush and the timing events all go on it
    torch.cuda.synchronize(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def make_step(m):
        def step():
            ctx.call("osc_drop_level_cache")  # level samples are rebuilt inside every step
            ctx.call("osc_flux_device", ctypes.c_void_p(d_obs.data_ptr()), n, energy, ctypes.byref(opts[m]),
                     ctypes.c_void_p(d_out[m].data_ptr()), ctypes.c_void_p(d_lvl.data_ptr()), sptr)
        return step

    res = {}
    for m in modes:
        if world > 1:
            dist.barrier()
        per, sps, lps, clocks = _time_device_steps(ctx, make_step(m), stream, flush, args.steps, args.warmup, local)
        ms = sum(per)
        t = torch.tensor([ms, float(sps * args.steps)], dtype=torch.float64, device=dev)
        if world > 1:
            tmax, tsum = t.clone(), t.clone()
            dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
            dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
            ms_max, samples_all = float(tmax[0]), float(tsum[1])
        else:
            ms_max, samples_all = ms, float(sps * args.steps)
        kms, kl = _kernel_time(ctx, make_step(m), flush, args.steps)
        long_n, long_ms = _long_run(make_step(m), stream, flush) if not args.quick else (0, 0.0)
        v, nv = ctypes.c_int(), ctypes.c_int()
        ctx.call("osc_get_variant", 2 if m == "mixed" else 0, ctypes.byref(v), ctypes.byref(nv))
        peak = ctypes.c_double()
        ctx.call("osc_measure_fma_peak", 0 if m == "fp64" else 1, ctypes.byref(peak))
        achieved = sps * args.steps * FLOP_PER_SAMPLE / (kms * 1e-3) / 1e12 if kms > 0 else None
        kname = _lib.variant_name(2 if m == "mixed" else 0, v.value)
        traffic = _profiled_traffic().get(kname)
        srt = sorted(per)
        res[m] = {"value": samples_all / (ms_max * 1e-3) / 1e9, "ms_per_step": ms_max / args.steps,
                  "samples_per_step": sps, "launches_per_step": lps, "variant": v.value, "clocks": clocks,
                  "roofline": {"bound": "fp64" if m == "fp64" else "fp32", "achieved": achieved, "peak": peak.value,
                               "unit": "TFLOP/s", "frac": (achieved / peak.value) if achieved else None,
                               "traffic": traffic, "kernel": kname, "flop_per_sample": FLOP_PER_SAMPLE,
                               "kernel_ms_per_step": kms / args.steps, "kernel_launches_per_step": kl / args.steps,
                               "peak_source": "in-run FMA-throughput loop on this GPU (osc_measure_fma_peak); the "
                                              "sample sums run on the %s pipe, not the tensor cores or HBM"
                                              % ("FP64" if m == "fp64" else "FP32/SFU"),
                               "step_ms_median": srt[len(srt) // 2], "step_ms_min": srt[0], "step_ms_max": srt[-1],
                               "long_run_steps": long_n, "long_run_s": long_ms * 1e-3,
                               "long_run_value": sps * long_n / (long_ms * 1e-3) / 1e9 if long_ms > 0 else None}}
    head = modes[-1]
    err = None
    if "mixed" in res:
        a, b = d_out["mixed"].cpu().numpy(), d_out["fp64"].cpu().numpy()
        err = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))

    if args.quick:
        if rank == 0:
            print(json.dumps({"quick": True, "compute": head, "modes": res, "mixed_vs_fp64_peak_rel_err": err}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    # e2e: the user's call through the C ABI with host buffers in pinned memory: observers in, flux and
    # levels out, copies inside the timed call.  Like the reference arm's step, the trajectory is the
    # one computed before the timed loop; the level samples are rebuilt every step.  A second figure
    # draws a new particle every step (host RK4 + spline + trajectory upload inside the timing).
    xyz_p = torch.from_numpy(np.ascontiguousarray(xyz)).pin_memory()
    out_p = torch.zeros(n, dtype=torch.float64).pin_memory()
    lvl_p = torch.zeros(n, dtype=torch.int32).pin_memory()
    xyz_h, out_h, lvl_h = xyz_p.numpy(), out_p.numpy(), lvl_p.numpy()  # numpy views of the pinned buffers
    nnc = ctypes.c_longlong()

    def e2e_run(new_particle):
        def e2e_step():
            if new_particle:
                s.set_new_particle(particle="ideal")  # drops the trajectory: RK4 + spline + upload again
            else:
                ctx.call("osc_drop_level_cache")
            ctx.call("osc_flux", _lib.dptr(xyz_h), n, energy, ctypes.byref(opts[head]), _lib.dptr(out_h),
                     _lib.i32ptr(lvl_h), ctypes.byref(nnc))
        e2e_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        times, samples = [], 0
        for i in range(max(1, min(args.steps, 20))):
            t0 = time.perf_counter()
            e2e_step()
            times.append(time.perf_counter() - t0)
            sm = ctypes.c_longlong()
            ctx.call("osc_last_stats", ctypes.byref(sm), None)
            samples += sm.value
        te = torch.tensor([sum(times), float(samples)], dtype=torch.float64, device=dev)
        if world > 1:
            tm, ts = te.clone(), te.clone()
            dist.all_reduce(tm, op=dist.ReduceOp.MAX)
            dist.all_reduce(ts, op=dist.ReduceOp.SUM)
            return float(ts[1]) / float(tm[0]) / 1e9
        return samples / sum(times) / 1e9

    e2e_value = e2e_run(False)
    e2e_traj_value = e2e_run(True)
    pd = None
    if "mixed" in modes:  # config 1's power density on the same grid, FP64 and mixed
        pd = power_density_leg(ctx, d_obs, n, stream, flush, min(args.steps, 50), max(3, args.warmup), local)
    h2d = xyz.nbytes + 8
    d2h = n * 8 + n * 4
    sharded = None
    if world > 1 and args.batched_steps > 0:  # every rank takes part in its collectives
        try:
            sharded = sharded_beam_leg(args.batched_steps, max(3, args.warmup), local, rank, world)
        except Exception as e:  # reported in the line; the headline stands
            sharded = {"error": "%s: %s" % (type(e).__name__, e)}
    if rank == 0:
        cpu = cpu_baseline_leg() if world == 1 else None
        r = res[head]
        roof = dict(r["roofline"])
        if "mixed" in res:  # the plain FP64 path of the same run, flat so that the record keeps it
            f = res["fp64"]
            roof.update({"fp64_value": f["value"], "fp64_ms_per_step": f["ms_per_step"],
                         "fp64_kernel": f["roofline"]["kernel"], "fp64_achieved": f["roofline"]["achieved"],
                         "fp64_peak": f["roofline"]["peak"], "fp64_frac": f["roofline"]["frac"],
                         "fp64_traffic": f["roofline"]["traffic"], "fp64_long_run_value": f["roofline"]["long_run_value"],
                         "mixed_over_fp64": r["value"] / f["value"], "mixed_vs_fp64_peak_rel_err": err})
        line = {"metric": METRIC, "value": r["value"], "unit": "Gsamples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32+f64", "data": "synthetic",
                "config": dict(product_config(world), compute=head),
                "e2e": {"value": e2e_value, "unit": "Gsamples/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "host_buffers": "pinned", "path": "osc_flux (C ABI), trajectory computed before the loop as in the reference arm",
                        "with_new_trajectory_value": e2e_traj_value,
                        "with_new_trajectory_h2d_bytes_per_step": h2d + 19 * 20001 * 8,
                        "with_new_trajectory_note": "new particle every step: host RK4 + spline + trajectory upload timed too"},
                "gpu_launches": r["launches_per_step"] * args.steps, "roofline": roof, "cpu_baseline": cpu,
                "clocks": r["clocks"]}
        if "mixed" in res:
            line["fp64"] = {"value": res["fp64"]["value"], "ms_per_step": res["fp64"]["ms_per_step"],
                            "roofline": res["fp64"]["roofline"], "clocks": res["fp64"]["clocks"]}
        if pd is not None:
            line["power_density"] = pd
            line["roofline"].update({"pd_value": pd["mixed"]["value"], "pd_fp64_value": pd["fp64"]["value"],
                                     "pd_mixed_over_fp64": pd["mixed_over_fp64"],
                                     "pd_mixed_vs_fp64_peak_rel_err": pd["mixed_vs_fp64_peak_rel_err"]["value"]})
        if world == 1 and args.batched_steps > 0:
            bw = max(3, args.warmup)
            line["batched"] = {"note": "inputs far larger than L2 (GBs of level records); device time = each "
                                       "chunk of jobs from first to last kernel, trajectories included",
                               "epu_beam_10k": beam_leg(args.batched_steps, bw, local),
                               "uneven_512": uneven_leg(args.batched_steps, bw, local)}
            line["tuning"] = tuning_leg(max(5, args.batched_steps), bw, local)
            bb, bu, bt = line["batched"]["epu_beam_10k"], line["batched"]["uneven_512"], line["tuning"]
            line["roofline"].update({  # the batched workloads' headline figures, flat so that the record keeps them
                "beam_value": bb["value"], "beam_fp64_value": bb["fp64"]["value"],
                "beam_mixed_over_fp64": bb["mixed_over_fp64"], "uneven_value": bu["value"],
                "uneven_fp64_value": bu["fp64"]["value"], "uneven_mixed_over_fp64": bu["mixed_over_fp64"],
                "tuning_grad_per_s": bt["value"], "tuning_fp64_grad_per_s": bt["fp64"]["value"],
                "tuning_grad_vs_fd": bt["grad_vs_richardson_fd"]["value"],
                "beam_cpu_reference_value": (bb["cpu_reference"] or {}).get("value"),
                "uneven_cpu_reference_value": (bu["cpu_reference"] or {}).get("value"),
                "tuning_cpu_reference_grad_per_s": (bt["cpu_reference"] or {}).get("value")})
        if sharded is not None:
            line["epu_beam_10k_sharded"] = sharded
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------
# Batched workloads (mixed precision through the batch path, FP64 through the single-trajectory
# path on a subset of the same particles / jobs)
# ---------------------------------------------------------------------------------------------
E1_EPU = 179.2558
BEAM_PARTICLES = 10000
BEAM_WORKLOAD = ("EPU beam: By=0.6T cos + Bx=0.4T sin, lambda=57mm, 30 periods; 3 GeV electrons, sigma_E=3 MeV, "
                 "emittance (0.9 nm, 8 pm), beta (1.5, 0.8) m, alpha 0; %d particles (seed 1), 16001-point RK4 each; "
                 "flux 101x101 on 8mm x 8mm at z=30m at E1=179.2558 eV; adaptive levels" % BEAM_PARTICLES)
UNEVEN_JOBS = 512
UNEVEN_WORKLOAD = ("%d uneven jobs (seed 2024): planar undulators lambda~U[15,100]mm, B0~U[0.2,1.2]T, N~U{10..200}, "
                   "4k-64k RK4 points; 1-4096 observers (rectangles, z~U[20,40]m) x 1-256 energies within E1 +-5%%; "
                   "adaptive levels" % UNEVEN_JOBS)


def setup_epu_beam(o, seed=1):
    o.add_bfield_undulator(bfield=[0, 0.6, 0], period=[0, 0, 0.057], nperiods=30, phase=-math.pi / 2)
    o.add_bfield_undulator(bfield=[0.4, 0, 0], period=[0, 0, 0.057], nperiods=30, phase=0)
    o.set_particle_beam(type="electron", energy_GeV=3, x0=[0, 0, 0], d0=[0, 0, 1], current=0.5,
                        sigma_energy_GeV=0.003, beta=[1.5, 0.8], alpha=[0, 0], emittance=[0.9e-9, 8e-12])
    o.set_ctstartstop(-1.5, 1.5)
    o.set_npoints_trajectory(16001)
    o.set_seed(seed)


def _e1_eV(bfield, period, energy_GeV=3.0):
    lam_cm = period * 100
    K = 0.9337 * bfield * lam_cm
    return 1000 * 0.9496 * energy_GeV ** 2 / (lam_cm * (1 + K * K / 2))


def uneven_jobs(seed=2024, n=UNEVEN_JOBS):
    import numpy as np
    from oscars_b200.batch import Job, undulator
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n):
        lam = rng.uniform(0.015, 0.10)
        B = rng.uniform(0.2, 1.2)
        N = int(rng.integers(10, 201))
        half = lam * (N + 2) / 2 + 0.2
        npts = int(np.clip(240 * (N + 2 + 0.4 / lam), 4096, 65536))  # ~240 points per period plus drifts
        nx, ny = int(rng.integers(1, 65)), int(rng.integers(1, 65))
        wx, wy = rng.uniform(0.001, 0.006, 2)
        z = rng.uniform(20, 40)
        xs = np.linspace(-wx / 2, wx / 2, nx) if nx > 1 else np.zeros(1)
        ys = np.linspace(-wy / 2, wy / 2, ny) if ny > 1 else np.zeros(1)
        X, Y = np.meshgrid(xs, ys, indexing="ij")
        obs = np.stack([X.ravel(), Y.ravel(), np.full(X.size, z)], 1)
        ne = int(rng.integers(1, 257))
        e1 = _e1_eV(B, lam)
        jb = Job(fields=[undulator([0, B, 0], [0, 0, lam], N, phase=-math.pi / 2)], energy_GeV=3.0,
                 ctstartstop=(-half, half), npoints=npts, obs=obs, energies_eV=np.linspace(0.95 * e1, 1.05 * e1, ne),
                 current=0.5)
        jb.setup = (lam, B, N, half, npts, nx, ny, wx, wy, z)  # for the reference CPU subset
        jobs.append(jb)
    return jobs


def _profiled(ctx, fn):
    """fn() with device profiling on: (result, device ms, samples, launches, wall s)."""
    import ctypes
    ctx.call("osc_set_profiling", 1)
    ctx.call("osc_get_profile", None, None, None, 1)
    t0 = time.perf_counter()
    r = fn()
    wall = time.perf_counter() - t0
    ms, ns = ctypes.c_double(), ctypes.c_longlong()
    ctx.call("osc_get_profile", ctypes.byref(ms), None, ctypes.byref(ns), 1)
    ctx.call("osc_set_profiling", 0)
    sm, ln = ctypes.c_longlong(), ctypes.c_longlong()
    ctx.call("osc_last_stats", ctypes.byref(sm), ctypes.byref(ln))
    return r, ms.value, sm.value, ln.value, wall


def _peak_err(a, b):
    import numpy as np
    a, b = np.asarray(a, dtype=np.float64).ravel(), np.asarray(b, dtype=np.float64).ravel()
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _cpu_reference():
    """(the reference's own CPU module, host threads) or (None, 0) when oracle/_ref is absent."""
    S = _quiet_import_reference()
    return (S, os.cpu_count() or 1) if S is not None else (None, 0)


def beam_cpu_reference(particles):
    """The reference CPU path on the first `particles` particles of the EPU beam (seed 1), all host
    threads: seconds for the 101 x 101 flux (particles are independent, so the time per particle
    extrapolates linearly to the 10k beam)."""
    S, cores = _cpu_reference()
    if S is None:
        return None, 0
    o = S.sr(nthreads=cores, gpu=0)
    setup_epu_beam(o)
    o.set_seed(1)
    t0 = time.perf_counter()
    o.calculate_flux_rectangle(energy_eV=E1_EPU, npoints=[101, 101], width=[0.008, 0.008], translation=[0, 0, 30],
                               nparticles=particles, nthreads=cores)
    return time.perf_counter() - t0, cores


def uneven_cpu_reference(jobs, n=8):
    """The reference CPU path on a subset of the uneven jobs: the first n with at least 2 x 2
    observers, each at the middle one of its energies, all host threads; (seconds, samples counted
    from the CPU path's own stop levels, jobs, cores)."""
    import numpy as np
    S, cores = _cpu_reference()
    if S is None:
        return None
    total_t, samples, used = 0.0, 0.0, 0
    for jb in jobs:
        lam, B, N, half, npts, nx, ny, wx, wy, z = jb.setup
        if nx < 2 or ny < 2:
            continue
        o = S.sr(nthreads=cores, gpu=0)
        o.add_bfield_undulator(bfield=[0, B, 0], period=[0, 0, lam], nperiods=N, phase=-math.pi / 2)
        o.set_particle_beam(type="electron", energy_GeV=3.0, x0=[0, 0, 0], d0=[0, 0, 1], current=0.5)
        o.set_ctstartstop(-half, half)
        o.set_npoints_trajectory(npts)
        o.calculate_trajectory()
        e = float(jb.energies_eV[len(jb.energies_eV) // 2])
        kw = dict(energy_eV=e, npoints=[nx, ny], width=[wx, wy], translation=[0, 0, z], nthreads=cores)
        t0 = time.perf_counter()
        o.calculate_flux_rectangle(**kw)
        total_t += time.perf_counter() - t0
        lev = np.array([v for _, v in o.calculate_flux_rectangle(**dict(kw, quantity="level"))])
        samples += float(np.sum(2.0 ** (lev + 1) - 1))
        used += 1
        if used == n:
            break
    return total_t, samples, used, cores


def tuning_cpu_reference(every=16, h=1e-3):
    """One central-difference gradient component of the field-tuning loss through the reference CPU
    path (all host threads), on every `every`-th of the 256 energies: two loss evaluations, each a new
    trajectory through the half-period-scaled undulator (given to the reference as a Python field
    function with the undulator's operations) and the 21 x 21 flux per energy at level 12.  Returns
    (seconds for the subset, scale to the full gradient = 82 components x every, cores)."""
    import numpy as np
    S, cores = _cpu_reference()
    if S is None:
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from cases import halfscale_function
    energies = np.linspace(0.95 * E1, 1.05 * E1, 256)[::every]
    s0 = 1 + np.random.default_rng(82).normal(0.0, 0.005, 82)

    def loss_eval(scale):
        o = S.sr(nthreads=cores, gpu=0)
        o.add_bfield_function(halfscale_function([0, 0.5, 0], [0, 0, 0.05], 41, -math.pi / 2, list(scale)))
        o.set_particle_beam(type="electron", energy_GeV=3, x0=[0, 0, 0], d0=[0, 0, 1], current=0.5)
        o.set_ctstartstop(-1.5, 1.5)
        o.set_npoints_trajectory(20001)
        for e in energies:
            o.calculate_flux_rectangle(energy_eV=float(e), npoints=[21, 21], width=[0.002, 0.002],
                                       translation=[0, 0, 30], precision=0, max_level=12, nthreads=cores)
    e20 = np.zeros(82)
    e20[20] = h
    t0 = time.perf_counter()
    loss_eval(s0 + e20)
    loss_eval(s0 - e20)
    return time.perf_counter() - t0, 82 * every, cores


def beam_leg(steps, warmup, local=0, fp64_particles=32, check_particles=16, check_level=12, particles=BEAM_PARTICLES,
             quick=False):
    """EPU beam, 10k particles: mixed (batched) timed on the device and end to end; FP64 (reference
    path, host RK4 per particle) on the whole beam; both routes on the first `fp64_particles`; mixed
    vs FP64 error at a fixed level on `check_particles`.  `particles` < 10000 and `quick` (the mixed timing alone) give
    the small cases of profiler runs."""
    import numpy as np
    from oscars_b200.sr import sr
    s = sr(gpu=1, device=local)
    setup_epu_beam(s)
    s._ctx.call("osc_set_beam_batch_threshold", 1)  # the batched route whatever the particle count
    kw = dict(energy_eV=E1_EPU, npoints=[101, 101], width=[0.008, 0.008], translation=[0, 0, 30], return_numpy=True)

    def run(np_, compute, **extra):
        s.set_seed(1)
        return s.calculate_flux_rectangle(nparticles=np_, compute=compute, **dict(kw, **extra))
    for _ in range(warmup):
        run(particles, "mixed")
    dev_ms = wall = 0.0
    samples = launches = 0
    with ClockSampler(local) as clk:
        for _ in range(steps):
            _, ms, sm, ln, w = _profiled(s._ctx, lambda: run(particles, "mixed"))
            dev_ms += ms
            wall += w
            samples += sm
            launches += ln
    if quick:
        return {"particles": particles, "value": samples / (dev_ms * 1e-3) / 1e9, "unit": "Gsamples/s",
                "ms_per_step": dev_ms / steps, "gpu_launches_per_step": launches // steps}
    run(fp64_particles, "fp64")
    _, ms64, sm64, _, w64 = _profiled(s._ctx, lambda: run(fp64_particles, "fp64"))
    # the FP64 path on the whole beam (the same work as the mixed batch)
    _, ms64a, sm64a, _, w64a = _profiled(s._ctx, lambda: run(particles, "fp64"))
    # the same particles in mixed precision on the per-particle route (host trajectories,
    # single-trajectory mixed kernels), the route below the default batch threshold, timed like the
    # FP64 path's kernels
    s._ctx.call("osc_set_beam_batch_threshold", 1 << 30)
    run(fp64_particles, "mixed")
    _, ms_mx, sm_mx, _, w_mx = _profiled(s._ctx, lambda: run(fp64_particles, "mixed"))
    s._ctx.call("osc_set_beam_batch_threshold", 1)
    a = run(check_particles, "mixed", precision=0, max_level=check_level)[1]
    b = run(check_particles, "fp64", precision=0, max_level=check_level)[1]
    mixed_e2e = samples / wall / 1e9
    fp64_e2e = sm64a / w64a / 1e9
    fp64_dev = sm64a / (ms64a * 1e-3) / 1e9
    mixed_dev = samples / (dev_ms * 1e-3) / 1e9
    # the reference CPU path on the first cpu_particles particles (the FP64 GPU path's stop levels --
    # identical to the reference's -- count their samples)
    cpu_particles = 16
    run(cpu_particles, "fp64")
    _, _, sm_cpu, _, _ = _profiled(s._ctx, lambda: run(cpu_particles, "fp64"))
    t_cpu, cores = beam_cpu_reference(cpu_particles)
    cpu = None if t_cpu is None else {
        "value": sm_cpu / t_cpu / 1e9, "unit": "Gsamples/s", "cores": cores, "kind": "reference",
        "sample": "first %d of the 10000 particles, 101 x 101, %.1f s; per particle %.2f s, so the 10000-particle "
                  "beam extrapolates to %.0f s" % (cpu_particles, t_cpu, t_cpu / cpu_particles,
                                                  t_cpu / cpu_particles * BEAM_PARTICLES)}
    return {"workload": BEAM_WORKLOAD, "steps": steps, "warmup": warmup,
            "value": samples / (dev_ms * 1e-3) / 1e9, "unit": "Gsamples/s", "ms_per_step": dev_ms / steps,
            "samples_per_step": samples // steps, "gpu_launches_per_step": launches // steps,
            "e2e": {"value": mixed_e2e, "unit": "Gsamples/s", "wall_s_per_step": wall / steps,
                    "path": "sr.calculate_flux_rectangle(nparticles=10000, compute='mixed', return_numpy=True)"},
            "fp64": {"value": fp64_dev, "e2e": fp64_e2e, "unit": "Gsamples/s", "particles": particles,
                     "path": "sr.calculate_flux_rectangle(nparticles=%d, compute='fp64') (reference method: host RK4 "
                             "per particle on worker threads, FP64 sums); value = device time of its sample-sum "
                             "kernels (the mixed value counts the whole batch, device trajectories included)"
                             % particles},
            "mixed_over_fp64": mixed_dev / fp64_dev, "mixed_over_fp64_e2e": mixed_e2e / fp64_e2e,
            "same_particles": {"particles": fp64_particles, "mixed_value": sm_mx / (ms_mx * 1e-3) / 1e9,
                               "mixed_e2e": sm_mx / w_mx / 1e9, "fp64_value": sm64 / (ms64 * 1e-3) / 1e9,
                               "fp64_e2e": sm64 / w64 / 1e9,
                               "mixed_over_fp64": (sm_mx / ms_mx) / (sm64 / ms64),
                               "mixed_over_fp64_e2e": (sm_mx / w_mx) / (sm64 / w64),
                               "path": "the same %d particles through sr.calculate_flux_rectangle, mixed and FP64 "
                                       "(both per particle: host trajectories on worker threads); device time of the "
                                       "sample-sum kernels" % fp64_particles},
            "mixed_vs_fp64_peak_rel_err": {"value": _peak_err(a, b), "particles": check_particles,
                                           "fixed_level": check_level},
            "cpu_reference": cpu, "clocks": clk.summary()}


def uneven_leg(steps, warmup, local=0, fp64_jobs=32, check_level=12, n_jobs=UNEVEN_JOBS, quick=False):
    """512 uneven jobs through osc_batch_flux: mixed timed on the device and end to end; FP64 (jobs
    one after another through the FP64 path) on the same jobs; mixed vs FP64 error at a fixed level on
    the first `fp64_jobs`.  `n_jobs` < 512 (the first jobs of the same sequence) and `quick`
    (the mixed timing alone) give the small cases of profiler runs."""
    from oscars_b200.batch import BatchRunner
    jobs = uneven_jobs()[:n_jobs]
    r = BatchRunner(local)
    for _ in range(warmup):
        r.flux(jobs, compute="mixed")
    dev_ms = wall = 0.0
    samples = launches = 0
    with ClockSampler(local) as clk:
        for _ in range(steps):
            _, ms, sm, ln, w = _profiled(r.ctx, lambda: r.flux(jobs, compute="mixed"))
            dev_ms += ms
            wall += w
            samples += sm
            launches += ln
    variant = r.variant()[0]
    if quick:
        return {"jobs": n_jobs, "value": samples / (dev_ms * 1e-3) / 1e9, "unit": "Gsamples/s",
                "ms_per_step": dev_ms / steps, "gpu_launches_per_step": launches // steps, "variant": variant}
    sub = jobs[:fp64_jobs]
    r.ctx.call("osc_set_variant", 0, 2)  # FP64 variant fixed: no per-shape tuning runs inside the timing
    r.flux(sub, compute="fp64")
    _, ms64, sm64, _, w64 = _profiled(r.ctx, lambda: r.flux(jobs, compute="fp64"))  # all jobs: the same work
    a = r.flux(sub, compute="mixed", precision=0, max_level=check_level)
    b = r.flux(sub, compute="fp64", precision=0, max_level=check_level)
    err = max(_peak_err(x, y) for x, y in zip(a, b))
    mixed_e2e = samples / wall / 1e9
    fp64_e2e = sm64 / w64 / 1e9
    fp64_dev = sm64 / (ms64 * 1e-3) / 1e9
    mixed_dev = samples / (dev_ms * 1e-3) / 1e9
    cr = uneven_cpu_reference(jobs)
    cpu = None if cr is None else {
        "value": cr[1] / cr[0] / 1e9, "unit": "Gsamples/s", "cores": cr[3], "kind": "reference",
        "sample": "first %d jobs with >= 2 x 2 observers, one energy each (the middle one), %.1f s" % (cr[2], cr[0])}
    return {"workload": UNEVEN_WORKLOAD, "steps": steps, "warmup": warmup,
            "value": samples / (dev_ms * 1e-3) / 1e9, "unit": "Gsamples/s", "ms_per_step": dev_ms / steps,
            "samples_per_step": samples // steps, "gpu_launches_per_step": launches // steps, "variant": variant,
            "e2e": {"value": mixed_e2e, "unit": "Gsamples/s", "wall_s_per_step": wall / steps,
                    "path": "oscars_b200.batch.BatchRunner.flux(jobs, compute='mixed')"},
            "fp64": {"value": fp64_dev, "e2e": fp64_e2e, "unit": "Gsamples/s", "jobs": len(jobs),
                     "path": "BatchRunner.flux(jobs, compute='fp64') (jobs one after another, host RK4); value = "
                             "device time of its sample-sum kernels (the mixed value counts the whole batch, device "
                             "trajectories included)"},
            "mixed_over_fp64": mixed_dev / fp64_dev, "mixed_over_fp64_e2e": mixed_e2e / fp64_e2e,
            "mixed_vs_fp64_peak_rel_err": {"value": err, "jobs": fp64_jobs, "fixed_level": check_level,
                                           "norm": "per job, max over jobs"},
            "cpu_reference": cpu, "clocks": clk.summary()}


def sharded_beam_leg(steps, warmup, local, rank, world):
    """The EPU beam split over the ranks (torchrun): every rank draws the same 10k particles,
    integrates particles rank, rank + W, ... (shard option, weight 1/N) and one NCCL all_reduce sums
    the 101 x 101 partial fluxes.  Device time per rank (profiled chunks + the all_reduce on the
    current stream), max over ranks; samples summed over ranks."""
    import ctypes
    import torch
    import torch.distributed as dist
    from oscars_b200.shard import allreduce_sum
    from oscars_b200.sr import sr
    s = sr(gpu=1, device=local)
    setup_epu_beam(s)
    s._ctx.call("osc_set_beam_batch_threshold", 1)  # each rank's share runs batched
    kw = dict(energy_eV=E1_EPU, npoints=[101, 101], width=[0.008, 0.008], translation=[0, 0, 30], return_numpy=True,
              nparticles=BEAM_PARTICLES, compute="mixed", shard=(rank, world))

    def run():
        s.set_seed(1)
        return allreduce_sum(s.calculate_flux_rectangle(**kw)[1])
    for _ in range(warmup):
        run()
    dev_ms = 0.0
    samples = 0
    stream = torch.cuda.current_stream()
    dist.barrier()
    torch.cuda.synchronize()
    for _ in range(steps):
        _, ms, sm, _, _ = _profiled(s._ctx, lambda: s.calculate_flux_rectangle(**kw))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        part = torch.zeros(101 * 101, dtype=torch.float64, device="cuda")
        a.record(stream)
        dist.all_reduce(part)
        b.record(stream)
        torch.cuda.synchronize()
        dev_ms += ms + a.elapsed_time(b)
        samples += sm
    t = torch.tensor([dev_ms, float(samples)], dtype=torch.float64, device="cuda")
    tmax, tsum = t.clone(), t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return {"workload": BEAM_WORKLOAD + "; particles round-robin over %d ranks, one NCCL all_reduce" % world,
            "steps": steps, "warmup": warmup, "value": float(tsum[1]) / (float(tmax[0]) * 1e-3) / 1e9,
            "unit": "Gsamples/s", "ms_per_step": float(tmax[0]) / steps, "scaling": "strong",
            "timing": "device time per rank (batch chunks + all_reduce), max over ranks"}


# ---------------------------------------------------------------------------------------------
# Differentiable field tuning: gradient of a flux loss with respect to 82 half-period amplitudes
# ---------------------------------------------------------------------------------------------
TUNING_WORKLOAD = ("41-period undulator B0=0.5T lambda=50mm with 82 half-period factors 1+delta, delta~N(0,0.005) "
                   "(seed 82); 3 GeV; 20001-point RK4; loss=sum (F-F_ideal)^2 over 21x21 observers (2mm x 2mm at "
                   "z=30m) x 256 energies over E1 +-5%; fixed level 12; radiation sums and their adjoint in mixed "
                   "precision (FP64 phase, FP32 amplitudes and reverse sweep), RK4 adjoint in FP64 from checkpoints "
                   "every 256 steps")


def tuning_leg(steps, warmup, local=0, check_params=(3, 20, 41, 70)):
    """One step = the forward flux and its adjoint gradient (osc_flux_vjp forward pass, then the
    backward pass reusing its sums); grad/s with compute='mixed' (the value) and 'fp64'; Richardson
    central differences (h = 1e-3, 3e-3) on a few factors as a check of the mixed gradient."""
    import numpy as np
    from oscars_b200.tuning import TuningProblem
    xs = np.linspace(-0.001, 0.001, 21)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    obs = np.stack([X.ravel(), Y.ravel(), np.full(X.size, 30.0)], 1)
    energies = np.linspace(0.95 * E1, 1.05 * E1, 256)
    s = 1 + np.random.default_rng(82).normal(0.0, 0.005, 82)

    def run(compute):
        p = TuningProblem(bfield=[0, 0.5, 0], period=[0, 0, 0.05], nperiods=41, obs=obs, energies_eV=energies,
                          level=12, gpu=local, compute=compute)
        F_ideal = p.flux(np.ones(82))
        for _ in range(warmup):
            p.vjp(s, 2 * (p.flux(s) - F_ideal))
            p.flux(np.ones(82))  # new factors: the next step recomputes the trajectory and the sums
        t_fwd = t_all = 0.0
        g = None
        with ClockSampler(local) as clk:
            for k in range(steps):
                sk = s if k % 2 == 0 else s * (1 + 1e-12)  # alternate factors: nothing carries over a step
                t0 = time.perf_counter()
                F = p.flux(sk)
                t1 = time.perf_counter()
                gk = p.vjp(sk, 2 * (F - F_ideal))[1]
                t2 = time.perf_counter()
                if k % 2 == 0:
                    g = gk
                t_fwd += t1 - t0
                t_all += t2 - t0
        return p, F_ideal, g, {"value": steps / t_all, "unit": "grad/s", "ms_per_step": 1e3 * t_all / steps,
                               "forward_ms": 1e3 * t_fwd / steps, "adjoint_ms": 1e3 * (t_all - t_fwd) / steps,
                               "clocks": clk.summary()}
    p, F_ideal, g, mx = run("mixed")
    _, _, g64, f64 = run("fp64")
    loss = lambda v: float(np.sum((p.flux(v) - F_ideal) ** 2))

    def central(k, h):
        e = np.zeros(82)
        e[k] = h
        return (loss(s + e) - loss(s - e)) / (2 * h)
    fd = np.array([(9 * central(k, 1e-3) - central(k, 3e-3)) / 8 for k in check_params])
    err = float(np.max(np.abs(g[list(check_params)] - fd)) / np.max(np.abs(fd)))
    tr = tuning_cpu_reference()
    cpu = None if tr is None else {
        "value": 1.0 / (tr[0] * tr[1]), "unit": "grad/s", "cores": tr[2], "kind": "reference",
        "sample": "one central-difference component on 16 of the 256 energies, %.1f s; the full gradient by "
                  "central differences is %d such subsets (82 components x 16), so %.0f s per gradient (derived)"
                  % (tr[0], tr[1], tr[0] * tr[1])}
    out = {"workload": TUNING_WORKLOAD, "steps": steps, "warmup": warmup}
    out.update(mx)
    out.update({"grad_vs_richardson_fd": {"value": err, "params": list(check_params), "steps": [1e-3, 3e-3]},
                "mixed_vs_fp64_grad_rel": float(np.max(np.abs(g - g64)) / np.max(np.abs(g64))),
                "fp64": f64,
                "path": "oscars_b200.tuning.TuningProblem(compute='mixed').flux + vjp (osc_flux_vjp forward, then "
                        "backward on the kept sums); wall clock, host buffers; a new trajectory every step",
                "cpu_reference": cpu})
    return out


def _free_port():
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--compute", default="mixed", choices=["fp64", "mixed"],
                    help="headline arithmetic; 'mixed' also times the FP64 path and reports both")
    ap.add_argument("--quick", action="store_true", help="device-resident timing only (for profiler runs)")
    ap.add_argument("--variant", type=int, default=-1,
                    help="force this compiled variant of the --compute kernel instead of autotuning (profiler runs)")
    ap.add_argument("--batched-steps", type=int, default=3,
                    help="timed steps of the batched workloads (EPU beam, uneven jobs); 0 skips them")
    ap.add_argument("--only", default="", choices=["", "beam", "uneven", "tuning", "sharded", "power_density"],
                    help="run one workload alone and print its JSON object (for profiler runs)")
    ap.add_argument("--particles", type=int, default=BEAM_PARTICLES,
                    help="with --only beam: particles of the beam (the first ones of the same seeded sequence)")
    ap.add_argument("--jobs", type=int, default=UNEVEN_JOBS,
                    help="with --only uneven: the first jobs of the same seeded sequence")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    elif args.only == "sharded":  # the split beam on the ranks of torchrun (or a 1-rank group)
        import torch
        import torch.distributed as dist
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        if world > 1:
            dist.init_process_group("nccl")
        else:
            dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0, world_size=1)
        r = sharded_beam_leg(args.batched_steps, args.warmup, local, rank, world)
        if rank == 0:
            print(json.dumps(r), flush=True)
        dist.destroy_process_group()
    elif args.only:
        import torch
        torch.cuda.set_device(0)
        if args.only == "power_density":
            r = power_density_only(args.steps, args.warmup)
        elif args.only == "beam":
            r = beam_leg(args.batched_steps, args.warmup, particles=args.particles, quick=args.quick)
        elif args.only == "uneven":
            r = uneven_leg(args.batched_steps, args.warmup, n_jobs=args.jobs, quick=args.quick)
        else:
            r = tuning_leg(args.batched_steps, args.warmup)
        print(json.dumps(r), flush=True)
    else:
        product_arm(args)


if __name__ == "__main__":
    main()
