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
``e2e``    the same job through the C ABI with host buffers: host RK4 + spline, host->device
           copies, kernels, device->host copy of the results, every step.
Under torchrun each rank runs its own job (energy E1 * (1 + 1e-3 rank)): no collective on the data
path, weak scaling; the reported time is the max over ranks.

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


def reference_arm(args):
    """The reference's own CPU implementation on all host cores (rank 0 only), same workload and
    metric; each step is the largest set of central grid rows that keeps the run to ~20 s."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    kind, cores, o = _cpu_impl()
    setup(o)
    o.calculate_trajectory()
    dt, _ = _cpu_flux_rows(o, kind, cores, 5)
    rows = int(max(5, min(GRID, (20.0 / max(1, args.steps)) / max(dt / 5, 1e-6))))
    rows -= (rows + 1) % 2  # odd: the row set stays centred on the axis
    times, samples = [], 0.0
    for _ in range(args.steps):
        dt, s = _cpu_flux_rows(o, kind, cores, rows)
        times.append(dt)
        samples += s
    total = sum(times)
    value = samples / total / 1e9
    desc = "central %d of 201 rows x 201 columns per step, %d steps, %d threads" % (rows, args.steps, cores)
    line = {"metric": METRIC, "value": value, "unit": "Gsamples/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": desc}, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "Gsamples/s", "cores": cores, "kind": kind, "sample": desc},
            "e2e": {"value": value, "unit": "Gsamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_leg():
    """The reference CPU path on all host cores, bounded to ~10-20 s of work."""
    kind, cores, o = _cpu_impl()
    setup(o)
    o.calculate_trajectory()
    dt, _ = _cpu_flux_rows(o, kind, cores, 5)
    rows = int(max(5, min(GRID, 15.0 / max(dt / 5, 1e-6))))
    rows -= (rows + 1) % 2
    dt, samples = _cpu_flux_rows(o, kind, cores, rows)
    return {"value": samples / dt / 1e9, "unit": "Gsamples/s", "cores": cores, "kind": kind,
            "sample": "central %d of 201 rows x 201 columns, one pass, %.2f s" % (rows, dt)}


def _time_device_steps(ctx, step, stream, flush, steps, warmup, local):
    """Per-step CUDA events on the launching stream, L2 flushed before every step (outside the
    events).  Returns (total ms, samples per step, launches per step, wave-kernel ms, clocks)."""
    import ctypes
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    sm, ln = ctypes.c_longlong(), ctypes.c_longlong()
    ctx.call("osc_last_stats", ctypes.byref(sm), ctypes.byref(ln))  # the job is identical every step
    ctx.call("osc_set_profiling", 1)
    ctx.call("osc_get_profile", None, None, None, 1)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with ClockSampler(local) as clk:
        time.sleep(0.1)
        for i in range(steps):
            flush.zero_()
            evs[i][0].record(stream)
            step()
            evs[i][1].record(stream)
        torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    kms, kl = ctypes.c_double(), ctypes.c_longlong()
    ctx.call("osc_get_profile", ctypes.byref(kms), ctypes.byref(kl), None, 1)
    ctx.call("osc_set_profiling", 0)
    return ms, sm.value, ln.value, kms.value, kl.value, clk.summary()


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
    stream = torch.cuda.current_stream(dev)
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
        ms, sps, lps, kms, kl, clocks = _time_device_steps(ctx, make_step(m), stream, flush, args.steps, args.warmup, local)
        t = torch.tensor([ms, float(sps * args.steps)], dtype=torch.float64, device=dev)
        if world > 1:
            tmax, tsum = t.clone(), t.clone()
            dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
            dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
            ms_max, samples_all = float(tmax[0]), float(tsum[1])
        else:
            ms_max, samples_all = ms, float(sps * args.steps)
        v, nv = ctypes.c_int(), ctypes.c_int()
        ctx.call("osc_get_variant", 2 if m == "mixed" else 0, ctypes.byref(v), ctypes.byref(nv))
        peak = ctypes.c_double()
        ctx.call("osc_measure_fma_peak", 0 if m == "fp64" else 1, ctypes.byref(peak))
        achieved = sps * args.steps * FLOP_PER_SAMPLE / (kms * 1e-3) / 1e12 if kms > 0 else None
        traffic = None
        prof_path = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(prof_path):
            traffic = json.load(open(prof_path)).get("k_fd_wave_%s" % m)
        res[m] = {"value": samples_all / (ms_max * 1e-3) / 1e9, "ms_per_step": ms_max / args.steps,
                  "samples_per_step": sps, "launches_per_step": lps, "variant": v.value, "clocks": clocks,
                  "roofline": {"bound": "fp64" if m == "fp64" else "fp32", "achieved": achieved, "peak": peak.value,
                               "unit": "TFLOP/s", "frac": (achieved / peak.value) if achieved else None,
                               "traffic": traffic, "kernel": "k_fd_wave_%s" % m, "flop_per_sample": FLOP_PER_SAMPLE,
                               "kernel_ms_per_step": kms / args.steps, "kernel_launches_per_step": kl / args.steps,
                               "peak_source": "in-run FMA-throughput loop on this GPU (osc_measure_fma_peak); the "
                                              "sample sums run on the %s pipe, not the tensor cores or HBM"
                                              % ("FP64" if m == "fp64" else "FP32/SFU")}}
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

    # e2e: host buffers through the C ABI, new trajectory every step (host RK4 + spline included)
    out_h = np.zeros(n)
    lvl_h = np.zeros(n, dtype=np.int32)
    nnc = ctypes.c_longlong()

    def e2e_step():
        s.set_new_particle(particle="ideal")  # drops the trajectory: RK4 + spline + upload again
        ctx.call("osc_flux", _lib.dptr(xyz), n, energy, ctypes.byref(opts[head]), _lib.dptr(out_h),
                 _lib.i32ptr(lvl_h), ctypes.byref(nnc))
    e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e2e_times, e2e_samples = [], 0
    for i in range(max(1, min(args.steps, 20))):
        t0 = time.perf_counter()
        e2e_step()
        e2e_times.append(time.perf_counter() - t0)
        sm = ctypes.c_longlong()
        ctx.call("osc_last_stats", ctypes.byref(sm), None)
        e2e_samples += sm.value
    te = torch.tensor([sum(e2e_times), float(e2e_samples)], dtype=torch.float64, device=dev)
    if world > 1:
        tm, ts = te.clone(), te.clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        dist.all_reduce(ts, op=dist.ReduceOp.SUM)
        e2e_value = float(ts[1]) / float(tm[0]) / 1e9
    else:
        e2e_value = e2e_samples / sum(e2e_times) / 1e9
    h2d = xyz.nbytes + 19 * 20001 * 8 + 8
    d2h = out_h.nbytes + lvl_h.nbytes
    if rank == 0:
        cpu = cpu_baseline_leg() if world == 1 else None
        r = res[head]
        line = {"metric": METRIC, "value": r["value"], "unit": "Gsamples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32+f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "compute": head, "l2": "flushed between steps (256 MB write)",
                           "parallelism": "independent job per rank" if world > 1 else "single GPU"},
                "e2e": {"value": e2e_value, "unit": "Gsamples/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": r["launches_per_step"] * args.steps, "roofline": r["roofline"], "cpu_baseline": cpu,
                "clocks": r["clocks"]}
        if "mixed" in res:
            f = res["fp64"]
            line["fp64"] = {"value": f["value"], "ms_per_step": f["ms_per_step"], "roofline": f["roofline"],
                            "clocks": f["clocks"]}
            line["mixed_over_fp64"] = r["value"] / f["value"]
            line["mixed_vs_fp64_peak_rel_err"] = err
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--compute", default="mixed", choices=["fp64", "mixed"],
                    help="headline arithmetic; 'mixed' also times the FP64 path and reports both")
    ap.add_argument("--quick", action="store_true", help="device-resident timing only (for profiler runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    else:
        product_arm(args)


if __name__ == "__main__":
    main()
