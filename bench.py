"""Benchmark of the B200 line-by-line core on the Venus-like PT-table workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one step): the 40-level Venus-like CO2 PT-table set -- 200,000
seeded synthetic lines over 4000-5000 cm-1, P log-spaced 92 -> 1e-4 atm,
T 735 -> 170 K, 96.5% CO2 by the ideal-gas law, cutoff 125 cm-1, tonkov
chi-factor, VAC target: 40 levels x 100 subintervals x 20,481 points.
Metric: line-grid evaluations per second (one evaluation = one line-shape
call of the reference's multigrid schedule, counted exactly by the library),
for the FP32-compensated form; the FP64 drop-in, the FP32c/FP64 ratio and the
FP32c error against the FP64 result are reported beside it.

Under torchrun every rank computes its own copy of the PT-table set (levels
are independent; no collective on the data path): weak scaling, the value is
the evaluations of all ranks over the slowest rank's time.

--impl reference times the CPU restatement of the reference's own algorithm
(oracle/, Fortran type map, all host threads) on a bounded sample of the same
workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "line-grid evals/s & s per 40-level PT set: FP32c vs FP64 GPU at <=1e-5 rel err"
UNIT = "line-grid evals/s"
WORKLOAD = "venus-co2-200k-lines-40-levels-4000-5000cm-1-cutoff125-tonkov-VAC"
FLOP_PER_EVAL = 12  # chi-corrected Lorentz evaluation + accumulation, FMA = 2
# cascade kernel: FP32 accumulators read (10,230 cells x 3) + one record written
CASCADE_BYTES_PER_RECORD = 10230 * 3 * 4 + 20481 * 4
# fine kernel DRAM traffic per unit (one level x subinterval), from one ncu
# capture of the two-level Venus case scaled by its units
FINE_TRAFFIC_PER_UNIT = 259_657  # (31,573,248 + 20,358,144) B / 200 units
# fine kernel warp instructions per unit, from the same capture: the kernel
# is issue-bound, so its issue rate is the roofline that describes it
FINE_WARP_INST_PER_UNIT = 755_935  # 151,187,000 warp instructions / 200 units
FINE_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one fine_kernel launch "
                       "on levels 1 and 21 (200 units), scaled by units: "
                       "profiles/fine_kernel_fp32c_venus_2levels.md")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", type=int, default=1, choices=[1, 2, 3, 4],
                    help="1: the Venus PT-table set (the headline, with the other configurations "
                         "measured after it); 2: the uneven batch of 64 profiles through one "
                         "autotuned, graph-captured launch sequence; 3: the adjoint; 4: the stress set")
    ap.add_argument("--scale", type=float, default=1.0, help="config 2 only: fraction of its size")
    ap.add_argument("--levels", default="",
                    help="config 1: comma-separated subset of the 40 levels (small profiling cases; "
                         "no other configurations)")
    ap.add_argument("--no-extra", action="store_true",
                    help="config 1: skip the measurement of configurations 2, 3 and 4")
    return ap.parse_args()


def workload():
    from marfa_b200 import synth
    return synth.config(1)


def tips_table():
    from marfa_b200 import data_path
    from marfa_b200.io import read_tips
    return read_tips(data_path("TIPS_subset.dat"))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- CPU legs
def cpu_baseline_sample(w, tips, levels, nthreads):
    """Oracle (Fortran type map) on `levels` of the workload; returns
    (evals, seconds)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    from marfa_b200.io import species_code
    p = w.profiles[0]
    o = O.Oracle(w.lines, tips, p.pressure[levels], p.temperature[levels], p.density[levels],
                 w.start_wv, w.end_wv, w.cutoff, target=w.target, chi=w.chi,
                 mol_code=species_code(w.molecule), precision=O.MIXED, nthreads=nthreads)
    t0 = time.perf_counter()
    _, _, ev = o.run(want64=False)
    dt = time.perf_counter() - t0
    return int(ev.sum()), dt


def run_reference(args, rank):
    if rank != 0:
        return
    w = workload()
    tips = tips_table()
    cores = os.cpu_count() or 1
    # each step: one level per host thread (bounded sample of the 40 levels)
    n = max(1, min(cores, 40))
    levels = list(np.linspace(0, 39, n).round().astype(int))
    if args.warmup > 0:  # one level, to page in the oracle and the line list
        cpu_baseline_sample(w, tips, levels[:1], 1)
    tot_ev, tot_t = 0, 0.0
    for _ in range(args.steps):
        ev, dt = cpu_baseline_sample(w, tips, levels, cores)
        tot_ev += ev
        tot_t += dt
    v = tot_ev / tot_t
    sample = f"{n} of 40 levels x 100 subintervals per step, {cores} threads, CPU restatement (Fortran type map)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 mixed",
        "data": "synthetic", "config": {"workload": WORKLOAD, "sample_levels": n},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# --------------------------------------------------------------- GPU leg
def hbm_peak():
    """Measured HBM copy bandwidth (GB/s) of this pool's B200s and where it came from."""
    f = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(f.read_text())["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback (earlier measurement on this pool)"


def timed_steps(ctx, run, counts, P, T, n, out, stream, steps, warmup):
    import torch
    for _ in range(warmup):
        ctx.compute_device(run, counts, P, T, n, out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ctx.compute_device(run, counts, P, T, n, out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    tm = ctx.timings()
    return ms, tm, int(tm["launches"]) * steps


def error_stats(out32, out64):
    """Max and 99.99th-percentile relative error of the FP32c records
    against the FP64 records over points with k > 1e-6 max(k), level by
    level (bounded device memory)."""
    import torch
    kmax = float(out64.max())
    mx, sample = 0.0, []
    for l in range(out64.shape[0]):
        a = out32[l].double()
        b = out64[l].double()
        m = b > 1e-6 * kmax
        rel = (a - b).abs()[m] / b[m]
        if rel.numel():
            mx = max(mx, float(rel.max()))
            sample.append(rel[:: max(1, rel.numel() // 100_000)])
    rel = torch.cat(sample) if sample else torch.zeros(1, dtype=torch.float64, device=out64.device)
    return mx, float(torch.quantile(rel, 0.9999))


def run_b200(args, rank, world, local_rank):
    import torch
    from marfa_b200 import build as B
    from marfa_b200.api import Context, Run
    B.build()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    w = workload()
    tips = tips_table()
    p = w.profiles[0]
    lv = slice(None) if not args.levels else [int(x) for x in args.levels.split(",")]
    P, T, n = (np.asarray(getattr(p, f), dtype=np.float64)[lv] for f in ("pressure", "temperature", "density"))
    L = len(P)
    ctx = Context(w.lines, tips, device=local_rank)
    run32 = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
                precision="fp32c")
    run64 = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
                precision="fp64")
    ev, evf = ctx.eval_count(run32, P, T, n, far=True)
    evals = int(ev.sum())
    far_evals = int(evf.sum())
    out32 = torch.empty((L, run32.n_sub, 20481), dtype=torch.float32, device="cuda")
    out64 = torch.empty_like(out32)
    stream = torch.cuda.Stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # FP32-compensated form (the headline), clocks sampled during the timed region
    barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ms32, tm32, launches = timed_steps(ctx, run32, [L], P, T, n, out32, stream, args.steps, args.warmup)
    clk = clocks.stop()
    barrier()
    # FP64 drop-in
    ms64, tm64, _ = timed_steps(ctx, run64, [L], P, T, n, out64, stream, args.steps, args.warmup)
    barrier()
    from marfa_b200.multi import reduce_step
    ms_max, total_evals = reduce_step(ms32, evals, dist)  # slowest rank, work of all ranks
    ms64, _ = reduce_step(ms64, evals, dist)
    value = total_evals / (ms_max * 1e-3)
    value64 = total_evals / (ms64 * 1e-3)
    max_rel, p9999 = error_stats(out32, out64)

    # end to end: host profile in, host (pinned) records out, through the C ABI
    host_out = torch.empty((L, run32.n_sub, 20481), dtype=torch.float32, pin_memory=True)
    ctx.compute(run32, P, T, n, out=host_out)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(3, args.steps)
    for _ in range(e2e_steps):
        ctx.compute(run32, P, T, n, out=host_out)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_ms, _ = reduce_step(e2e_s * 1e3, evals, dist)
    e2e_s = e2e_ms * 1e-3
    h2d = 3 * L * 8
    d2h = host_out.numel() * 4

    # roofline of the dominant kernel (measured FMA peak of this GPU: the
    # shape kernels run on the non-tensor FP32 pipe) and the cascade's HBM
    # fraction
    fp32_peak = np.zeros(1)
    fp64_peak = np.zeros(1)
    probe = ctypes.CDLL(str(B.PROBE))
    probe.marfa_probe_fma_peak.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    if probe.marfa_probe_fma_peak(local_rank, fp32_peak.ctypes.data, fp64_peak.ctypes.data):
        raise RuntimeError("FMA throughput probe failed")
    fams = {k: tm32[k] for k in ("prep", "sort", "far", "fine", "cascade")}
    dom = max(fams, key=fams.get)
    fam_evals = {"far": far_evals, "fine": evals - far_evals}
    roof = None
    if dom in fam_evals:
        achieved = FLOP_PER_EVAL * fam_evals[dom] / (tm32[dom] * 1e-3) / 1e12
        peak = fp32_peak[0] / 1e12
        roof = {"kernel": f"{dom}_kernel (fp32c)", "bound": "fp32", "achieved": achieved,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": "FFMA throughput measured by bench.py on this GPU",
                "traffic": (FINE_TRAFFIC_PER_UNIT * L * run32.n_sub
                            if dom == "fine" and FINE_TRAFFIC_PER_UNIT else None),
                "traffic_source": FINE_TRAFFIC_SOURCE if dom == "fine" else None}
    far_roof = FLOP_PER_EVAL * far_evals / (tm32["far"] * 1e-3) / 1e12
    # issue roofline of the fine kernel: warp instructions per second against
    # one instruction per scheduler per clock (4 per SM) at the sampled clock
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    sm_mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    issue_peak = sms * 4 * sm_mhz * 1e6
    issue = FINE_WARP_INST_PER_UNIT * L * run32.n_sub / (tm32["fine"] * 1e-3)
    fine_issue = {"kernel": "fine_kernel (fp32c)", "achieved": issue / 1e12, "peak": issue_peak / 1e12,
                  "unit": "T warp-instructions/s", "frac": issue / issue_peak,
                  "peak_source": f"{sms} SMs x 4 schedulers x {sm_mhz:.0f} MHz (sampled)",
                  "inst_source": "ncu smsp__inst_executed.sum of the capture in "
                                 "profiles/fine_kernel_fp32c_venus_2levels.md, per unit"}
    hbm, hbm_src = hbm_peak()
    records = L * run32.n_sub
    cascade_gbs = records * CASCADE_BYTES_PER_RECORD / (tm32["cascade"] * 1e-3) / 1e9
    ctx.close()
    del out32, out64, host_out
    torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        levels = [0, 13, 26, 39]
        cev, cdt = cpu_baseline_sample(w, tips, levels, 1)
        cpu = {"value": cev / cdt, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "levels 1, 14, 27, 40 of 40 x 100 subintervals, 1 thread, CPU "
                         "restatement of the reference (Fortran type map), "
                         f"{cev} evaluations in {cdt:.1f} s"}

    # the other configurations of the plan, measured in the same run
    extra = None
    if rank == 0 and world == 1 and not args.no_extra and not args.levels:
        extra = {"uneven_batch": run_uneven(args, local_rank, steps=3, warmup=1),
                 "differentiation": run_adjoint(local_rank),
                 "stress": run_stress(local_rank)}

    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32 (compensated) + fp64 offsets",
            "data": "synthetic",
            "config": {"workload": WORKLOAD if not args.levels else f"{WORKLOAD} (levels {args.levels})",
                       "lines": int(len(w.lines) - 1), "levels": L,
                       "subintervals": run32.n_sub, "cutoff_cm-1": w.cutoff, "chi": w.chi,
                       "target": w.target, "l2": "inputs larger than L2 (576 MB line state, "
                       "328 MB records per step)", "parallelism": f"replicas x{world}"},
            "s_per_pt_set": ms_max * 1e-3,
            "evals_per_step": evals,
            "fp64_value": value64, "fp64_ms_per_step": ms64,
            "fp32c_over_fp64": ms64 / ms_max,
            "max_rel_err_fp32c_vs_fp64": max_rel, "p9999_rel_err_fp32c_vs_fp64": p9999,
            "kernel_ms": {k: round(v, 4) for k, v in fams.items()},
            "kernel_ms_fp64": {k: round(tm64[k], 4) for k in fams},
            "roofline": roof,
            "far_kernel_tflops": far_roof,
            "fine_issue_roofline": fine_issue,
            "fma_peak_tflops": {"fp32": fp32_peak[0] / 1e12, "fp64": fp64_peak[0] / 1e12},
            "cascade_hbm": {"achieved_gbs": cascade_gbs, "peak_gbs": hbm, "frac": cascade_gbs / hbm,
                            "peak_source": hbm_src,
                            "bytes_per_record": CASCADE_BYTES_PER_RECORD},
            "cpu_baseline": cpu,
            "e2e": {"value": total_evals / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clk,
            "configs": extra,
        }))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_uneven(args, local_rank, steps, warmup):
    """The uneven batch: 64 synthetic profiles of 10-100 levels (P log-uniform
    1e-4..100 atm, T uniform 150-750 K) over an H2O-like list of 30,000 lines,
    10-3000 cm-1, cutoff 25 cm-1, FP32c.  The launch parameters are autotuned
    on the first profile, the computation of all profiles is captured once in
    a CUDA graph, and every timed step replays it (restaging the profile
    tables).  The records stay on the device (92 GB at full size)."""
    import torch
    from marfa_b200 import build as B, synth
    from marfa_b200.api import Context, Run
    B.build()
    torch.cuda.set_device(local_rank)
    w = synth.config(2, args.scale)
    counts = [len(p.pressure) for p in w.profiles]
    cat = lambda f: np.concatenate([np.asarray(getattr(p, f), dtype=np.float64) for p in w.profiles])
    P, T, n = cat("pressure"), cat("temperature"), cat("density")
    L = sum(counts)
    ctx = Context(w.lines, tips_table(), device=local_rank)
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
              precision="fp32c")
    evals = int(ctx.eval_count(run, P, T, n).sum())
    p0 = w.profiles[0]
    tune = ctx.autotune(run, p0.pressure, p0.temperature, p0.density)
    out = torch.empty((L, run.n_sub, 20481), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    g = ctx.graph(run, counts, P, T, n, out.data_ptr())
    for _ in range(warmup):
        g.launch(P, T, n, stream.cuda_stream)
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        g.launch(P, T, n, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / steps
    ctx.synchronize()
    tm = ctx.timings()
    g.close()
    ctx.close()
    rec_bytes = int(out.numel() * 4)
    del out
    torch.cuda.empty_cache()
    return {
        "metric": "line-grid evals/s (uneven batch, FP32c, graph replay)", "value": evals / (ms * 1e-3),
        "unit": UNIT, "steps": steps, "warmup": warmup, "ms_per_step": ms,
        "workload": "uneven-64-profiles-h2o-30k-lines-10-3000cm-1-cutoff25", "scale": args.scale,
        "profiles": len(counts), "levels": L, "subintervals": run.n_sub,
        "lines": int(len(w.lines) - 1), "record_bytes_on_device": rec_bytes,
        "evals_per_step": evals, "autotuned": tune, "graph_launches_per_step": 1,
        "gpu_launches_per_step": int(tm["launches"]), "clocks": clk,
    }


def run_adjoint(local_rank, calls=3):
    """The differentiation workload: 40,000 lines over 4000-4200 cm-1, 10
    Venus levels, ACS; the vector-Jacobian product of the FP64 records for a
    Gaussian cotangent (seed 3) with respect to level T, P and per-line S,
    gamma_air, through the C ABI (host cotangent in, host gradients out)."""
    import torch
    from marfa_b200 import synth
    from marfa_b200.api import Context, Run
    w = synth.config(3)
    p = w.profiles[0]
    ctx = Context(w.lines, tips_table(), device=local_rank)
    run = Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule, chi=w.chi,
              precision="fp64")
    L = len(p.pressure)
    cot = np.random.default_rng(3).standard_normal((L, run.n_sub, 20481))
    ctx.vjp(run, p.pressure, p.temperature, p.density, cot)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(calls):
        ctx.vjp(run, p.pressure, p.temperature, p.density, cot)
    vjp_ms = (time.perf_counter() - t0) / calls * 1e3
    out = torch.empty((L, run.n_sub, 20481), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    fwd_ms, _, _ = timed_steps(ctx, run, [L], p.pressure, p.temperature, p.density, out, stream, 3, 1)
    ctx.close()
    return {"workload": "diff-40k-lines-10-levels-4000-4200cm-1-tonkov-ACS", "levels": L,
            "subintervals": run.n_sub, "vjp_ms_per_call": vjp_ms, "calls": calls,
            "fp64_forward_ms": fwd_ms,
            "vjp": "dL/dT, dL/dP per level and dL/dS, dL/dgamma_air per line, host cotangent "
                   f"({cot.nbytes} B) in, host gradients out"}


def run_stress(local_rank, steps=2):
    """The stress workload: 2,000,000 lines over 500-10000 cm-1 (S
    log-uniform 1e-30..1e-19), 100 levels of the Venus profile shape, cutoff
    250 cm-1, tonkov, VAC; FP32c against the FP64 drop-in on the device."""
    import torch
    from marfa_b200 import synth
    from marfa_b200.api import Context, Run
    w = synth.config(4)
    p = w.profiles[0]
    ctx = Context(w.lines, tips_table(), device=local_rank)
    mk = lambda prec: Run(w.start_wv, w.end_wv, w.cutoff, target=w.target, molecule=w.molecule,
                          chi=w.chi, precision=prec)
    run32, run64 = mk("fp32c"), mk("fp64")
    L = len(p.pressure)
    evals = int(ctx.eval_count(run32, p.pressure, p.temperature, p.density).sum())
    out32 = torch.empty((L, run32.n_sub, 20481), dtype=torch.float32, device="cuda")
    out64 = torch.empty_like(out32)
    stream = torch.cuda.Stream()
    ms32, tm32, _ = timed_steps(ctx, run32, [L], p.pressure, p.temperature, p.density, out32, stream, steps, 1)
    ms64, _, _ = timed_steps(ctx, run64, [L], p.pressure, p.temperature, p.density, out64, stream, 1, 1)
    mx, p9999 = error_stats(out32, out64)
    ctx.close()
    del out32, out64
    torch.cuda.empty_cache()
    return {"workload": "stress-2M-lines-100-levels-500-10000cm-1-cutoff250-tonkov-VAC", "levels": L,
            "subintervals": run32.n_sub, "evals_per_step": evals, "ms_per_step": ms32,
            "value": evals / (ms32 * 1e-3), "unit": UNIT, "fp64_ms_per_step": ms64,
            "fp32c_over_fp64": ms64 / ms32, "max_rel_err_fp32c_vs_fp64": mx,
            "p9999_rel_err_fp32c_vs_fp64": p9999,
            "kernel_ms": {k: round(tm32[k], 3) for k in ("prep", "sort", "far", "fine", "cascade")}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
    elif args.config == 2:
        if rank == 0:
            print(json.dumps(run_uneven(args, local_rank, args.steps, args.warmup)))
    elif args.config == 3:
        if rank == 0:
            print(json.dumps(run_adjoint(local_rank, max(1, args.steps))))
    elif args.config == 4:
        if rank == 0:
            print(json.dumps(run_stress(local_rank, max(1, args.steps))))
    else:
        run_b200(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
