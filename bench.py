#!/usr/bin/env python
"""
Benchmark of the ALE tracer step on B200: advect_fct (SSP-RK3 WENO5-Z + Zalesak FCT) of a T/S stack followed by the
PPM_H4 remap of both fields, on the 512 x 512 x 50 curvilinear basin (FP64, seeded synthetic data).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload basin|zstar_box]

Metric: tracer cell-steps/s = nt * N * ny * nx * steps / time.  One "step" is one advect_fct + remap of the whole
stack.  `value` is device-resident throughput (inputs already in HBM, CUDA events on the launching stream, max over
ranks); `e2e` is the same step through the reference's two drop-in calls (TracerAdvection.advect_fct,
remap_columns) with pinned host tensors, host<->device copies inside the timed region, and beside it (`one_call`)
the repository's ``ale_tracer_step``, which keeps the advected stack on the device.  The stack (210 MB) and every geometry array
(105 MB each) exceed the 126 MB L2, so no flush is needed between steps.

Multi-GPU: the path does not shard (one domain per GPU, "replicas only"); under torchrun every rank runs its own
replica and `value` sums the cell-steps of all ranks over the slowest rank's time.

`--impl reference` times the reference's CPU implementation (the C restatement in oracle/, OpenMP on every host
core; rank 0 only) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def ranks_from_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) of this process as torchrun sets them (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x: float, device) -> float:
    """The largest x over all ranks of the process group (the job's time is its slowest rank's); x itself without
    a group.  ``device``: where the reduction tensor lives (CUDA for NCCL, CPU for gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, ms: float) -> float:
    """Whole-job throughput of weak-scaled replicas: every rank's units over the slowest rank's time [units/s]."""
    return units_per_rank * world / (ms / 1e3)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="basin", choices=["basin", "zstar_box"])
    ap.add_argument("--basin-size", type=int, nargs=3, default=[512, 512, 50], metavar=("NX", "NY", "NZ"),
                    help="size of the basin workload (a smaller one for profiling captures)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--ref-seconds", type=float, default=150.0,
                    help="time budget of the timed steps of --impl reference (it stops early past it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batched-steps", type=int, default=50,
                    help="steps of the 64-uneven-domains batch report (0: skip)")
    ap.add_argument("--mixed-steps", type=int, default=100,
                    help="steps of the mixed-precision accuracy report at 1024x1024x75, 6 tracers (0: skip)")
    ap.add_argument("--serve-jobs", type=int, default=200, help="jobs of the served-stream report (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=15.0, help="Poisson arrival rate of the served stream [1/s]")
    ap.add_argument("--no-neighbours", action="store_true", help="skip the regrid / diffusion / velocity-remap timings")
    return ap.parse_args()


def make_workload(name: str, size=(512, 512, 50)):
    from pyocean_b200 import workloads as W
    return W.basin(nx=size[0], ny=size[1], n=size[2]) if name == "basin" else W.zstar_box()


def workload_config(w, world: int) -> dict:
    """The ``config`` of both arms' JSON lines: the workload, its shape and the step's schemes."""
    nt, n, ny, nx = w.C.shape
    return {"workload": w.name, "nt": nt, "nz": n, "ny": ny, "nx": nx,
            "remap": {0: "pcm", 1: "plm", 2: "ppm_h4"}[w.remap_scheme], "limiter": "fct",
            "weno": "z" if w.scheme == "weno5" else "js",
            "l2": (f"inputs larger than L2 ({w.C.nbytes / 1e6:.0f} MB stack, {w.V0.nbytes / 1e6:.0f} MB per geometry "
                   "array); no flush" if w.C.nbytes > 126e6 else "inputs smaller than L2; no flush"),
            "parallelism": f"replicas x{world}"}


# From one ncu capture of a step of this workload with the current kernels (the seven advect_fct kernels and the
# remap): DRAM bytes read + written per call, and FP64 thread instructions (DFMA + DMUL + DADD) per call.  The
# line carries the capture's date beside them (NCU_CAPTURED); a kernel change needs a new capture.
NCU_PER_CALL = {
    "basin_512x512x50_nt2": {"advect_fct": {"dram_bytes": 9515066880, "fp64_inst": 18348363343},
                             "remap_columns": {"dram_bytes": 793686784, "fp64_inst": 3091276864}},
}
NCU_CAPTURED = ("2026-12-04: DRAM bytes from a one-pass ncu capture (dram__bytes_read.sum, dram__bytes_write.sum) of "
                "one step of the basin 512x512x50 workload; FP64 instruction counts of advect_fct from the full-set "
                "capture of 2026-12-03 (same kernels), of the remap from a capture of its kernel on 2026-12-04")
FP64_LANES_PER_SM, SMS = 64, 148


def peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
    return dict(hbm_gbs=6650.0, source="fallback")


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ------------------------------------------------------------------------------------------------ CPU baseline
def cpu_sample(w, budget_s: float, max_steps: int = 5, warmup: int = 0) -> dict:
    """The reference algorithm on the host (oracle/ C restatement, OpenMP over every core): ``warmup`` untimed
    steps, then whole steps of the same workload until ``max_steps`` steps or ~budget_s seconds have passed (at
    least one), timed with perf_counter."""
    from oracle import oracle as O
    ncores = os.cpu_count() or 1
    O.set_threads(ncores)
    adv = O.TracerAdvection(scheme=w.scheme, time="ssprk3", dt=w.dt, ob=O.OpenEdges(w.open))
    adv.per = O.Periodic(w.periodic)

    def step(C):
        A = adv.advect_fct(C, w.V0, w.V1, w.Qx, w.Qy, w.ok)
        return np.stack([O.remap_columns(w.h_src, A[m], w.h_tgt, w.remap_scheme, w.wet) for m in range(A.shape[0])])

    C = w.C
    for _ in range(warmup):
        C = step(C)
    steps, t_total = 0, 0.0
    while True:
        t0 = time.perf_counter()
        C = step(C)
        t_total += time.perf_counter() - t0
        steps += 1
        if t_total >= budget_s or steps >= max_steps:
            break
    value = w.tracer_cells * steps / t_total
    return dict(value=value, unit="tracer cell-steps/s", cores=O.num_threads(), kind="port",
                sample=f"{steps} full step(s) of {w.name} (advect_fct + remap of every tracer), "
                       f"{t_total:.1f} s on {O.num_threads()} threads of {cpu_model()}",
                seconds=t_total, steps=steps)


# ------------------------------------------------------------------------------------------------ clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int) -> None:
        self.gpu = gpu_index
        self.proc = None

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["no samples"])
        return dict(sm_mhz=statistics.median(sm), sm_max_mhz=max(smax), reasons=sorted(reasons),
                    samples=len(sm), power_w_max=max(power) if power else None)


# ------------------------------------------------------------------------------------------------ GPU arm
def run_ours(args, rank: int, world: int, local_rank: int) -> dict | None:
    import torch

    from pyocean_b200 import _lib
    from pyocean_b200.remap import remap_columns
    from pyocean_b200.step import ALETracerStep, ale_tracer_step
    from pyocean_b200.tracers import OpenEdges, TracerAdvection
    from pyocean_b200.periodic import Periodic
    from pyocean_b200 import workloads as W

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = make_workload(args.workload, args.basin_size)
    nt, n, ny, nx = w.C.shape
    flags = (_lib.PERIODIC_X if "x" in w.periodic else 0) | (_lib.PERIODIC_Y if "y" in w.periodic else 0)
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                     # noqa: E731
    C0, V0, V1, Qx, Qy = g(w.C), g(w.V0), g(w.V1), g(w.Qx), g(w.Qy)
    ok = g(w.ok.view(np.uint8) if w.ok.dtype == np.bool_ else w.ok.astype(np.uint8))
    wet = g(w.wet.astype(np.uint8))
    hs, ht = g(w.h_src), g(w.h_tgt)
    stepper = ALETracerStep(nt, n, ny, nx, w.dt, flags, w.remap_scheme, device=dev)
    bufs = [C0.clone(), torch.empty_like(C0)]
    stream = torch.cuda.current_stream(dev)

    def one_step(i, ev=None):
        src, dst = bufs[i % 2], bufs[(i + 1) % 2]
        if ev is not None:
            ev[0].record(stream)
        a = stepper.advect(src, V0, V1, Qx, Qy, ok)
        if ev is not None:
            ev[1].record(stream)
        stepper.remap(hs, a, ht, wet, dst)
        if ev is not None:
            ev[2].record(stream)

    for i in range(args.warmup):
        one_step(i)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t_start.record(stream)
    for i in range(args.steps):
        one_step(args.warmup + i, evs[i])
    t_end.record(stream)
    torch.cuda.synchronize()
    ms = t_start.elapsed_time(t_end)
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    adv_ms = [e[0].elapsed_time(e[1]) for e in evs]
    rem_ms = [e[1].elapsed_time(e[2]) for e in evs]
    # finite, conserved result (a cheap guard against timing a broken kernel)
    res = bufs[(args.warmup + args.steps) % 2]
    assert bool(torch.isfinite(res[:, :, w.wet]).all()), "non-finite tracer values after the timed steps"

    ms = max_over_ranks(ms, dev)

    # ---- the mixed-precision form of the same step (FP32 WENO weights, FP64 limiter / bookkeeping / remap)
    mixed_stepper = ALETracerStep(nt, n, ny, nx, w.dt, flags, w.remap_scheme, device=dev, mixed=True)
    stepper = mixed_stepper
    for i in range(args.warmup):
        one_step(i)
    torch.cuda.synchronize()
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    mevs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    m0.record(stream)
    for i in range(args.steps):
        one_step(args.warmup + i, mevs[i])
    m1.record(stream)
    torch.cuda.synchronize()
    mixed_ms = m0.elapsed_time(m1)
    mixed_adv = float(np.mean([e[0].elapsed_time(e[1]) for e in mevs]))
    mixed_ms = max_over_ranks(mixed_ms, dev)
    del mixed_stepper

    # ---- end to end through the public API, pinned host tensors, copies inside the timed region
    adv = TracerAdvection(scheme=w.scheme, time="ssprk3", dt=w.dt, ob=OpenEdges(w.open))
    adv.per = Periodic(w.periodic)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()               # noqa: E731
    hC, hV0, hV1, hQx, hQy, hok = pin(w.C), pin(w.V0), pin(w.V1), pin(w.Qx), pin(w.Qy), pin(w.ok)
    hhs, hht, hwet = pin(w.h_src), pin(w.h_tgt), pin(w.wet)
    h2d = sum(int(t.numel() * t.element_size()) for t in (hC, hV0, hV1, hQx, hQy, hok, hhs, hht, hwet))
    d2h = int(hC.numel() * hC.element_size())
    stack = int(hC.numel() * hC.element_size())

    def timed(step, n):
        """Device time of n chained steps of `step` on the host arrays (after five untimed ones, which fill the
        device and pinned-host caching allocators with every block the chain holds at once: a new 210 MB pinned
        block costs ~100 ms)."""
        hc = hC
        for _ in range(5):
            hc = step(hc)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        hc = hC
        for _ in range(n):
            hc = step(hc)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    def copy_gbs(src, dst, reps=5):
        """Bandwidth of one plain stream-ordered copy of a pinned host block (either direction)."""
        dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(reps):
            dst.copy_(src, non_blocking=True)
        c1.record(stream)
        torch.cuda.synchronize()
        return reps * src.numel() * src.element_size() / (c0.elapsed_time(c1) / 1e3) / 1e9

    e2e_ms = e2e_two_ms = float("nan")
    h2d_gbs = d2h_gbs = float("nan")
    if args.e2e_steps > 0:
        blk = torch.empty_like(hV0, device=dev)
        h2d_gbs, d2h_gbs = copy_gbs(hV0, blk), copy_gbs(blk, hV0.clone().pin_memory())
        del blk
        # the step as one call (the advected stack stays on the device) ...
        e2e_ms = timed(lambda c: ale_tracer_step(adv, c, hV0, hV1, hQx, hQy, hok, hhs, hht, w.remap_scheme, hwet),
                       args.e2e_steps)
        # ... and as the reference's two drop-in calls (the advected stack goes back to the host between them)
        e2e_two_ms = timed(lambda c: remap_columns(hhs, adv.advect_fct(c, hV0, hV1, hQx, hQy, hok), hht,
                                                   w.remap_scheme, hwet), args.e2e_steps)
    e2e_ms = max_over_ranks(e2e_ms, dev)
    e2e_two_ms = max_over_ranks(e2e_two_ms, dev)

    cells = w.tracer_cells
    value = job_rate(cells * args.steps, world, ms)
    ab = W.algorithmic_bytes(w)
    pk = peaks()
    adv_avg, rem_avg = float(np.mean(adv_ms)), float(np.mean(rem_ms))
    adv_gbs = ab["advect"] / (adv_avg / 1e3) / 1e9
    rem_gbs = ab["remap"] / (rem_avg / 1e3) / 1e9
    dominant = ("advect_fct", adv_gbs, adv_avg, ab["advect"]) if adv_avg >= rem_avg else \
        ("remap_columns", rem_gbs, rem_avg, ab["remap"])
    ncu = NCU_PER_CALL.get(w.name, {})
    sm_hz = (clk.get("sm_mhz") or 1965.0) * 1e6
    fp64_rate = FP64_LANES_PER_SM * SMS * sm_hz                  # FP64 thread instructions per second at this clock

    def fp64_part(name, ms):
        if name not in ncu:
            return None
        t_min = ncu[name]["fp64_inst"] / fp64_rate
        return {"fp64_inst_per_call": ncu[name]["fp64_inst"], "issue_bound_ms": 1e3 * t_min,
                "frac": t_min / (ms / 1e3)}
    line = {
        "metric": "tracer cell-steps/s at 512^2x50 (advect_fct + PPM_H4 remap, FP64)",
        "value": value,
        "unit": "tracer cell-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded basin: Gaussian-bump bathymetry, 15% land, T/S stratification, eddy flow)",
        "config": workload_config(w, world),
        "roofline": {"bound": "hbm", "kernel": dominant[0], "achieved": dominant[1], "peak": pk["hbm_gbs"],
                     "unit": "GB/s", "frac": dominant[1] / pk["hbm_gbs"], "peak_source": pk["source"],
                     "traffic": ncu.get(dominant[0], {}).get("dram_bytes"),
                     "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum summed over the call's kernels",
                     "traffic_captured": NCU_CAPTURED,
                     "algorithmic_bytes_per_launch": dominant[3],
                     "avg_launch_ms": dominant[2],
                     "fp64_issue_bound": {"advect_fct": fp64_part("advect_fct", adv_avg),
                                          "remap_columns": fp64_part("remap_columns", rem_avg),
                                          "peak": "64 FP64 lanes x 148 SMs x median SM clock under load"},
                     "parts": {"advect_fct": {"ms": adv_avg, "GB/s": adv_gbs, "bytes": ab["advect"]},
                               "remap_columns": {"ms": rem_avg, "GB/s": rem_gbs, "bytes": ab["remap"]},
                               "step": {"ms": ms / args.steps,
                                        "GB/s": ab["step"] / (ms / args.steps / 1e3) / 1e9}}},
        "e2e": {"value": job_rate(cells, world, e2e_two_ms), "unit": "tracer cell-steps/s",
                "h2d_bytes_per_step": h2d + stack, "d2h_bytes_per_step": d2h + stack, "ms_per_step": e2e_two_ms,
                "api": "TracerAdvection.advect_fct + remap_columns (the reference's two drop-in calls) on pinned "
                       "host tensors",
                "one_call": {"value": job_rate(cells, world, e2e_ms), "ms_per_step": e2e_ms,
                             "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                             "api": "pyocean_b200.ale_tracer_step (advect_fct then remap_columns in one call, the "
                                    "advected stack kept on the device) on pinned host tensors",
                             "copy_bound_ms": 1e3 * max(h2d / h2d_gbs, d2h / d2h_gbs) / 1e9},
                "copy_bound_ms": 1e3 * max((h2d + stack) / h2d_gbs, (d2h + stack) / d2h_gbs) / 1e9,
                "copy_gbs": {"h2d": h2d_gbs, "d2h": d2h_gbs,
                             "what": "one plain pinned copy of a 105 MB block each way, timed alone; the bound is the "
                                     "larger direction's bytes at that rate (the two directions overlap)"}},
        "mixed": {"value": job_rate(cells * args.steps, world, mixed_ms), "ms_per_step": mixed_ms / args.steps,
                  "advect_fct_ms": mixed_adv, "speedup_vs_f64": ms / mixed_ms,
                  "what": "pocean_advect_fct_mixed (FP32 WENO5 weights and face values, FP64 fluxes, limiter and "
                          "bookkeeping) + FP64 PPM_H4 remap, same workload"},
        "gpu_launches": stepper.launches_per_step * args.steps,
        "clocks": clk,
    }
    return line


def main():
    args = parse()
    rank, world, local_rank = ranks_from_env()
    if args.impl == "reference":
        if rank != 0:
            return
        w = make_workload(args.workload, args.basin_size)
        # the arm's own steps: K whole steps after min(W, 1) untimed ones, cut short after --ref-seconds so that
        # the run ends within a few minutes
        s = cpu_sample(w, args.ref_seconds, max_steps=args.steps, warmup=min(args.warmup, 1))
        line = {"metric": "tracer cell-steps/s at 512^2x50 (advect_fct + PPM_H4 remap, FP64)", "value": s["value"],
                "unit": "tracer cell-steps/s", "n_gpus": world, "steps": s["steps"], "warmup": min(args.warmup, 1),
                "ms_per_step": 1e3 * s["seconds"] / s["steps"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (same seeded workload)", "impl": "reference",
                "config": workload_config(w, world), "cpu_baseline": {k: s[k] for k in
                                                                      ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": s["value"], "unit": "tracer cell-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local_rank))
    line = run_ours(args, rank, world, local_rank)
    import torch
    torch.cuda.empty_cache()
    # the single-GPU reports run on one GPU only (a scaling run holds its GPUs for the timed replicas alone)
    if not args.no_neighbours and world == 1:
        from pyocean_b200.neighbours_report import neighbours_report
        line["neighbours"] = neighbours_report()
        torch.cuda.empty_cache()
    if args.batched_steps > 0 and world == 1:
        from pyocean_b200.batch_report import batched_report
        line["batched"] = batched_report(steps=args.batched_steps)
        torch.cuda.empty_cache()
    if args.mixed_steps > 0 and world == 1:
        from pyocean_b200.accuracy import mixed_report
        line["mixed_accuracy"] = mixed_report(steps=args.mixed_steps, nx=1024, ny=1024, n=75, nt=6,
                                              yardsticks=("ale",))
        torch.cuda.empty_cache()
    if args.serve_jobs > 0 and world == 1:
        from pyocean_b200.serve import serve_report
        line["served"] = serve_report(n_jobs=args.serve_jobs, rate=args.serve_rate)
        torch.cuda.empty_cache()
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            s = cpu_sample(make_workload(args.workload, args.basin_size), args.cpu_seconds)
            line["cpu_baseline"] = {k: s[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
