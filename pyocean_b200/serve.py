"""
Continuous-batching server of advect-and-remap jobs on one GPU.

A job is a z* box (nx, ny, nz, nt tracers, seed) to be advanced ``steps`` ALE tracer steps (advect_fct + PPM_H4
remap of every tracer).  Jobs arrive over time.  The server keeps every admitted job's state (tracer stacks,
thicknesses, transports, workspace) resident in HBM and advances ALL admitted jobs together, one batched step at a
time (every pass one launch over all jobs, as in ``batch.DomainBatch``).  Between steps it admits the jobs that have
arrived — in arrival order, while the HBM budget and the slot count allow — and retires the jobs that have run
their steps, so a job that arrives while others run joins the next step instead of waiting for them (continuous
batching, as LLM servers batch requests per decoding iteration).  Which admitted jobs a step advances is the
policy's (``Server._select``).  By default (``adaptive``) it depends on the backlog: while the admitted jobs'
remaining work is short (below ``backlog_cells`` tracer cell-steps, about 1.5 s of GPU work), the oldest job plus
the small jobs that fit beside it without slowing it by more than ``share`` (5 %), so the long jobs of the tail keep
close to their run-alone time while short jobs never wait behind them; once the backlog is longer, every admitted
job, so the GPU runs the largest batches and the queue drains at the batched rate.  A step that advances one job
alone runs the single-domain entry points (same results: the batched kernels compute each domain as they do), as a
batched launch over one domain costs 12-15 % more.  The host only enqueues work: it runs at most
``max_ahead`` iterations ahead of the GPU, so the device queue never drains while jobs are active.

Per job the report has the latency from arrival to the completion of its last step on the device (CUDA event
timestamps against a start event taken with the host clock's zero), and the queueing delay before admission.  The
same stream can be served one job at a time (``max_slots=1``, ``batched=False``: each job alone with the
single-domain entry points) for comparison.  A job's result is independent of what else runs beside it: the batched
kernels compute each domain exactly as the single-domain entry points do.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from . import workloads as W
from .batch import Domain, _Plan, sequential_step


@dataclass
class Job:
    id: int
    arrival: float            # seconds after the start of the stream
    nx: int
    ny: int
    nz: int
    nt: int
    steps: int
    seed: int
    # filled in by the server
    admitted: float = math.nan
    latency_s: float = math.nan
    done_steps: int = 0
    flip: int = 0             # the current state is in C_next
    dom: Domain | None = None
    done_event: torch.cuda.Event | None = None
    result: torch.Tensor | None = None
    digest: torch.Tensor | None = None
    nbytes: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def cell_steps(self) -> int:
        return self.nt * self.nz * self.ny * self.nx * self.steps


def job_stream(n_jobs: int, seed: int = 0, rate: float = 20.0, size_lo=(32, 32, 10), size_hi=(512, 512, 75),
               steps=(10, 200), tracers=(1, 4)) -> list[Job]:
    """``n_jobs`` jobs with Poisson arrivals at ``rate`` per second; nx, ny and nz each lognormal between the
    bounds (median at their geometric mean, the bounds at -/+ 2 sigma, clipped), steps and tracer counts uniform."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_jobs))
    lo, hi = np.log(np.asarray(size_lo, float)), np.log(np.asarray(size_hi, float))
    mu, sig = 0.5 * (lo + hi), 0.25 * (hi - lo)
    dims = np.exp(np.clip(rng.normal(mu, sig, (n_jobs, 3)), lo, hi)).round().astype(int)
    nsteps = rng.integers(steps[0], steps[1] + 1, n_jobs)
    ntr = rng.integers(tracers[0], tracers[1] + 1, n_jobs)
    return [Job(i, float(t[i]), int(dims[i, 0]), int(dims[i, 1]), int(dims[i, 2]), int(ntr[i]), int(nsteps[i]),
                seed * 100003 + i) for i in range(n_jobs)]


def job_bytes(nx: int, ny: int, nz: int, nt: int) -> int:
    """HBM a job holds while admitted: three stacks, six geometry fields, the masks and the FCT workspace."""
    cells = nz * ny * nx
    ws = _lib.lib().pocean_advect_fct_workspace_bytes(nt, nz, ny, nx)
    return 24 * nt * cells + 8 * (4 * cells + nz * ny * (nx + 1) + nz * (ny + 1) * nx) + cells + ny * nx + ws


def make_domain(job: Job, device) -> Domain:
    f = W.zstar_box_device(job.seed, job.nx, job.ny, job.nz, job.nt, device)
    return Domain.from_tensors(f["C"], f["V0"], f["V1"], f["Qx"], f["Qy"], f["ok"], f["h_src"], f["h_tgt"],
                               f["wet"], f["flags"], f["dt"], f["remap_scheme"])


class Server:
    """Serves a job stream; ``run`` returns the per-job and aggregate report."""

    POLICIES = ("adaptive", "oldest_first", "all")

    def __init__(self, device=None, mixed: bool = True, batched: bool = True, max_slots: int = 256,
                 hbm_budget: int | None = None, max_ahead: int = 3, max_steps_per_iter: int = 4,
                 tile_rows: int = 8, remap_nf: int = 2, keep_results: bool = False, policy: str = "adaptive",
                 fill_cells: int = 4_000_000, share: float = 0.05, backlog_cells: float = 6e9) -> None:
        if policy not in self.POLICIES:
            raise ValueError(f"policy {policy!r}: use one of {self.POLICIES}")
        self.policy, self.fill_cells, self.share = policy, int(fill_cells), float(share)
        self.backlog_cells = float(backlog_cells)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.mixed, self.batched = bool(mixed), bool(batched)
        self.max_slots = 1 if not batched else int(max_slots)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.6 * free)
        self.hbm_budget = int(hbm_budget)
        self.max_ahead, self.kmax = int(max_ahead), int(max_steps_per_iter)
        self.tile_rows, self.remap_nf = int(tile_rows), int(remap_nf)
        self.keep_results = bool(keep_results)

    def run(self, jobs: list[Job], clock=time.perf_counter) -> dict:
        dev = self.device
        stream = torch.cuda.current_stream(dev)
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        waiting: deque[Job] = deque()
        active: list[Job] = []
        used = 0
        peak_used = 0
        peak_active = 0
        inflight: deque[torch.cuda.Event] = deque()
        plan = None
        step_set = None
        plan_buf = torch.empty(_lib.lib().pocean_batch_device_bytes(self.max_slots), dtype=torch.uint8, device=dev)
        parity = 0
        iters = launches = 0
        rejected = []
        occupancy = []
        torch.cuda.synchronize(dev)
        start = torch.cuda.Event(enable_timing=True)
        t0 = clock()
        start.record(stream)
        while pending or waiting or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            changed = False
            while waiting and len(active) < self.max_slots:
                j = waiting[0]
                j.nbytes = job_bytes(j.nx, j.ny, j.nz, j.nt)
                if j.nbytes > self.hbm_budget:            # can never fit: refused
                    rejected.append(waiting.popleft())
                    continue
                if used + j.nbytes > self.hbm_budget:
                    break                                  # first in line waits for memory
                waiting.popleft()
                j.admitted = now
                j.dom = make_domain(j, dev)
                used += j.nbytes
                active.append(j)
                changed = True
            peak_used, peak_active = max(peak_used, used), max(peak_active, len(active))
            if not active:
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (clock() - t0))))
                continue
            if changed or step_set is None:
                step_set = self._select(active)
                plan = None             # built for the stepped jobs with their current orientation
            k = min(self.kmax, min(j.steps - j.done_steps for j in step_set))
            if self.batched and len(step_set) > 1:
                if plan is None:
                    plan = _Plan([j.dom.as_struct(swapped=bool(j.flip)) for j in step_set], self.tile_rows, dev,
                                 buf=plan_buf, stream=stream.cuda_stream)
                    parity = 0
                for _ in range(k):
                    plan.step(parity, self.remap_nf, self.mixed, stream.cuda_stream)
                    parity ^= 1
                launches += k * self._launches(step_set)
            else:
                for j in step_set:
                    for s in range(k):
                        sequential_step([j.dom], j.flip ^ (s & 1), mixed=self.mixed, stream=stream.cuda_stream)
                launches += k * sum(7 + (j.nt >= 2) + (j.nt % 2) + 1 for j in step_set)
            iters += 1
            occupancy.append(len(step_set))
            done = []
            for j in step_set:
                j.done_steps += k
                j.flip ^= k & 1
                if j.done_steps == j.steps:
                    done.append(j)
            if done:
                for j in done:
                    self._retire(j, stream)
                    used -= j.nbytes
                active = [j for j in active if j.done_steps < j.steps]
                step_set = None         # chosen again (and its plan built) before the next step
            ev = torch.cuda.Event()
            ev.record(stream)
            inflight.append(ev)
            while len(inflight) > self.max_ahead:
                inflight.popleft().synchronize()
        torch.cuda.synchronize(dev)
        served = [j for j in jobs if j.done_event is not None]
        for j in served:
            j.latency_s = start.elapsed_time(j.done_event) / 1e3 - j.arrival
        lat = np.array([j.latency_s for j in served]) if served else np.zeros(1)
        end = max((start.elapsed_time(j.done_event) / 1e3 for j in served), default=0.0)
        first = min((j.arrival for j in served), default=0.0)
        work = sum(j.cell_steps for j in served)
        return dict(jobs=len(jobs), served=len(served), rejected=len(rejected),
                    mode=("batched" if self.batched else "one job at a time") + (" mixed" if self.mixed else " f64"),
                    p50_s=float(np.percentile(lat, 50)), p95_s=float(np.percentile(lat, 95)),
                    p99_s=float(np.percentile(lat, 99)), mean_s=float(lat.mean()), max_s=float(lat.max()),
                    makespan_s=end - first, cell_steps=work, throughput=work / max(end - first, 1e-9),
                    unit="tracer cell-steps/s", iterations=iters, gpu_launches=launches,
                    mean_active=float(np.mean(occupancy)) if occupancy else 0.0, peak_active=peak_active,
                    peak_hbm_bytes=peak_used, hbm_budget=self.hbm_budget)

    def _select(self, active: list[Job]) -> list[Job]:
        """The jobs the next steps advance.  ``all``: every admitted job (processor sharing).  ``oldest_first``: the
        job that arrived first, plus the others in increasing remaining work while the combined step stays within
        max(fill_cells, (1 + share) x the oldest job's step): the oldest job is never slowed by more than ``share``
        (so a long job's latency stays close to running it alone), and small jobs fill the GPU beside it.
        ``adaptive``: ``all`` while the admitted jobs' remaining tracer cell-steps exceed ``backlog_cells``, else
        ``oldest_first``.  One job at a time (not batched): the oldest alone."""
        oldest = min(active, key=lambda j: (j.arrival, j.id))
        if not self.batched:
            return [oldest]
        cells = lambda j: j.nt * j.nz * j.ny * j.nx                                     # noqa: E731
        if self.policy == "all" or (self.policy == "adaptive" and
                                    sum((j.steps - j.done_steps) * cells(j) for j in active) > self.backlog_cells):
            return list(active)
        budget = max(self.fill_cells, (1.0 + self.share) * cells(oldest))
        chosen, used = [oldest], cells(oldest)
        for j in sorted((j for j in active if j is not oldest), key=lambda j: ((j.steps - j.done_steps) * cells(j),
                                                                            j.arrival)):
            if used + cells(j) <= budget:
                chosen.append(j)
                used += cells(j)
        return chosen

    def _launches(self, active) -> int:
        if self.remap_nf == 2:
            return 7 + any(j.nt >= 2 for j in active) + any(j.nt % 2 for j in active) + 1
        return 9

    def _retire(self, j: Job, stream) -> None:
        """Marks the job done on the device and releases its buffers (stream-ordered: the caching allocator hands
        them out again only to work that follows on this stream)."""
        d = j.dom
        res = d.C_next if j.flip else d.C
        j.digest = (res * d.V0[None]).sum(dim=(1, 2, 3))       # tracer content, kept on the device
        j.done_event = torch.cuda.Event(enable_timing=True)
        j.done_event.record(stream)
        if self.keep_results:
            j.result = res
        j.dom = None


def serve_report(n_jobs: int = 200, rate: float = 15.0, seed: int = 0, device=None, batched_f64: bool = False,
                 saturated: bool = True, policies: bool = True) -> dict:
    """Serves the seeded Poisson stream batched in mixed precision (the served form) and one job at a time with the
    plain FP64 kernels, then (``saturated``) both once more with every job arriving at once (their saturated
    throughput); ``batched_f64`` adds the batched FP64 form, ``policies`` the served form under the two fixed
    step-set policies (``all``, ``oldest_first``) beside the default one.  Latencies in seconds."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    # warm-up: load the library and the kernels, fill the allocator's pools
    Server(dev).run(job_stream(8, seed=seed + 7, rate=1e9))
    Server(dev, mixed=False, batched=False).run(job_stream(4, seed=seed + 7, rate=1e9))
    stream = lambda r: job_stream(n_jobs, seed=seed, rate=r)                             # noqa: E731
    out = dict(stream=dict(jobs=n_jobs, rate_per_s=rate, seed=seed, sizes="nx, ny lognormal 32..512, nz lognormal "
                           "10..75 (bounds at 2 sigma), steps uniform 10..200, tracers uniform 1..4, z* boxes "
                           "generated on the device per job"))
    out["batched_mixed"] = Server(dev, mixed=True).run(stream(rate))
    out["one_at_a_time_f64"] = Server(dev, mixed=False, batched=False).run(stream(rate))
    if policies:
        out["batched_mixed_all_jobs_every_step"] = Server(dev, mixed=True, policy="all").run(stream(rate))
        out["batched_mixed_oldest_first"] = Server(dev, mixed=True, policy="oldest_first").run(stream(rate))
    if batched_f64:
        out["batched_f64"] = Server(dev, mixed=False).run(stream(rate))
    out["p99_ratio_plain_vs_served"] = out["one_at_a_time_f64"]["p99_s"] / out["batched_mixed"]["p99_s"]
    if saturated:
        out["saturated_batched_mixed"] = Server(dev, mixed=True).run(stream(1e9))
        out["saturated_one_at_a_time_f64"] = Server(dev, mixed=False, batched=False).run(stream(1e9))
        out["saturated_throughput_ratio_served_vs_plain"] = (out["saturated_batched_mixed"]["throughput"] /
                                                             out["saturated_one_at_a_time_f64"]["throughput"])
    return out


if __name__ == "__main__":
    import json
    import sys
    # python -m pyocean_b200.serve [jobs] [rate] [--no-saturated] [--no-batched-f64] [--no-policies]
    pos = [x for x in sys.argv[1:] if not x.startswith("--")]
    n = int(pos[0]) if pos else 200
    r = float(pos[1]) if len(pos) > 1 else 15.0
    print(json.dumps(serve_report(n, r, batched_f64="--no-batched-f64" not in sys.argv,
                                  saturated="--no-saturated" not in sys.argv,
                                  policies="--no-policies" not in sys.argv)))
