"""
The batched uneven-domains measurement: 64 independent z* boxes (nx, ny log-uniform in 96..384, nz in {30, 50, 75},
one tracer each), a 50-step sequence captured as one CUDA graph with autotuned tile shapes, against the same 64
domains stepped one after another with the single-domain entry points.

    python -m pyocean_b200.batch_report [steps]

Reports aggregate tracer cell-steps/s of: the batched FP64 graph, the batched mixed-precision graph, the sequential
plain launches (eager) and the sequential launches captured in a graph (which removes launch overhead but not the
idle SMs of small domains); and whether the batched FP64 result equals the sequential one bit for bit.
"""
from __future__ import annotations

import time

import torch

from . import workloads as W
from .batch import Domain, DomainBatch, sequential_launches, sequential_step


def _timed(fn, stream) -> float:
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def batched_report(steps: int = 50, seed: int = 0, ndom: int = 64, device=None, tune_steps: int = 2) -> dict:
    if steps < 2 or steps % 2:
        raise ValueError("steps must be even")
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    t0 = time.perf_counter()
    doms = [Domain.from_workload(w, dev) for w in W.uneven_domains(seed=seed, ndom=ndom)]
    gen_s = time.perf_counter() - t0
    cells = sum(d.cells for d in doms)
    init = [d.C.clone() for d in doms]
    stream = torch.cuda.current_stream(dev)

    def restore():
        for d, c in zip(doms, init):
            d.C.copy_(c)

    # sequential plain launches, eager
    for p in (0, 1):
        sequential_step(doms, p)
    restore()
    seq_ms = _timed(lambda: [sequential_step(doms, i % 2) for i in range(steps)], stream)
    seq_final = [d.C.clone() for d in doms]

    # sequential launches captured in one graph
    restore()
    gs = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        with torch.cuda.graph(gs, stream=side):
            for i in range(steps):
                sequential_step(doms, i % 2, stream=side.cuda_stream)
    stream.wait_stream(side)
    restore()
    seq_graph_ms = _timed(gs.replay, stream)
    del gs

    # batched FP64: autotuned tile shapes, the sequence captured as one graph
    restore()
    batch = DomainBatch(doms)
    tune = batch.autotune(steps=tune_steps)
    g = batch.capture(steps)
    restore()
    batch.parity = 0
    bat_ms = _timed(g.replay, stream)
    equal = all(torch.equal(d.C, s) for d, s in zip(doms, seq_final))
    del g

    # batched mixed precision
    restore()
    mb = DomainBatch(doms, tile_rows=tune["tile_rows"], remap_nf=tune["remap_nf"], mixed=True)
    gm = mb.capture(steps)
    restore()
    mix_ms = _timed(gm.replay, stream)
    err = max(float((d.C - s).abs().max() / s.abs().max()) for d, s in zip(doms, seq_final))
    del gm
    rate = lambda ms: cells * steps / (ms / 1e3)                                          # noqa: E731
    out = dict(workload=f"{ndom} uneven z* boxes (nx, ny log-uniform 96..384, nz in 30/50/75, seed {seed})",
               domains=ndom, tracer_cells_per_step=cells, steps=steps,
               batched_f64=dict(value=rate(bat_ms), ms_per_step=bat_ms / steps, launches_per_step=batch.launches_per_step),
               batched_mixed=dict(value=rate(mix_ms), ms_per_step=mix_ms / steps, max_rel_err_vs_f64=err),
               sequential_eager=dict(value=rate(seq_ms), ms_per_step=seq_ms / steps,
                                     launches_per_step=sequential_launches(doms)),
               sequential_graph=dict(value=rate(seq_graph_ms), ms_per_step=seq_graph_ms / steps),
               speedup_batched_vs_sequential=seq_ms / bat_ms, speedup_mixed_batched_vs_sequential=seq_ms / mix_ms,
               batched_bitwise_equal_to_sequential=bool(equal), autotune=tune, generate_s=gen_s,
               unit="tracer cell-steps/s")
    return out


def idle_report(seed: int = 0, ndom: int = 64, steps: int = 20, device=None) -> dict:
    """Two plain warm-up steps and one more plain step of the batched FP64 step (launches 19-27 of the run: under
    an ncu launch list, the sum of their durations against the step time of the replayed graph that follows bounds
    what any scheduling of the same passes could save between them), then that graph's device time per step."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    doms = [Domain.from_workload(w, dev) for w in W.uneven_domains(seed=seed, ndom=ndom)]
    batch = DomainBatch(doms)
    stream = torch.cuda.current_stream(dev)
    batch.step(2)
    torch.cuda.synchronize()
    batch.step(1)
    torch.cuda.synchronize()
    g = batch.capture(steps)
    g.replay()
    graph_ms = min(_timed(g.replay, stream) for _ in range(3)) / steps
    del g
    return dict(workload=f"{ndom} uneven z* boxes (seed {seed})", graph_ms_per_step=graph_ms,
                launches_per_step=batch.launches_per_step, tracer_cells_per_step=batch.cells)


if __name__ == "__main__":
    # python -m pyocean_b200.batch_report [steps]   |   python -m pyocean_b200.batch_report idle
    import json
    import sys
    if len(sys.argv) > 1 and sys.argv[1] == "idle":
        print(json.dumps(idle_report()))
    else:
        print(json.dumps(batched_report(steps=int(sys.argv[1]) if len(sys.argv) > 1 else 50)))
