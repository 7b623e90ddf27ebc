"""
Error of the mixed-precision step against the FP64 path (whose results equal the reference's bit for bit).

``mixed_report`` runs the same sequence of ALE tracer steps (advect_fct + PPM_H4 remap of every tracer) twice on
the GPU — FP64 and mixed (FP32 WENO5 weights and face values) — and reports per tracer the max and RMS error of the
mixed result against the FP64 one (absolute and relative to the field's range), the undershoot / overshoot of the
mixed result below / above the initial range, and the relative change of the tracer content through the advection
(sum V1 c_new vs sum V0 c) and through the remap (column sums of h c), each taken over the whole run.

As a yardstick of how strongly the scheme itself amplifies tiny perturbations over the run (WENO weights and FCT
switching at fronts are not smooth functions of the data), the FP64 path is also run from initial fields moved by
one unit in the last place, and its difference to the unperturbed FP64 run is reported beside the mixed error.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import workloads as W
from .step import ALETracerStep


def mixed_report(steps: int = 100, nx: int = 1024, ny: int = 1024, n: int = 75, nt: int = 6, seed: int = 0,
                 device=None) -> dict:
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    w = W.basin(seed=seed, nx=nx, ny=ny, n=n, nt=nt, passive="tophat")
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                     # noqa: E731
    V0, V1, Qx, Qy = g(w.V0), g(w.V1), g(w.Qx), g(w.Qy)
    ok = g(w.ok.view(np.uint8))
    wet = g(w.wet.astype(np.uint8))
    hs, ht = g(w.h_src), g(w.h_tgt)
    flags = 0
    out = {}
    lo = w.C.reshape(nt, -1).min(axis=1)
    hi = w.C.reshape(nt, -1).max(axis=1)
    for mode in ("f64", "mixed", "f64_ulp"):
        mixed = mode == "mixed"
        step = ALETracerStep(nt, n, ny, nx, w.dt, flags, w.remap_scheme, device=dev, mixed=mixed)
        c = g(w.C if mode != "f64_ulp" else np.nextafter(w.C, np.inf))
        nxt = torch.empty_like(c)
        adv_err = np.zeros(nt)
        rem_err = np.zeros(nt)
        for _ in range(steps):
            a = step.advect(c, V0, V1, Qx, Qy, ok)
            before = (V0[None] * c).sum(dim=(1, 2, 3))
            after = (V1[None] * a).sum(dim=(1, 2, 3))
            adv_err = np.maximum(adv_err, (torch.abs(after - before) / torch.abs(before)).cpu().numpy())
            step.remap(hs, a, ht, wet, nxt)
            cin = (hs[None] * a).sum(dim=(1, 2, 3))
            cout = (ht[None] * nxt).sum(dim=(1, 2, 3))
            rem_err = np.maximum(rem_err, (torch.abs(cout - cin) / torch.abs(cin)).cpu().numpy())
            c, nxt = nxt, c
        out[mode] = (c.cpu().numpy(), adv_err, rem_err)
        del step
        torch.cuda.empty_cache()
    ref, _, _ = out["f64"]
    mix, adv_m, rem_m = out["mixed"]
    ulp, _, _ = out["f64_ulp"]
    _, adv_f, rem_f = out["f64"]
    wetc = np.broadcast_to(w.wet[None], (n, ny, nx))
    names = ["T", "S"] + [f"passive{m - 1}" for m in range(2, nt)]
    tracers = []
    for m in range(nt):
        d = (mix[m] - ref[m])[wetc]
        rng = float(hi[m] - lo[m]) or 1.0
        tracers.append(dict(
            tracer=names[m], max_abs_err=float(np.abs(d).max()), rms_abs_err=float(np.sqrt(np.mean(d * d))),
            max_rel_err=float(np.abs(d).max() / max(np.abs(ref[m][wetc]).max(), 1e-300)),
            max_err_over_range=float(np.abs(d).max() / rng),
            f64_one_ulp_max_abs_diff=float(np.abs((ulp[m] - ref[m])[wetc]).max()),
            f64_one_ulp_rms_abs_diff=float(np.sqrt(np.mean((ulp[m] - ref[m])[wetc] ** 2))),
            undershoot=float(max(0.0, lo[m] - mix[m][wetc].min())), overshoot=float(max(0.0, mix[m][wetc].max() - hi[m])),
            f64_undershoot=float(max(0.0, lo[m] - ref[m][wetc].min())),
            f64_overshoot=float(max(0.0, ref[m][wetc].max() - hi[m])),
            content_change_advect_mixed=float(adv_m[m]), content_change_advect_f64=float(adv_f[m]),
            content_change_remap_mixed=float(rem_m[m]), content_change_remap_f64=float(rem_f[m])))
    return dict(workload=w.name, steps=steps, dtype="mixed (FP32 WENO5 weights/faces) vs f64", tracers=tracers)


if __name__ == "__main__":
    import json
    import sys
    _lib.lib()
    steps = int(sys.argv[1]) if len(sys.argv) > 1 else 100
    print(json.dumps(mixed_report(steps=steps)))
