"""
Error of the mixed-precision step against the FP64 path (whose results equal the reference's bit for bit).

``mixed_report`` runs the same sequence of steps several times on the GPU and reports, per tracer, the max and RMS
error against the FP64 run (absolute and relative to the tracer's initial range), the undershoot / overshoot below
/ above the initial range, and the relative change of the tracer content through the advection (sum V1 c_new vs
sum V0 c) and through the remap (column sums of h c), each the largest over the run.  Two sequences:

* ``advect``: advect_fct alone, step after step (the operator whose arithmetic the mixed form changes: FP32 WENO5
  weights and face values);
* ``ale``: the ALE tracer step, advect_fct then the PPM_H4 remap of every tracer from the Lagrangian thicknesses
  back onto the target grid, step after step.

The ALE sequence amplifies any perturbation of its state, whatever its source: the remap's limiters (CW84, the
edge bounding and the discontinuity check) switch discontinuously at fronts, and the advection carries each switch
on.  Yardsticks measure that amplification with FP64 arithmetic only, each reported as its max error against the
FP64 run (over the tracer's range):

* ``f64_one_ulp``: the FP64 sequence started from initial fields moved up by one unit in the last place;
* ``mixed_first_step_only``: the FP64 sequence whose first step alone is the mixed one;
* ``f64_ulp_noise_every_step``: the FP64 sequence with every value moved by one unit in the last place, up or down
  at random (seeded), after every step — a perturbation at every step, as the mixed arithmetic makes, but ~10^6
  times smaller than its per-step error;
* ``f64_rel_noise_every_step``: the same with every value multiplied by 1 + e u, u uniform in [-1, 1], for
  e = 1e-13 and 1e-10 (the mixed form's per-step error is below ~1e-10 of the range).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import workloads as W
from .step import ALETracerStep


REL_NOISE = (1e-13, 1e-10)


def _run(w, dev, steps: int, mixed_steps: int, remap: bool, ulp: bool, noise: float = 0.0):
    """Final stack of `steps` steps (the first `mixed_steps` mixed, the rest FP64) and the largest relative content
    changes through the advection and the remap; ``ulp``: start one ulp up; ``noise``: after every step, -1 moves
    every value one ulp up or down at random, e > 0 multiplies it by 1 + e u (u uniform in [-1, 1])."""
    nt, n, ny, nx = w.C.shape
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                     # noqa: E731
    V0, V1, Qx, Qy = g(w.V0), g(w.V1), g(w.Qx), g(w.Qy)
    ok = g(w.ok.view(np.uint8))
    wet = g(w.wet.astype(np.uint8))
    hs, ht = g(w.h_src), g(w.h_tgt)
    f64 = ALETracerStep(nt, n, ny, nx, w.dt, 0, w.remap_scheme, device=dev, mixed=False)
    mix = ALETracerStep(nt, n, ny, nx, w.dt, 0, w.remap_scheme, device=dev, mixed=True) if mixed_steps else None
    c = g(np.nextafter(w.C, np.inf) if ulp else w.C)
    nxt = torch.empty_like(c)
    gen = torch.Generator(device=dev)
    gen.manual_seed(12345)
    pinf = torch.full((), np.inf, dtype=torch.float64, device=dev)
    ninf = -pinf
    adv_err = torch.zeros(nt, dtype=torch.float64, device=dev)
    rem_err = torch.zeros(nt, dtype=torch.float64, device=dev)
    for s in range(steps):
        st = mix if s < mixed_steps else f64
        a = st.advect(c, V0, V1, Qx, Qy, ok)
        before = (V0[None] * c).sum(dim=(1, 2, 3))
        after = (V1[None] * a).sum(dim=(1, 2, 3))
        adv_err = torch.maximum(adv_err, (after - before).abs() / before.abs())
        if remap:
            st.remap(hs, a, ht, wet, nxt)
            cin = (hs[None] * a).sum(dim=(1, 2, 3))
            cout = (ht[None] * nxt).sum(dim=(1, 2, 3))
            rem_err = torch.maximum(rem_err, (cout - cin).abs() / cin.abs())
        else:
            nxt.copy_(a)
        if noise < 0:
            up = torch.rand(nxt.shape, generator=gen, device=dev) < 0.5
            nxt.copy_(torch.where(up, torch.nextafter(nxt, pinf), torch.nextafter(nxt, ninf)))
        elif noise > 0:
            u = torch.rand(nxt.shape, generator=gen, device=dev, dtype=torch.float64) * 2.0 - 1.0
            nxt.mul_(1.0 + noise * u)
            del u
        c, nxt = nxt, c
    del f64, mix
    return c, adv_err.cpu().numpy(), rem_err.cpu().numpy()


def mixed_report(steps: int = 100, nx: int = 1024, ny: int = 1024, n: int = 75, nt: int = 6, seed: int = 0,
                 device=None, sequences=("advect", "ale"), yardsticks=("advect", "ale")) -> dict:
    """The report of the module docstring; ``yardsticks``: the sequences that also run the two FP64 sensitivity
    runs (reported as None elsewhere)."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    w = W.basin(seed=seed, nx=nx, ny=ny, n=n, nt=nt, passive="tophat")
    lo = w.C.reshape(nt, -1).min(axis=1)
    hi = w.C.reshape(nt, -1).max(axis=1)
    rng = np.where(hi > lo, hi - lo, 1.0)
    wetc = torch.from_numpy(np.broadcast_to(w.wet[None], (n, ny, nx)).copy()).to(dev)
    names = ["T", "S"] + [f"passive{m - 1}" for m in range(2, nt)]

    def stats(d):
        d = torch.where(wetc[None], d, torch.zeros_like(d))
        mx = d.abs().amax(dim=(1, 2, 3)).cpu().numpy()
        rms = torch.sqrt((d * d).sum(dim=(1, 2, 3)) / wetc.sum()).cpu().numpy()
        return mx, rms

    out = dict(workload=w.name, steps=steps, dtype="mixed (FP32 WENO5 weights / faces) against FP64",
               sequences={})
    for seq in sequences:
        remap = seq == "ale"
        ref, adv_f, rem_f = _run(w, dev, steps, 0, remap, False)
        mix, adv_m, rem_m = _run(w, dev, steps, steps, remap, False)
        mx, rms = stats(mix - ref)
        cw = torch.where(wetc[None], mix, torch.full_like(mix, np.nan))
        mn = torch.nan_to_num(cw, nan=np.inf).amin(dim=(1, 2, 3)).cpu().numpy()
        mxv = torch.nan_to_num(cw, nan=-np.inf).amax(dim=(1, 2, 3)).cpu().numpy()
        del mix, cw
        ulp_mx = ulp_rms = one_mx = noise_mx = None
        rel_mx = {}
        if seq in yardsticks:
            ulp, _, _ = _run(w, dev, steps, 0, remap, True)
            ulp_mx, ulp_rms = stats(ulp - ref)
            del ulp
            one, _, _ = _run(w, dev, steps, 1, remap, False)
            one_mx, _ = stats(one - ref)
            del one
            nz, _, _ = _run(w, dev, steps, 0, remap, False, noise=-1.0)
            noise_mx, _ = stats(nz - ref)
            del nz
            for e in REL_NOISE:
                nz, _, _ = _run(w, dev, steps, 0, remap, False, noise=e)
                rel_mx[e], _ = stats(nz - ref)
                del nz
        del ref
        torch.cuda.empty_cache()
        tracers = []
        for m in range(nt):
            tracers.append(dict(
                tracer=names[m], max_abs_err=float(mx[m]), rms_abs_err=float(rms[m]),
                max_err_over_range=float(mx[m] / rng[m]), rms_err_over_range=float(rms[m] / rng[m]),
                f64_one_ulp_max_over_range=None if ulp_mx is None else float(ulp_mx[m] / rng[m]),
                f64_one_ulp_rms_over_range=None if ulp_rms is None else float(ulp_rms[m] / rng[m]),
                mixed_first_step_only_max_over_range=None if one_mx is None else float(one_mx[m] / rng[m]),
                f64_ulp_noise_every_step_max_over_range=None if noise_mx is None else float(noise_mx[m] / rng[m]),
                f64_rel_noise_every_step_max_over_range=(None if not rel_mx else
                                                         {f"{e:.0e}": float(v[m] / rng[m]) for e, v in rel_mx.items()}),
                undershoot=float(max(0.0, lo[m] - mn[m])), overshoot=float(max(0.0, mxv[m] - hi[m])),
                content_change_advect_mixed=float(adv_m[m]), content_change_advect_f64=float(adv_f[m]),
                content_change_remap_mixed=float(rem_m[m]) if remap else None,
                content_change_remap_f64=float(rem_f[m]) if remap else None))
        out["sequences"][seq] = tracers
    return out


if __name__ == "__main__":
    import json
    import sys
    _lib.lib()
    # python -m pyocean_b200.accuracy [steps [nx ny nz [sequence ...]]]
    steps = int(sys.argv[1]) if len(sys.argv) > 1 else 100
    size = [int(x) for x in sys.argv[2:5]] if len(sys.argv) > 4 else [1024, 1024, 75]
    seqs = tuple(sys.argv[5:]) or ("advect", "ale")
    print(json.dumps(mixed_report(steps=steps, nx=size[0], ny=size[1], n=size[2], sequences=seqs, yardsticks=seqs)))
