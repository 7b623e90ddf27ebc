"""
The mixed-precision FCT step (pocean_advect_fct_mixed: FP32 WENO5 weights and face values, FP64 fluxes, limiter
and bookkeeping) against the FP64 reference arithmetic.  Its bar: at most 1e-5 relative tracer
error, tracer content conserved to 1e-13 relative, and the FCT bounds kept.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import case_open, case_periodic, load_golden
import pyocean_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_ERR = 1e-5
CONSERVATION = 1e-13

FCT = load_golden("fct")


def _rel_err(got, ref):
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.parametrize("case", sorted(c for c in FCT if not bool(FCT[c]["unlimited"])))
def test_mixed_step_is_within_1e5_of_reference(case):
    rec = FCT[case]
    adv = P.TracerAdvection(scheme=str(rec["scheme"]), time="ssprk3", dt=float(rec["dt"]),
                            ob=P.OpenEdges(case_open(rec)), precision="mixed")
    adv.per = P.Periodic(case_periodic(rec))
    out = adv.advect_fct(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["ok"], inflow=rec.get("inflow"))
    assert _rel_err(out, rec["out"]) <= REL_ERR


@pytest.fixture(scope="module")
def patches():
    from pyocean_b200 import workloads as W
    return W.basin(seed=4, nx=192, ny=160, n=12, nt=4, passive="tophat")


def test_mixed_multistep_error_conservation_and_bounds(patches):
    import torch
    w = patches
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()                 # noqa: E731
    C, V0, V1, Qx, Qy, ok = dev(w.C), dev(w.V0), dev(w.V1), dev(w.Qx), dev(w.Qy), dev(w.ok)
    f64 = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=w.dt)
    mix = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=w.dt, precision="mixed")
    a = b = C
    lo = C.amin(dim=(1, 2, 3)).cpu().numpy()
    hi = C.amax(dim=(1, 2, 3)).cpu().numpy()
    for _ in range(20):                               # V0 == V1 here (divergence-free flow): the step repeats
        a = f64.advect_fct(a, V0, V1, Qx, Qy, ok)
        b = mix.advect_fct(b, V0, V1, Qx, Qy, ok)
    a, b = a.cpu().numpy(), b.cpu().numpy()
    for m in range(a.shape[0]):
        assert _rel_err(b[m], a[m]) <= REL_ERR, m
        c0 = (w.V0 * w.C[m]).sum()
        cb = (w.V1 * b[m]).sum()
        assert abs(cb - c0) <= CONSERVATION * abs(c0), m
        wet = w.ok
        span = hi[m] - lo[m]
        assert b[m][wet].min() >= lo[m] - 1e-12 * span and b[m][wet].max() <= hi[m] + 1e-12 * span, m


def test_mixed_matches_oracle_on_ragged_open_periodic_case():
    rng = np.random.default_rng(12)
    n, ny, nx = 4, 37, 70
    h = rng.uniform(1.0, 5.0, (n, ny, nx))
    V0 = 1e6 * h
    Qx = rng.uniform(-0.4, 0.4, (n, ny, nx + 1)) * 1e3 * np.concatenate([h[..., :1], h], -1)
    Qy = rng.uniform(-0.4, 0.4, (n, ny + 1, nx)) * 1e3 * np.concatenate([h[:, :1], h], 1)
    Qx[..., -1] = Qx[..., 0]
    V1 = V0 - 30.0 * (Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:] - Qy[:, :-1])
    ok = V1 > 0
    T = 7.0 + rng.normal(0, 1, (n, ny, nx))
    C = np.stack([T, T ** 2])
    infl = np.stack([np.full(T.shape, 9.0), np.full(T.shape, 81.0)])
    ref = O.TracerAdvection(scheme="weno5", time="ssprk3", dt=30.0, ob=O.OpenEdges(("south", "north")))
    ref.per = O.Periodic(("x",))
    gpu = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=30.0, ob=P.OpenEdges(("south", "north")),
                            precision="mixed")
    gpu.per = P.Periodic(("x",))
    r = ref.advect_fct(C, V0, V1, Qx, Qy, ok, inflow=infl)
    g = gpu.advect_fct(C, V0, V1, Qx, Qy, ok, inflow=infl)
    for m in range(2):
        assert _rel_err(g[m], r[m]) <= REL_ERR
