"""
The mixed-precision FCT step (pocean_advect_fct_mixed: FP32 WENO5 weights and face values, FP64 fluxes, limiter
and bookkeeping) against the FP64 reference arithmetic.

Its bar: at most 1e-5 relative tracer error for the operator it changes (one step against the golden cases, and
100 steps of advect_fct on a basin with four top-hat tracers against the FP64 path), tracer content conserved to
1e-13 relative, and the FCT bounds kept.  Over 100 ALE steps (advect_fct + PPM_H4 remap) the FP64 path itself
carries a one-ulp change of its initial fields to about 4e-5 of a tracer's range (the remap's limiters switch
discontinuously at fronts), so there the test asserts an RMS error of at most 1e-5 of the range, a max error of at
most 1e-3 of the range, and conservation to 1e-13.
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
def report():
    from pyocean_b200.accuracy import mixed_report
    return mixed_report(steps=100, nx=256, ny=256, n=20, nt=6, seed=0)


def test_mixed_advection_100_steps_within_1e5_conserving_and_bounded(report):
    for t in report["sequences"]["advect"]:
        assert t["max_err_over_range"] <= REL_ERR, t
        assert t["content_change_advect_mixed"] <= CONSERVATION, t
        assert t["undershoot"] <= 1e-12 and t["overshoot"] <= 1e-12, t


def test_mixed_ale_steps_rms_error_and_conservation(report):
    for t in report["sequences"]["ale"]:
        assert t["rms_err_over_range"] <= REL_ERR, t
        assert t["max_err_over_range"] <= 1e-3, t
        assert t["content_change_advect_mixed"] <= CONSERVATION, t
        assert t["content_change_remap_mixed"] <= CONSERVATION, t


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


@pytest.mark.parametrize("scale", [1e-35, 1e12])
@pytest.mark.parametrize("scheme", ["weno5", "weno5js"])
def test_mixed_keeps_fp64_where_fp32_would_lose_the_stencil(scale, scheme):
    # stencils whose variation FP32 cannot carry (below 1e-30, or above 1e8 for the absolute-epsilon forms) take the
    # FP64 arithmetic: the mixed step of a field scaled to 1e-35 or 1e12 stays within the bar of the FP64 result
    rng = np.random.default_rng(21)
    n, ny, nx = 3, 29, 41
    h = rng.uniform(1.0, 5.0, (n, ny, nx))
    V0 = 1e6 * h
    Qx = rng.uniform(-0.4, 0.4, (n, ny, nx + 1)) * 1e3 * np.concatenate([h[..., :1], h], -1)
    Qy = rng.uniform(-0.4, 0.4, (n, ny + 1, nx)) * 1e3 * np.concatenate([h[:, :1], h], 1)
    Qx[..., 0] = Qx[..., -1] = 0.0
    Qy[:, 0] = Qy[:, -1] = 0.0
    V1 = V0 - 30.0 * (Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:] - Qy[:, :-1])
    ok = V1 > 0
    C = scale * (1.0 + rng.normal(0, 0.3, (2, n, ny, nx)))
    ref = O.TracerAdvection(scheme=scheme, time="ssprk3", dt=30.0)
    gpu = P.TracerAdvection(scheme=scheme, time="ssprk3", dt=30.0, precision="mixed")
    r = ref.advect_fct(C, V0, V1, Qx, Qy, ok)
    g = gpu.advect_fct(C, V0, V1, Qx, Qy, ok)
    assert np.all(np.isfinite(g))
    for m in range(2):
        assert _rel_err(g[m], r[m]) <= REL_ERR
