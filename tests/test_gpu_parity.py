"""
Parity of the CUDA path (libpocean_b200.so through the pyocean_b200 drop-ins) with the reference.

* Golden vectors produced by the reference itself (tests/golden/): every FCT, RK3 and remap case.  The bar is the
  required parity tolerance, 1e-12 relative (with an absolute floor of 1e-12 x the field's magnitude for values that
  cross zero); the FP64 kernels evaluate the reference's expressions in its order without FMA contraction, so the
  measured difference is 0 and a second test asserts bit-for-bit equality.
* Larger seeded cases (ragged tile edges, periodic axes, open edges, inflow) against the CPU oracle.
* Full-size (512 x 512 x 50, 2 tracers) properties: conservation to round-off, no new extrema, oracle agreement.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import case_open, case_periodic, load_golden
import pyocean_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-12          # required parity tolerance of the plain FP64 kernels against the reference

FCT = load_golden("fct")
RK3 = load_golden("rk3")
RK3X = load_golden("rk3_ext")
HLP = load_golden("helpers")
REM = load_golden("remap")


def close(got, ref, rtol=RTOL):
    got, ref = np.asarray(got), np.asarray(ref)
    assert got.shape == ref.shape
    scale = np.nanmax(np.abs(ref)) if ref.size else 0.0
    np.testing.assert_allclose(got, ref, rtol=rtol, atol=rtol * scale, equal_nan=True)


def _adv(rec):
    time = str(rec["time"]) if "time" in rec else "ssprk3"
    adv = P.TracerAdvection(scheme=str(rec["scheme"]), time=time, dt=float(rec["dt"]),
                            ob=P.OpenEdges(case_open(rec)))
    adv.per = P.Periodic(case_periodic(rec))
    return adv


def _run_fct(rec):
    adv = _adv(rec)
    adv.record_open_flux = "open_flux" in rec
    fi = int(rec["flux_face_i"]) if "flux_face_i" in rec else None
    res = adv.advect_fct(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["ok"],
                         unlimited=bool(rec["unlimited"]), inflow=rec.get("inflow"), flux_face_i=fi)
    out, fx = (res if fi is not None else (res, None))
    return adv, out, fx


@pytest.mark.parametrize("case", sorted(FCT))
def test_advect_fct_matches_reference(case):
    rec = FCT[case]
    adv, out, fx = _run_fct(rec)
    close(out, rec["out"])
    if fx is not None:
        close(fx, rec["fx_i"])
    if "open_flux" in rec:
        close(adv.last_open_flux, rec["open_flux"], rtol=1e-13)


@pytest.mark.parametrize("case", sorted(FCT))
def test_advect_fct_is_bitwise_equal_to_reference(case):
    rec = FCT[case]
    _, out, fx = _run_fct(rec)
    np.testing.assert_array_equal(out, rec["out"])
    if fx is not None:
        np.testing.assert_array_equal(fx, rec["fx_i"])


@pytest.mark.parametrize("case", sorted(RK3))
def test_advect_rk3_matches_reference_bitwise(case):
    rec = RK3[case]
    adv = _adv(rec)
    fi = int(rec["flux_face_i"]) if "flux_face_i" in rec else None
    res = adv.advect(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["Fz"], rec["ok"],
                     inflow=rec.get("inflow"), flux_face_i=fi)
    out, fx = (res if fi is not None else (res, None))
    close(out, rec["out"])
    np.testing.assert_array_equal(out, rec["out"])
    if fx is not None:
        np.testing.assert_array_equal(fx, rec["fx_i"])


@pytest.mark.parametrize("case", sorted(RK3X))
def test_advect_numpy_path_schemes_match_reference_bitwise(case):
    """upwind3 / upwind1 faces and the 'pc' predictor-corrector step (the reference's NumPy RHS path)."""
    rec = RK3X[case]
    adv = _adv(rec)
    fi = int(rec["flux_face_i"]) if "flux_face_i" in rec else None
    res = adv.advect(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["Fz"], rec["ok"],
                     inflow=rec.get("inflow"), flux_face_i=fi)
    out, fx = (res if fi is not None else (res, None))
    np.testing.assert_array_equal(out, rec["out"])
    if fx is not None:
        np.testing.assert_array_equal(fx, rec["fx_i"])


@pytest.mark.parametrize("case", ["coef_plm", "coef_ppm_h4"])
def test_reconstruct_matches_reference_bitwise(case):
    rec = REM[case]
    coef = np.empty((rec["h"].size, 3))
    got = P.reconstruct(rec["h"], rec["u"], int(rec["scheme"]), P.remap.H_NEGLECT, P.remap.H_NEGLECT_EDGE, coef)
    np.testing.assert_array_equal(got, rec["coef"])
    np.testing.assert_array_equal(coef, rec["coef"])


def test_reconstruct_of_many_columns_equals_the_oracle_column_by_column():
    rng = np.random.default_rng(31)
    n, ny, nx = 12, 5, 7
    h = rng.uniform(0.0, 3.0, (n, ny, nx))
    h[3, 1, 2] = 0.0
    h[5:9, 2, 4] = 1e-12                                      # vanished layers inside a column
    u = rng.normal(10.0, 2.0, (n, ny, nx))
    for scheme in (P.PCM, P.PLM, P.PPM_H4):
        got = P.reconstruct(h, u, scheme)
        assert got.shape == (n, ny, nx, 3)
        for j in range(ny):
            for i in range(nx):
                np.testing.assert_array_equal(got[:, j, i], O.reconstruct(h[:, j, i], u[:, j, i], scheme))
    with pytest.raises(ValueError):
        P.reconstruct(h, u, P.PPM_H4, h_neglect=1e-20)


@pytest.mark.parametrize("case", sorted(HLP))
def test_single_stage_helpers_match_reference_bitwise(case):
    """faces_h, upwind_faces_h, flux_x, rhs, rhs_numpy (tracers.py:139-206) on unpadded arrays."""
    rec = HLP[case]
    adv = _adv(rec)
    C, Qx, Qy, Fz, ok, infl = rec["C"], rec["Qx"], rec["Qy"], rec["Fz"], rec["ok"], rec.get("inflow")
    fx, fy = adv.faces_h(C, Qx, Qy, ok, inflow=infl)
    np.testing.assert_array_equal(fx, rec["faces_h_x"])
    np.testing.assert_array_equal(fy, rec["faces_h_y"])
    ux, uy = adv.upwind_faces_h(C, Qx, Qy, inflow=infl)
    np.testing.assert_array_equal(ux, rec["upwind_x"])
    np.testing.assert_array_equal(uy, rec["upwind_y"])
    np.testing.assert_array_equal(adv.flux_x(C, Qx, Qy, ok, inflow=infl), rec["flux_x"])
    np.testing.assert_array_equal(adv.flux_x(C, Qx, Qy, ok, centred=True, inflow=infl), rec["flux_x_centred"])
    np.testing.assert_array_equal(adv.rhs(C, Qx, Qy, Fz, ok, inflow=infl), rec["rhs"])
    np.testing.assert_array_equal(adv.rhs(C, Qx, Qy, Fz, ok, centred=True, inflow=infl), rec["rhs_centred"])
    np.testing.assert_array_equal(adv.rhs_numpy(C, Qx, Qy, Fz, ok, inflow=infl), rec["rhs_numpy"])


@pytest.mark.parametrize("group", ["cols", "n0n1"])
@pytest.mark.parametrize("scheme", ["pcm", "plm", "ppm_h4"])
def test_remap_columns_match_reference_bitwise(group, scheme):
    rec = REM[group]
    out = P.remap_columns(rec["h_src"], rec["f_src"], rec["h_tgt"], P.SCHEMES[scheme], rec["wet"])
    close(out, rec["out_" + scheme])
    np.testing.assert_array_equal(out, rec["out_" + scheme])


@pytest.mark.parametrize("case", sorted(c for c in REM if c.startswith("short")))
def test_short_columns_match_reference_bitwise(case):
    rec = REM[case]
    np.testing.assert_array_equal(P.remap_column(rec["h_src"], rec["f_src"], rec["h_tgt"], int(rec["scheme"])),
                                  rec["out"])


def test_remap_stack_of_fields_equals_per_field_calls():
    rec = REM["cols"]
    f2 = np.stack([rec["f_src"], rec["f_src"] * 2.0 - 3.0])
    both = P.remap_columns(rec["h_src"], f2, rec["h_tgt"], P.PPM_H4, rec["wet"])
    for m in range(2):
        np.testing.assert_array_equal(both[m], P.remap_columns(rec["h_src"], f2[m], rec["h_tgt"], P.PPM_H4,
                                                               rec["wet"]))


# ---------------------------------------------------------------- known answers of the reference's own tests
def test_ppm_end_values_with_vanished_layers_known_answer():
    # tests/test_vertical_remap.py:198-202 (values of MOM6 end_value_h4)
    u1 = P.remap_column([0, 1, 0, 0, 2, 3, 1], [5, 10, 11, 12, 13, 15, 16], np.ones(7), P.PPM_H4)
    np.testing.assert_allclose(u1, [10, 12.642, 13.358, 14.338, 15.052, 15.61, 16], atol=1e-3)


@pytest.mark.parametrize("scheme", [P.PCM, P.PLM, P.PPM_H4])
def test_identity_remap_and_conservation(scheme):
    # tests/test_vertical_remap.py:21-38
    rng = np.random.default_rng(0)
    h = rng.uniform(0.5, 3.0, 12)
    u = rng.normal(10, 2, 12)
    np.testing.assert_allclose(P.remap_column(h, u, h, scheme), u, rtol=1e-14)
    rng = np.random.default_rng(1)
    h0 = rng.uniform(0.0, 4.0, 20)
    h0[[3, 4, 11]] = 0.0
    u0 = rng.normal(15, 3, 20)
    h1 = rng.uniform(0.1, 2.0, 15)
    h1 *= h0.sum() / h1.sum()
    u1 = P.remap_column(h0, u0, h1, scheme)
    assert abs((h1 * u1).sum() - (h0 * u0).sum()) <= 1e-12 * abs((h0 * u0).sum())


def test_fully_vanished_column_keeps_its_values():
    # tests/test_vertical_remap.py:219-225
    for scheme in (P.PCM, P.PLM, P.PPM_H4):
        u0 = np.array([20.0, 21.0, 22.0, 23.0])
        np.testing.assert_array_equal(P.remap_column(np.zeros(4), u0, np.zeros(4), scheme), u0)
        np.testing.assert_allclose(P.remap_column(np.zeros(4), u0, np.zeros(2), scheme), 21.5)


def test_fct_pulse_stays_bounded_where_unlimited_overshoots():
    # tests/test_sigma_ale.py:1308-1325
    rec = FCT["pulse"]
    adv = _adv(rec)
    out = adv.advect_fct(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["ok"])
    assert out.min() >= -1e-12 and out.max() <= 1 + 1e-12
    un = adv.advect_fct(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["ok"], unlimited=True)
    assert un.max() > 1 + 1e-3


def _box_advection(w):
    adv = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=w.dt, ob=P.OpenEdges(()))
    adv.per = P.Periodic(w.periodic)
    return adv


@pytest.mark.parametrize("js", [False, True])
def test_constant_field_stays_constant(js):
    # tests/test_sigma_ale.py:1328-1339: C = 1 with V1 = V0 - dt div Q stays 1 (atol 1e-12), FCT and plain RK3
    from pyocean_b200 import workloads as W
    w = W.zstar_box(seed=3, nx=48, ny=40, n=6, nt=2)
    adv = _box_advection(w)
    adv.tracer_scheme = "weno5js" if js else "weno5"
    C = np.ones_like(w.C)
    out = adv.advect_fct(C, w.V0, w.V1, w.Qx, w.Qy, w.ok)
    np.testing.assert_allclose(out, 1.0, rtol=0, atol=1e-12)
    Fz = np.zeros((w.C.shape[1] + 1,) + w.C.shape[2:])
    out = adv.advect(C, w.V0, w.V1, w.Qx, w.Qy, Fz, w.ok)
    np.testing.assert_allclose(out, 1.0, rtol=0, atol=1e-12)


@pytest.mark.parametrize("scheme,time", [("upwind3", "ssprk3"), ("upwind1", "ssprk3"), ("weno5", "pc"),
                                         ("upwind3", "pc")])
def test_numpy_path_schemes_keep_a_constant_field_and_conserve(scheme, time):
    # the same identity for advect's NumPy-path schemes (tracers.py:110-151, 324-330), and tracer content
    # conservation (sum V1 c_new = sum V0 c on a periodic box, rtol 1e-12)
    from pyocean_b200 import workloads as W
    w = W.zstar_box(seed=3, nx=48, ny=40, n=6, nt=2)
    adv = _box_advection(w)
    adv.tracer_scheme, adv.tracer_time = scheme, time
    Fz = np.zeros((w.C.shape[1] + 1,) + w.C.shape[2:])
    out = adv.advect(np.ones_like(w.C), w.V0, w.V1, w.Qx, w.Qy, Fz, w.ok)
    np.testing.assert_allclose(out, 1.0, rtol=0, atol=1e-12)
    out = adv.advect(w.C, w.V0, w.V1, w.Qx, w.Qy, Fz, w.ok)
    for t in range(w.C.shape[0]):
        np.testing.assert_allclose((w.V1 * out[t]).sum(), (w.V0 * w.C[t]).sum(), rtol=1e-12)


def test_each_tracer_of_a_stack_stays_within_its_own_bounds_and_content():
    # tests/test_sigma_ale.py:1342-1360, 1375-1384: per-tracer bounds and conservation (rtol 1e-12) of a stack with
    # very different ranges, over 10 FCT steps of a periodic box
    from pyocean_b200 import workloads as W
    w = W.zstar_box(seed=4, nx=64, ny=48, n=5, nt=3)
    rng = np.random.default_rng(8)
    C = np.empty_like(w.C)
    C[0] = rng.uniform(0.0, 1.0, C[0].shape)                                    # passive in [0, 1]
    C[1] = 30.0 + 10.0 * (rng.random(C[1].shape) > 0.5)                         # a two-valued field in {30, 40}
    C[2] = 1e-3 * np.sin(np.arange(C.shape[-1]) / 3.0)[None, None]             # small signed values
    adv = _box_advection(w)
    lo, hi = C.reshape(3, -1).min(1), C.reshape(3, -1).max(1)
    c = C
    for _ in range(10):                         # each step takes the volumes V0 -> V1 = V0 - dt div Q
        c1 = adv.advect_fct(c, w.V0, w.V1, w.Qx, w.Qy, w.ok)
        np.testing.assert_allclose((c1 * w.V1[None]).reshape(3, -1).sum(1), (c * w.V0[None]).reshape(3, -1).sum(1),
                                   rtol=1e-12)
        for t in range(3):
            tol = 1e-12 * max(abs(lo[t]), abs(hi[t]))
            assert c1[t].min() >= lo[t] - tol and c1[t].max() <= hi[t] + tol, t
        c = c1
    assert np.all(np.isfinite(c))


# ---------------------------------------------------------------- larger seeded cases against the oracle
def _random_case(seed, nt, n, ny, nx, open_=(), periodic=(), inflow=False, land=0.1):
    rng = np.random.default_rng(seed)
    h = rng.uniform(1.0, 5.0, (n, ny, nx))
    active = rng.random((ny, nx)) > land
    V0 = 1e6 * h * active
    Qx = rng.uniform(-0.4, 0.4, (n, ny, nx + 1)) * 1e3 * np.concatenate([h[..., :1], h], -1)
    Qy = rng.uniform(-0.4, 0.4, (n, ny + 1, nx)) * 1e3 * np.concatenate([h[:, :1], h], 1)
    ax = np.zeros((ny, nx + 1), bool); ax[:, 1:-1] = active[:, 1:] & active[:, :-1]
    ay = np.zeros((ny + 1, nx), bool); ay[1:-1] = active[1:] & active[:-1]
    if "x" in periodic:
        ax[:, 0] = ax[:, -1] = active[:, 0] & active[:, -1]
    if "y" in periodic:
        ay[0] = ay[-1] = active[0] & active[-1]
    for e, sl in (("west", np.s_[:, 0]), ("east", np.s_[:, -1])):
        if e in open_:
            ax[sl] = active[:, 0 if e == "west" else -1]
    for e, sl in (("south", np.s_[0]), ("north", np.s_[-1])):
        if e in open_:
            ay[sl] = active[0 if e == "south" else -1]
    Qx *= ax
    Qy *= ay
    if "x" in periodic:
        Qx[..., -1] = Qx[..., 0]
    if "y" in periodic:
        Qy[:, -1] = Qy[:, 0]
    dt = 30.0
    V1 = V0 - dt * (Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:] - Qy[:, :-1])
    ok = active[None] & (V1 > 0)
    T = 7.0 + rng.normal(0, 1, (n, ny, nx))
    C = np.stack([T, T ** 2, rng.uniform(0, 1, T.shape)][:nt])
    infl = np.stack([np.full(T.shape, 9.0), np.full(T.shape, 81.0), np.full(T.shape, 0.5)][:nt]) if inflow else None
    return C, V0, V1, Qx, Qy, ok, dt, infl


CASES = [
    (1, 3, 5, 37, 70, ("west", "east", "south", "north"), (), True),
    (2, 2, 4, 33, 65, ("west",), (), False),
    (3, 2, 3, 29, 96, (), ("x",), False),
    (4, 1, 6, 40, 40, ("south",), ("x",), True),
    (5, 2, 3, 19, 23, (), ("x", "y"), False),
    (6, 3, 2, 9, 130, ("east", "north"), (), True),
]


@pytest.mark.parametrize("seed,nt,n,ny,nx,open_,per,inflow", CASES)
@pytest.mark.parametrize("scheme", ["weno5", "weno5js"])
def test_advect_fct_matches_oracle_on_ragged_tiles(seed, nt, n, ny, nx, open_, per, inflow, scheme):
    C, V0, V1, Qx, Qy, ok, dt, infl = _random_case(seed, nt, n, ny, nx, open_, per, inflow)
    ref = O.TracerAdvection(scheme=scheme, time="ssprk3", dt=dt, ob=O.OpenEdges(open_))
    ref.per = O.Periodic(per)
    gpu = P.TracerAdvection(scheme=scheme, time="ssprk3", dt=dt, ob=P.OpenEdges(open_))
    gpu.per = P.Periodic(per)
    fi = nx // 3
    r_out, r_fx = ref.advect_fct(C, V0, V1, Qx, Qy, ok, inflow=infl, flux_face_i=fi)
    g_out, g_fx = gpu.advect_fct(C, V0, V1, Qx, Qy, ok, inflow=infl, flux_face_i=fi)
    np.testing.assert_array_equal(g_out, r_out)
    np.testing.assert_array_equal(g_fx, r_fx)
    Fz = np.random.default_rng(seed).normal(size=(n + 1, ny, nx)) * 1e2
    Fz[0] = Fz[-1] = 0.0
    np.testing.assert_array_equal(gpu.advect(C, V0, V1, Qx, Qy, Fz, ok, inflow=infl),
                                  ref.advect(C, V0, V1, Qx, Qy, Fz, ok, inflow=infl))


@pytest.mark.parametrize("seed,nt,n,ny,nx,open_,per,inflow", CASES)
@pytest.mark.parametrize("scheme,time", [("upwind3", "ssprk3"), ("upwind1", "ssprk3"), ("weno5", "pc"),
                                         ("upwind3", "pc")])
def test_advect_numpy_path_schemes_match_oracle_on_ragged_tiles(seed, nt, n, ny, nx, open_, per, inflow, scheme,
                                                                 time):
    C, V0, V1, Qx, Qy, ok, dt, infl = _random_case(seed, nt, n, ny, nx, open_, per, inflow)
    ref = O.TracerAdvection(scheme=scheme, time=time, dt=dt, ob=O.OpenEdges(open_))
    ref.per = O.Periodic(per)
    gpu = P.TracerAdvection(scheme=scheme, time=time, dt=dt, ob=P.OpenEdges(open_))
    gpu.per = P.Periodic(per)
    Fz = np.random.default_rng(seed + 50).normal(size=(n + 1, ny, nx)) * 1e2
    Fz[0] = Fz[-1] = 0.0
    fi = nx // 3
    g_out, g_fx = gpu.advect(C, V0, V1, Qx, Qy, Fz, ok, inflow=infl, flux_face_i=fi)
    r_out, r_fx = ref.advect(C, V0, V1, Qx, Qy, Fz, ok, inflow=infl, flux_face_i=fi)
    np.testing.assert_array_equal(g_out, r_out)
    np.testing.assert_array_equal(g_fx, r_fx)


def test_torch_tensors_stay_on_the_device():
    C, V0, V1, Qx, Qy, ok, dt, _ = _random_case(9, 2, 4, 20, 30)
    gpu = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=dt)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()                  # noqa: E731
    out = gpu.advect_fct(t(C), t(V0), t(V1), t(Qx), t(Qy), t(ok))
    assert isinstance(out, torch.Tensor) and out.is_cuda
    np.testing.assert_array_equal(out.cpu().numpy(), gpu.advect_fct(C, V0, V1, Qx, Qy, ok))


# ---------------------------------------------------------------- full size (512 x 512 x 50, T and S)
@pytest.fixture(scope="module")
def basin():
    from pyocean_b200 import workloads as W
    return W.basin(seed=1)


def test_full_size_step_conserves_and_matches_oracle(basin):
    w = basin
    gpu = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=w.dt)
    A = gpu.advect_fct(w.C, w.V0, w.V1, w.Qx, w.Qy, w.ok)
    ref = O.TracerAdvection(scheme="weno5", time="ssprk3", dt=w.dt)
    np.testing.assert_array_equal(A, ref.advect_fct(w.C, w.V0, w.V1, w.Qx, w.Qy, w.ok))
    # closed basin: content V1 c_new equals V0 c_old to round-off, per tracer
    for m in range(A.shape[0]):
        before = (w.V0 * w.C[m]).sum()
        after = (w.V1 * A[m]).sum()
        assert abs(after - before) <= 1e-12 * abs(before)
    # no new extrema (FCT bounds)
    wetc = w.ok
    for m in range(A.shape[0]):
        assert A[m][wetc].min() >= w.C[m][wetc].min() - 1e-12 * abs(w.C[m][wetc].min())
        assert A[m][wetc].max() <= w.C[m][wetc].max() * (1 + 1e-12)
    R = P.remap_columns(w.h_src, A, w.h_tgt, P.PPM_H4, w.wet)
    for m in range(A.shape[0]):
        np.testing.assert_array_equal(R[m], O.remap_columns(w.h_src, A[m], w.h_tgt, O.PPM_H4, w.wet))
        cin = (w.h_src * A[m]).sum(0)[w.wet]
        cout = (w.h_tgt * R[m]).sum(0)[w.wet]
        assert np.all(np.abs(cout - cin) <= 1e-12 * np.abs(cin) + 1e-9)


def _oracle_steps(w, steps):
    """``steps`` ALE tracer steps (advect_fct, then the remap of every tracer) with the oracle."""
    adv = O.TracerAdvection(scheme=w.scheme, time="ssprk3", dt=w.dt, ob=O.OpenEdges(w.open))
    adv.per = O.Periodic(w.periodic)
    C = w.C
    for _ in range(steps):
        A = adv.advect_fct(C, w.V0, w.V1, w.Qx, w.Qy, w.ok)
        C = np.stack([O.remap_columns(w.h_src, A[m], w.h_tgt, w.remap_scheme, w.wet) for m in range(A.shape[0])])
    return C


def _gpu_steps(w, steps):
    from pyocean_b200 import _lib
    from pyocean_b200.step import ALETracerStep
    dev = torch.device("cuda", 0)
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                      # noqa: E731
    nt, n, ny, nx = w.C.shape
    flags = (_lib.PERIODIC_X if "x" in w.periodic else 0) | (_lib.PERIODIC_Y if "y" in w.periodic else 0)
    st = ALETracerStep(nt, n, ny, nx, w.dt, flags, w.remap_scheme, device=dev)
    V0, V1, Qx, Qy = g(w.V0), g(w.V1), g(w.Qx), g(w.Qy)
    ok, wet, hs, ht = g(w.ok.astype(np.uint8)), g(w.wet.astype(np.uint8)), g(w.h_src), g(w.h_tgt)
    c, nxt = g(w.C), torch.empty((nt, n, ny, nx), dtype=torch.float64, device=dev)
    for _ in range(steps):
        st.step(c, V0, V1, Qx, Qy, ok, hs, ht, wet, nxt)
        c, nxt = nxt, c
    return c.cpu().numpy()


def test_zstar_box_100_steps_bitwise():
    # the 64 x 64 x 20 z* box, periodic in x: 100 steps of advect_fct + PPM_H4 remap, equal to the oracle
    from pyocean_b200 import workloads as W
    w = W.zstar_box(seed=0)
    np.testing.assert_array_equal(_gpu_steps(w, 100), _oracle_steps(w, 100))


def test_basin_five_full_size_steps_bitwise():
    # the 512 x 512 x 50 basin (T and S): five steps, equal to the oracle
    from pyocean_b200 import workloads as W
    w = W.basin(seed=3)
    np.testing.assert_array_equal(_gpu_steps(w, 5), _oracle_steps(w, 5))


@pytest.mark.parametrize("nt,n,ny,nx", [(1, 1, 1, 1), (2, 1, 1, 5), (1, 3, 5, 1), (2, 2, 2, 3), (1, 6, 1, 1)])
@pytest.mark.parametrize("scheme,time", [("weno5", "ssprk3"), ("weno5js", "ssprk3"), ("upwind3", "ssprk3"),
                                         ("upwind1", "ssprk3"), ("weno5", "pc"), ("upwind3", "pc")])
def test_degenerate_shapes_match_the_oracle(nt, n, ny, nx, scheme, time):
    # single cells, single rows and columns, single layers: every stencil reaches out of the domain
    rng = np.random.default_rng(nt * 1000 + n * 100 + ny * 10 + nx)
    open_ = ("west", "east", "south", "north")
    h = rng.uniform(1.0, 5.0, (n, ny, nx))
    V0 = 1e6 * h
    Qx = rng.uniform(-0.3, 0.3, (n, ny, nx + 1)) * 1e3
    Qy = rng.uniform(-0.3, 0.3, (n, ny + 1, nx)) * 1e3
    V1 = V0 - 10.0 * (Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:] - Qy[:, :-1])
    ok = V1 > 0
    C = rng.normal(10.0, 1.0, (nt, n, ny, nx))
    infl = rng.normal(11.0, 1.0, C.shape)
    Fz = rng.normal(size=(n + 1, ny, nx)) * 1e2
    Fz[0] = Fz[-1] = 0.0
    ref = O.TracerAdvection(scheme=scheme, time=time, dt=10.0, ob=O.OpenEdges(open_))
    gpu = P.TracerAdvection(scheme=scheme, time=time, dt=10.0, ob=P.OpenEdges(open_))
    np.testing.assert_array_equal(gpu.advect(C, V0, V1, Qx, Qy, Fz, ok, inflow=infl),
                                  ref.advect(C, V0, V1, Qx, Qy, Fz, ok, inflow=infl))
    np.testing.assert_array_equal(gpu.rhs(C, Qx, Qy, Fz, ok, inflow=infl), ref.rhs(C, Qx, Qy, Fz, ok, inflow=infl))
    np.testing.assert_array_equal(gpu.flux_x(C, Qx, Qy, ok, centred=True, inflow=infl),
                                  ref.flux_x(C, Qx, Qy, ok, centred=True, inflow=infl))
    if time == "ssprk3":
        np.testing.assert_array_equal(gpu.advect_fct(C, V0, V1, Qx, Qy, ok, inflow=infl),
                                      ref.advect_fct(C, V0, V1, Qx, Qy, ok, inflow=infl))
        for a, b in zip(gpu.upwind_faces_h(C, Qx, Qy, inflow=infl), ref.upwind_faces_h(C, Qx, Qy, inflow=infl)):
            np.testing.assert_array_equal(a, b)
    for scheme_r in (P.PCM, P.PLM, P.PPM_H4):
        h_tgt = rng.uniform(0.5, 2.0, (n, ny, nx))
        h_tgt *= h.sum(0) / h_tgt.sum(0)
        wet = np.ones((ny, nx), bool)
        np.testing.assert_array_equal(P.remap_columns(h, C[0], h_tgt, scheme_r, wet),
                                      O.remap_columns(h, C[0], h_tgt, scheme_r, wet))
        np.testing.assert_array_equal(P.reconstruct(h, C[0], scheme_r)[:, 0, 0],
                                      O.reconstruct(h[:, 0, 0], C[0][:, 0, 0], scheme_r))
