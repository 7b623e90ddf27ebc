"""The Lagrangian layer-transport step on the GPU: the donor-cell layer flux, the freshwater volumes, the
Lagrangian thickness at a signed-zero tie and the whole ``ALELayerTransport`` step (PPM and donor-cell fluxes,
freshwater, periodic x, the PPM flux on periodic x and x+y axes, open edges, limited flows) — bit for bit against
the reference's golden vectors and the oracle."""
from __future__ import annotations

from types import SimpleNamespace as NS

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import oracle as O
from pyocean_b200 import producers as P
from pyocean_b200 import workloads as W

pytestmark = pytest.mark.gpu
LT = load_golden("layer_transport")
LT.update(load_golden("layer_transport_ext"))
LT_CASES = ["lt_ppm", "lt_upwind", "lt_ppm_fw", "lt_upwind_perx", "lt_ppm_strong", "lt_upwind_strong",
            "lt_ppm_perx", "lt_ppm_perxy", "lt_ppm_open", "lt_upwind_open", "lt_ppm_perx_open_sn"]


@pytest.mark.parametrize("case", ["upwind", "upwind_empty"])
def test_upwind_transport_matches_reference_bitwise(case):
    rec = LT[case]
    np.testing.assert_array_equal(P.upwind_transport_x(rec["q_e"], rec["q_w"], rec["ut"], rec["L"], rec["Q_bt"]),
                                  rec["Q"])


@pytest.mark.parametrize("case", ["fw_thickness", "fw_volume"])
def test_freshwater_volumes_match_reference_bitwise(case):
    rec = LT[case]
    V, nl = P.freshwater_volumes(rec["V"], rec["dV"], rec["floor"])
    np.testing.assert_array_equal(V, rec["V_new"])
    assert nl == int(rec["n_limited"]) > 0
    if case == "fw_thickness":                              # the scalar floor of the ALE call
        V2, nl2 = P.freshwater_volumes(rec["V"], rec["dV"], float(rec["floor"][0, 0]))
        np.testing.assert_array_equal(V2, rec["V_new"])
        assert nl2 == nl


def test_lagrangian_thickness_signed_zero_matches_reference():
    rec = LT["lagrangian_negzero"]
    out = P.lagrangian_thickness(rec["h"], rec["divq"], float(rec["dt"]), rec["area"])
    np.testing.assert_array_equal(out, rec["h_dag"])
    assert not np.signbit(out).any()


def _call(rec, device=None):
    """ALELayerTransport (the GPU mirror) on a golden case; ``device``: CUDA tensors in, tensors out."""
    per = tuple(str(a) for a in rec["periodic"])
    g = (lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)) if device else (lambda a: a)   # noqa: E731
    fs = NS(theta=float(rec["theta"]), active=rec["active"], Lu=rec["Lu"], Lv=rec["Lv"])
    lt = P.ALELayerTransport(fs=fs, H=rec["H"], area=rec["area"], dt=float(rec["dt"]),
                             thickness_flux=str(rec["thickness_flux"]),
                             vi_geom={"dx_t": rec["dx_t"], "dy_t": rec["dy_t"]})
    if per:
        lt.per = NS(x="x" in per, y="y" in per)
    st = NS(h=g(rec["h"]), u=g(rec["u"]), v=g(rec["v"]), eta=rec["eta"])
    fluxes = NS(wet_u=rec["wet_u"], wet_v=rec["wet_v"], Du=rec["Du"], Dv=rec["Dv"],
                fw=g(rec["fw"]) if "fw" in rec else None)
    open_ = tuple(str(e) for e in rec["open"]) if "open" in rec else ()
    if open_:
        lt.ob = NS(open=open_, theta_bc=float(rec["theta_bc"]))
        fluxes.open_Du, fluxes.open_Dv = g(rec["open_Du"]), g(rec["open_Dv"])
        fluxes.open_Qu, fluxes.open_Qv = g(rec["open_Qu"]), g(rec["open_Qv"])
    return lt(st, rec["eta_new"], g(rec["u_new"]), g(rec["v_new"]), fluxes, float(rec["theta_bc"]), open_,
              g(rec["wu"]), g(rec["wv"]), g(rec["qe"]), g(rec["qw"]), g(rec["qn"]), g(rec["qs"]))


def _keys(rec):
    return ("Qx", "Qy", "V0", "V1", "ok", "h_dagger") + (("h_fw", "V_fw") if "fw" in rec else ())


def _field(lf, key):
    return {"h_dagger": lf.h_dagger}.get(key, getattr(lf, key, None))


@pytest.mark.parametrize("case", LT_CASES)
def test_layer_transport_step_matches_reference_bitwise(case):
    rec = LT[case]
    lf = _call(rec)
    for key in _keys(rec):
        np.testing.assert_array_equal(_field(lf, key), rec[key], err_msg=key)
    assert lf.n_limited == int(rec["n_limited"])
    assert not np.asarray(lf.Fz).any() and np.asarray(lf.Fz).shape == (rec["h"].shape[0] + 1,) + rec["h"].shape[1:]


@pytest.mark.parametrize("case", ["lt_ppm_fw", "lt_upwind_strong"])
def test_layer_transport_step_on_device_tensors(case):
    rec = LT[case]
    lf = _call(rec, torch.device("cuda", 0))
    assert isinstance(lf.Qx, torch.Tensor) and lf.Qx.is_cuda
    for key in _keys(rec):
        np.testing.assert_array_equal(_field(lf, key).cpu().numpy(), rec[key], err_msg=key)


@pytest.mark.parametrize("case", ["lt_ppm_perxy", "lt_ppm_open"])
def test_layer_transport_periodic_and_open_on_device_tensors(case):
    rec = LT[case]
    lf = _call(rec, torch.device("cuda", 0))
    for key in _keys(rec):
        np.testing.assert_array_equal(_field(lf, key).cpu().numpy(), rec[key], err_msg=key)


def test_layer_transport_argument_errors():
    rec = LT["lt_ppm"]
    fs = NS(theta=0.6, active=rec["active"], Lu=rec["Lu"], Lv=rec["Lv"])
    lt = P.ALELayerTransport(fs=fs, H=rec["H"], area=rec["area"], dt=600.0, thickness_flux="ppm",
                             vi_geom={"dx_t": rec["dx_t"], "dy_t": rec["dy_t"]})
    st = NS(h=rec["h"], u=rec["u"], v=rec["v"], eta=rec["eta"])
    fl = NS(wet_u=rec["wet_u"], wet_v=rec["wet_v"], Du=rec["Du"], Dv=rec["Dv"], fw=None,
            open_Du=rec["Du"], open_Dv=rec["Dv"], open_Qu=rec["Du"], open_Qv=rec["Dv"])
    args = (rec["wu"], rec["wv"], rec["qe"], rec["qw"], rec["qn"], rec["qs"])
    with pytest.raises(ValueError, match="open-boundary"):             # open edges need the open-boundary object
        lt(st, rec["eta_new"], rec["u_new"], rec["v_new"], fl, 0.5, ("west",), *args)
    with pytest.raises(ValueError, match="thickness_flux"):
        P.ALELayerTransport(fs=fs, H=rec["H"], area=rec["area"], dt=600.0, thickness_flux="pcm", vi_geom={})


@pytest.mark.parametrize("flux", ["ppm", "upwind"])
def test_full_size_layer_transport_against_oracle(flux):
    # the basin's layers (256 x 192 x 30) with a smooth flow and freshwater
    w = W.basin(seed=6, nx=256, ny=192, n=30)
    rng = np.random.default_rng(5)
    n, ny, nx = w.h_src.shape
    act = w.wet
    h = np.where(act[None], w.h_src, 0.0)
    H = h.sum(0)
    area = rng.uniform(3.6e6, 4.4e6, (ny, nx))
    Lu, Lv = rng.uniform(1900.0, 2100.0, (ny, nx + 1)), rng.uniform(1900.0, 2100.0, (ny + 1, nx))
    dx, dy = rng.uniform(1900.0, 2100.0, (ny, nx)), rng.uniform(1900.0, 2100.0, (ny, nx))
    wet_u = np.zeros((ny, nx + 1), bool)
    wet_u[:, 1:-1] = act[:, 1:] & act[:, :-1]
    wet_v = np.zeros((ny + 1, nx), bool)
    wet_v[1:-1] = act[1:] & act[:-1]
    Du = np.zeros((ny, nx + 1))
    Du[:, 1:-1] = np.minimum(H[:, 1:], H[:, :-1])
    Dv = np.zeros((ny + 1, nx))
    Dv[1:-1] = np.minimum(H[1:], H[:-1])
    u_old, u_new = (rng.normal(0.0, 0.2, (n, ny, nx + 1)) * wet_u for _ in range(2))
    v_old, v_new = (rng.normal(0.0, 0.2, (n, ny + 1, nx)) * wet_v for _ in range(2))
    qe, qw = O.face_transport_thickness(h, H, act, True)
    qn, qs = O.face_transport_thickness(np.ascontiguousarray(h.swapaxes(1, 2)), H.T, act.T, True)
    wu = O.face_fractions(0.5 * (qe + qw))
    wv = np.ascontiguousarray(O.face_fractions(0.5 * (qn + qs)).swapaxes(1, 2))
    fw = rng.normal(0.0, 1.0, (ny, nx)) * 1e-6
    dt = 300.0
    ref = O.ale_layer_transport(h, u_old, v_old, u_new, v_new, wet_u, wet_v, wu, wv, Lu, Lv, Du, Dv, qe, qw, qn, qs,
                                act, area, dx, dy, dt, 0.6, 0.5, flux, (False, False), fw)
    fs = NS(theta=0.6, active=act, Lu=Lu, Lv=Lv)
    lt = P.ALELayerTransport(fs=fs, H=H, area=area, dt=dt, thickness_flux=flux, vi_geom={"dx_t": dx, "dy_t": dy})
    lf = lt(NS(h=h, u=u_old, v=v_old, eta=np.zeros((ny, nx))), np.zeros((ny, nx)), u_new, v_new,
            NS(wet_u=wet_u, wet_v=wet_v, Du=Du, Dv=Dv, fw=fw), 0.5, (), wu, wv, qe, qw, qn, qs)
    for key in ("Qx", "Qy", "V0", "V1", "ok", "h_fw", "V_fw"):
        np.testing.assert_array_equal(getattr(lf, key), ref[key], err_msg=key)
    np.testing.assert_array_equal(lf.h_dagger, ref["h_dagger"])
    assert lf.n_limited == ref["n_limited"]
