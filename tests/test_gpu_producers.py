"""The producers of the step's inputs on the GPU, bit for bit against the reference's golden vectors and the
oracle: face transport thickness, transport velocity, PPM edges and transport, outflow limiter, Lagrangian
thickness."""
from __future__ import annotations

import warnings

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import oracle as O
from pyocean_b200 import producers as P

pytestmark = pytest.mark.gpu
PR = load_golden("producers")


@pytest.mark.parametrize("case", ["ftt_clip", "ftt_noclip"])
def test_face_transport_thickness(case):
    rec = PR[case]
    q_e, q_w = P.face_transport_thickness(rec["h"], rec["H"], rec["active"], bool(rec["clip"]))
    np.testing.assert_array_equal(q_e, rec["q_e"])
    np.testing.assert_array_equal(q_w, rec["q_w"])


def test_transport_velocity():
    rec = PR["tvel"]
    ut, Qb = P.transport_velocity(rec["u_new"], rec["u_old"], rec["last_wet"], rec["w"], rec["L"], rec["D"],
                                  float(rec["theta"]), float(rec["theta_bc"]))
    np.testing.assert_array_equal(ut, rec["ut"])
    np.testing.assert_array_equal(Qb, rec["Qb"])
    with pytest.raises(ValueError, match="transport_velocity: shapes"):
        P.transport_velocity(rec["u_new"], rec["u_old"][:-1], rec["last_wet"], rec["w"], rec["L"], rec["D"], 0.6)


def test_ppm_edges():
    rec = PR["ppm_edges"]
    h_w, h_e = P.ppm_edges_x(rec["h"], rec["active"])
    np.testing.assert_array_equal(h_w, rec["h_w"])
    np.testing.assert_array_equal(h_e, rec["h_e"])


@pytest.mark.parametrize("case", ["ppm_transport_it20", "ppm_transport_it1"])
def test_ppm_transport(case):
    rec = PR[case]
    out = P.ppm_transport_x(rec["h"], rec["ut"], rec["L"], rec["Q_bt"], rec["q_e"], rec["q_w"], rec["active"],
                            float(rec["dt"]), rec["dx"], int(rec["max_iter"]))
    np.testing.assert_array_equal(out, rec["Qx"])


@pytest.mark.parametrize("case", sorted(c for c in PR if c.startswith("limit_")))
def test_limit_outflow(case):
    rec = PR[case]
    args = (rec["h"], rec["Qx"], rec["Qy"], rec["area"], float(rec["dt"]), rec["active"])
    per = tuple(bool(x) for x in rec["periodic"])
    if str(rec["status"]) == "raised":
        with pytest.raises(RuntimeError):
            P.limit_outflow(*args, periodic=per)
        return
    Qx, Qy, nl = P.limit_outflow(*args, periodic=per)
    assert nl == int(rec["n_limited"])
    np.testing.assert_array_equal(Qx, rec["Qx_out"])
    np.testing.assert_array_equal(Qy, rec["Qy_out"])
    if nl == 0:
        assert Qx is rec["Qx"] and Qy is rec["Qy"]                 # the inputs themselves, as the reference


@pytest.mark.parametrize("case", ["lagrangian_calm", "lagrangian_limited", "lagrangian_strong"])
def test_lagrangian_thickness(case):
    rec = PR[case]
    args = (rec["h"], rec["divq"], float(rec["dt"]), rec["area"])
    if bool(rec["raises"]):
        with pytest.raises(RuntimeError, match="emptied in the Lagrangian step"):
            P.lagrangian_thickness(*args)
        return
    np.testing.assert_array_equal(P.lagrangian_thickness(*args), rec["h_dag"])


def _state(seed, n, ny, nx):
    rng = np.random.default_rng(seed)
    H = rng.uniform(20.0, 400.0, (ny, nx))
    active = rng.random((ny, nx)) > 0.1
    h = np.stack([H / n * rng.uniform(0.5, 1.5, (ny, nx)) for _ in range(n)])
    h[0, :, : nx // 5] = 0.0
    h = np.where(active[None], h, np.nan)
    dx = rng.uniform(1800.0, 2200.0, (ny, nx))
    return rng, H, active, h, dx


def test_larger_chain_against_oracle_both_axes():
    # face thickness -> transport velocity -> PPM transport (x, and y on swapped axes as the reference calls it) ->
    # outflow limiter -> Lagrangian thickness, all on device tensors, against the oracle
    n, ny, nx = 20, 96, 128
    rng, H, active, h, dx = _state(7, n, ny, nx)
    dev = torch.device("cuda", 0)
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                    # noqa: E731
    dt = 300.0
    res = {}
    for axis in ("x", "y"):
        sw = (lambda a: a) if axis == "x" else (lambda a: np.swapaxes(a, -1, -2))      # noqa: E731
        hs, Hs, acts, dxs = sw(h), sw(H), sw(active), sw(dx)
        nb_, na_ = hs.shape[1], hs.shape[2]
        q_e, q_w = P.face_transport_thickness(g(hs), g(Hs), g(acts.astype(np.uint8)), True)
        oq_e, oq_w = O.face_transport_thickness(hs, Hs, acts, True)
        assert np.array_equal(q_e.cpu().numpy(), oq_e) and np.array_equal(q_w.cpu().numpy(), oq_w)
        w = O.face_fractions(0.5 * (oq_e + oq_w))
        u1 = rng.normal(0, 0.5, (n, nb_, na_ + 1))
        u0 = rng.normal(0, 0.5, (n, nb_, na_ + 1))
        lw = rng.random((nb_, na_ + 1)) > 0.1
        Lf = rng.uniform(1800.0, 2200.0, (nb_, na_ + 1))
        D = rng.uniform(20.0, 400.0, (nb_, na_ + 1))
        ut, Qb = P.transport_velocity(g(u1), g(u0), g(lw.astype(np.uint8)), g(w), g(Lf), g(D), 0.6, 0.5)
        out_, oQb = O.transport_velocity(u1, u0, lw, w, Lf, D, 0.6, 0.5)
        assert np.array_equal(ut.cpu().numpy(), out_) and np.array_equal(Qb.cpu().numpy(), oQb)
        Q_bt = oQb * rng.uniform(0.9, 1.1, oQb.shape)
        Q = P.ppm_transport_x(g(hs), ut, g(Lf), g(Q_bt), q_e, q_w, g(acts.astype(np.uint8)), dt, g(dxs))
        oQ = O.ppm_transport_x(hs, out_, Lf, Q_bt, oq_e, oq_w, acts, dt, dxs)
        np.testing.assert_array_equal(Q.cpu().numpy(), oQ)
        res[axis] = oQ if axis == "x" else np.swapaxes(oQ, -1, -2)
    hz = np.where(active[None], np.nan_to_num(h), 0.0)
    area = dx * 2000.0
    Qx, Qy = res["x"] * 4.0, res["y"] * 4.0                       # strong enough to need limiting somewhere
    try:
        oQx, oQy, onl = O.limit_outflow(hz, Qx, Qy, area, dt, active)
        status = "ok"
    except RuntimeError:
        status = "raised"
    if status == "raised":
        with pytest.raises(RuntimeError):
            P.limit_outflow(g(hz), g(Qx), g(Qy), g(area), dt, g(active.astype(np.uint8)))
        return
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        gQx, gQy, nl = P.limit_outflow(g(hz), g(Qx), g(Qy), g(area), dt, g(active.astype(np.uint8)))
    assert nl == onl
    np.testing.assert_array_equal(gQx.cpu().numpy(), oQx)
    np.testing.assert_array_equal(gQy.cpu().numpy(), oQy)
    div = oQx[..., 1:] - oQx[..., :-1] + oQy[:, 1:] - oQy[:, :-1]
    A = np.where(active, area, 0.0)
    try:
        ref = O.lagrangian_thickness(hz, div, dt, A)
    except RuntimeError:
        with pytest.raises(RuntimeError):
            P.lagrangian_thickness(g(hz), g(div), dt, g(A))
        return
    np.testing.assert_array_equal(P.lagrangian_thickness(g(hz), g(div), dt, g(A)).cpu().numpy(), ref)
