"""
Known-answer tests of the FCT step ported from the reference's own suite (tests/test_sigma_ale.py), re-expressed
without the model: a one-row z* box (dx = dy = 1 km, 30 s step, 10 m layers) with the reference's transports,
volumes and masks fed directly.  Each case also equals the CPU oracle bit for bit.

* tests/test_sigma_ale.py:1328-1339 — FCT with unit coefficients (unlimited) is the plain SSP-RK3 result (atol 1e-12);
* tests/test_sigma_ale.py:1342-1360 — FCT conserves (rtol 1e-12) and keeps high order on a smooth profile: its error
  against the exact half-cell shift is at most 1.5 x the unlimited scheme's;
* tests/test_sigma_ale.py:1363-1372 — a 1 mm cell receiving water of other values stays within their range.
* tests/test_components_tracers.py:12-27 — the values entering an open edge are the inflow argument's.
"""
from __future__ import annotations

import numpy as np
import pytest

import pyocean_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DX, DT, H = 1000.0, 30.0, 10.0


def _box(nx, nz=4, h=None):
    """Thicknesses (nz, 1, nx), volumes, zero transports and the reference's ok rule of a one-row box."""
    h = np.full((nz, 1, nx), H) if h is None else h
    V = h * DX * DX
    Qx = np.zeros((nz, 1, nx + 1))
    Qy = np.zeros((nz, 2, nx))
    return h, V, Qx, Qy


def _close(V, Qx, Qy):
    V1 = V - DT * (Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:] - Qy[:, :-1])
    return V1, V1 > 0


def _pair():
    gpu = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=DT, ob=P.OpenEdges(()))
    gpu.per = P.Periodic(())
    ref = O.TracerAdvection(scheme="weno5", time="ssprk3", dt=DT)
    ref.per = O.Periodic(())
    return gpu, ref


def test_fct_with_unit_coefficients_is_the_rk3_result():
    nx = 40
    h, V, Qx, Qy = _box(nx)
    rng = np.random.default_rng(0)
    Qx[:, :, 1:-1] = rng.uniform(-0.3, 0.3, Qx[:, :, 1:-1].shape) * DX * h[:, :, 1:]
    V1, ok = _close(V, Qx, Qy)
    T = (np.sin(np.arange(nx) / 5.0)[None, None, None, :] + 2.0) * np.ones((1,) + V.shape)
    Fz = np.zeros((V.shape[0] + 1, 1, nx))
    gpu, ref = _pair()
    rk3 = gpu.advect(T, V, V1, Qx, Qy, Fz, ok)
    un = gpu.advect_fct(T, V, V1, Qx, Qy, ok, unlimited=True)
    np.testing.assert_allclose(un, rk3, rtol=0, atol=1e-12)
    np.testing.assert_array_equal(rk3, ref.advect(T, V, V1, Qx, Qy, Fz, ok))
    np.testing.assert_array_equal(un, ref.advect_fct(T, V, V1, Qx, Qy, ok, unlimited=True))


def test_fct_conserves_and_keeps_high_order_on_a_smooth_profile():
    nx = 80
    h, V, Qx, Qy = _box(nx)
    x = np.arange(nx)
    T0 = (1.0 + 0.5 * np.sin(2 * np.pi * x / nx))[None, None, None, :].repeat(V.shape[0], 1)
    Qx[:, :, 1:-1] = 0.5 * DX / DT * h[:, :, 1:] * DX                       # Courant 0.5 eastwards
    Qx[:, :, -1] = 0.0
    Qx[:, :, 1] = 0.0
    V1, ok = _close(V, Qx, Qy)
    Fz = np.zeros((V.shape[0] + 1, 1, nx))
    gpu, ref = _pair()
    exact = 1.0 + 0.5 * np.sin(2 * np.pi * (x - 0.5) / nx)                  # shifted by half a cell
    errs = {}
    for limiter in ("fct", "none"):
        if limiter == "fct":
            out = gpu.advect_fct(T0, V, V1, Qx, Qy, ok)
            np.testing.assert_array_equal(out, ref.advect_fct(T0, V, V1, Qx, Qy, ok))
        else:
            out = gpu.advect(T0, V, V1, Qx, Qy, Fz, ok)
            np.testing.assert_array_equal(out, ref.advect(T0, V, V1, Qx, Qy, Fz, ok))
        np.testing.assert_allclose((V1 * out[0]).sum(), (V * T0[0]).sum(), rtol=1e-12)
        errs[limiter] = np.abs(out[0, 0, 0, 5:-5] - exact[5:-5]).max()
    assert errs["fct"] <= 1.5 * errs["none"], errs


def test_fct_bounds_a_thin_layer_receiving_other_water():
    nx = 20
    h = np.full((4, 1, nx), H)
    h[1, 0, 10] = 1e-3                                                      # a 1 mm cell in layer 1
    h, V, Qx, Qy = _box(nx, h=h)
    T = np.ones((1,) + V.shape)
    T[0, 1, 0, 10] = 0.0
    T[0, 1, 0, :10] = 5.0
    Qx[1, 0, 10] = 2.0                                                      # inflow 2 m3/s, outflow 1 m3/s
    Qx[1, 0, 11] = 1.0
    V1, ok = _close(V, Qx, Qy)
    gpu, ref = _pair()
    out = gpu.advect_fct(T, V, V1, Qx, Qy, ok)
    np.testing.assert_array_equal(out, ref.advect_fct(T, V, V1, Qx, Qy, ok))
    assert 0.0 - 1e-12 <= out[0, 1, 0, 10] <= 5.0 + 1e-12


def test_inflow_is_an_explicit_argument():
    # tests/test_components_tracers.py:12-27: the values entering through an open edge come from the inflow argument
    # only; another inflow changes the west-edge cells, the same inflow gives the same result
    nx, ny, nz = 16, 4, 3
    rng = np.random.default_rng(12)
    h = rng.uniform(5.0, 15.0, (nz, ny, nx))
    V = h * DX * DX
    hf = np.concatenate([h[..., :1], h], axis=-1)
    Qx = rng.uniform(0.05, 0.3, (nz, ny, nx + 1)) * DX * hf                  # eastward: inflow on the west edge
    Qy = np.zeros((nz, ny + 1, nx))
    Qy[:, 1:-1] = rng.uniform(-0.1, 0.1, (nz, ny - 1, nx)) * DX * h[:, 1:]
    V1, ok = _close(V, Qx, Qy)
    T = rng.normal(12.0, 2.0, (nz, ny, nx))
    stack = np.stack([T, T ** 2])
    gpu = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=DT, ob=P.OpenEdges(("west", "east")))
    gpu.per = P.Periodic(())
    ref = O.TracerAdvection(scheme="weno5", time="ssprk3", dt=DT, ob=O.OpenEdges(("west", "east")))
    ref.per = O.Periodic(())
    T_in = np.full(T.shape, 30.0)
    a = gpu.advect_fct(stack, V, V1, Qx, Qy, ok, inflow=np.stack([T_in, T_in ** 2]))
    b = gpu.advect_fct(stack, V, V1, Qx, Qy, ok, inflow=np.stack([T_in - 10, (T_in - 10) ** 2]))
    diff = np.any(a != b, axis=(0, 1))
    assert diff.any() and diff[:, 0].all()
    c = gpu.advect_fct(stack, V, V1, Qx, Qy, ok, inflow=np.stack([T_in, T_in ** 2]))
    np.testing.assert_array_equal(a, c)
    np.testing.assert_array_equal(a, ref.advect_fct(stack, V, V1, Qx, Qy, ok, inflow=np.stack([T_in, T_in ** 2])))
