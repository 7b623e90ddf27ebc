"""
The reference's remap known-answer tests (tests/test_vertical_remap.py), run through the GPU remap
(`pyocean_b200.remap_column` / `remap_columns`) with the reference's inputs and tolerances; every result also equals
the CPU oracle's bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import pyocean_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SCHEMES = [P.PCM, P.PLM, P.PPM_H4]


def _remap(h0, u0, h1, scheme):
    h0, u0, h1 = (np.asarray(a, float) for a in (h0, u0, h1))
    got = P.remap_column(h0, u0, h1, scheme)
    np.testing.assert_array_equal(got, O.remap_column(h0, u0, h1, scheme))
    return got


@pytest.mark.parametrize("scheme", SCHEMES)
def test_identity_when_grid_unchanged(scheme):                      # :21-26
    rng = np.random.default_rng(0)
    h = rng.uniform(0.5, 3.0, 12)
    u = rng.normal(10, 2, 12)
    np.testing.assert_allclose(_remap(h, u, h, scheme), u, rtol=1e-14)


@pytest.mark.parametrize("scheme", SCHEMES)
def test_conservation_to_roundoff(scheme):                          # :29-38
    rng = np.random.default_rng(1)
    h0 = rng.uniform(0.0, 4.0, 20)
    h0[[3, 4, 11]] = 0.0
    u0 = rng.normal(15, 3, 20)
    h1 = rng.uniform(0.1, 2.0, 15)
    h1 *= h0.sum() / h1.sum()
    u1 = _remap(h0, u0, h1, scheme)
    assert abs((h1 * u1).sum() - (h0 * u0).sum()) <= 1e-12 * abs((h0 * u0).sum())


def test_pcm_piecewise_constant_values():                           # :41-44
    np.testing.assert_allclose(_remap([1, 1], [1.0, 3.0], [2.0], P.PCM), [2.0])
    np.testing.assert_allclose(_remap([1, 1], [1.0, 3.0], [0.5, 1.5], P.PCM), [1.0, (0.5 + 3.0) / 1.5])


def test_vanished_target_takes_local_value():                       # :47-51
    u1 = _remap([1.0, 1.0], [1.0, 3.0], [1.0, 0.0, 1.0], P.PCM)
    assert np.isfinite(u1).all()
    np.testing.assert_allclose(u1[[0, 2]], [1.0, 3.0])
    assert 1.0 <= u1[1] <= 3.0


def test_roundoff_mismatch_in_total_thickness():                    # :54-60
    h0, u0 = np.array([1.0, 2.0, 3.0]), np.array([4.0, 5.0, 6.0])
    h1 = np.array([3.0, 3.0 + 1e-13])
    u1 = _remap(h0, u0, h1, P.PCM)
    assert np.all((u1 >= 4.0 - 1e-12) & (u1 <= 6.0 + 1e-12))
    assert abs((h1 * u1).sum() - (h0 * u0).sum()) < 1e-11


def test_source_thicker_than_target_last_target_absorbs():          # :63-70
    h0, u0 = np.array([1.0, 2.0, 3.0 + 1e-9]), np.array([4.0, 5.0, 6.0])
    h1 = np.array([3.0, 3.0])
    u1 = _remap(h0, u0, h1, P.PCM)
    assert abs((h1 * u1).sum() - (h0 * u0).sum()) < 1e-12


@pytest.mark.parametrize("scheme", [P.PCM, P.PPM_H4])
def test_target_thicker_than_source_adds_no_content(scheme):        # :73-80
    h0, u0 = np.array([1.0, 2.0, 3.0]), np.array([4.0, 5.0, 6.0])
    h1 = np.array([3.0, 3.0 + 1e-9])
    u1 = _remap(h0, u0, h1, scheme)
    assert abs((h1 * u1).sum() - (h0 * u0).sum()) < 1e-12


@pytest.mark.parametrize("scheme", [P.PCM, P.PLM])
def test_no_new_extrema(scheme):                                    # :96-104
    rng = np.random.default_rng(3)
    h0 = rng.uniform(0.2, 2.0, 30)
    u0 = np.where(np.arange(30) < 15, 10.0, 20.0) + rng.normal(0, 0.5, 30)
    h1 = rng.uniform(0.1, 1.0, 50)
    h1 *= h0.sum() / h1.sum()
    u1 = _remap(h0, u0, h1, scheme)
    assert u1.min() >= u0.min() - 1e-12 and u1.max() <= u0.max() + 1e-12


def test_plm_less_diffusive_than_pcm_on_smooth_profile():          # :107-121
    h0 = np.full(40, 1.0)
    u0 = np.sin(2 * np.pi * (np.arange(40) + 0.5) / 40)
    hs = np.concatenate([[0.3], np.full(39, 1.0), [0.7]])
    err = {}
    for scheme in (P.PCM, P.PLM):
        u = u0.copy()
        for _ in range(10):
            u = _remap(hs, _remap(h0, u, hs, scheme), h0, scheme)
        err[scheme] = np.abs(u - u0).max()
    assert err[P.PLM] < 0.5 * err[P.PCM]


def test_ppm_no_new_extrema_and_conservation():                     # :138-146
    rng = np.random.default_rng(4)
    h0 = rng.uniform(0.2, 2.0, 40)
    u0 = np.where(np.arange(40) < 20, 10.0, 20.0) + rng.normal(0, 0.3, 40)
    h1 = rng.uniform(0.1, 1.0, 60)
    h1 *= h0.sum() / h1.sum()
    u1 = _remap(h0, u0, h1, P.PPM_H4)
    assert u1.min() >= u0.min() - 1e-12 and u1.max() <= u0.max() + 1e-12
    assert abs((h1 * u1).sum() - (h0 * u0).sum()) <= 1e-12 * abs((h0 * u0).sum())


def test_ppm_less_diffusive_than_plm():                             # :149-159
    h0 = np.full(40, 1.0)
    u0 = np.sin(2 * np.pi * (np.arange(40) + 0.5) / 40)
    hs = np.concatenate([[0.3], np.full(39, 1.0), [0.7]])
    err = {}
    for scheme in (P.PLM, P.PPM_H4):
        u = u0.copy()
        for _ in range(10):
            u = _remap(hs, _remap(h0, u, hs, scheme), h0, scheme)
        err[scheme] = np.abs(u - u0).max()
    assert err[P.PPM_H4] < err[P.PLM]


def test_short_columns_reduce_order():                              # :162-167
    for n in (1, 2, 3):
        h0 = np.ones(n)
        u0 = np.arange(n, dtype=float)
        np.testing.assert_allclose(_remap(h0, u0, h0, P.PPM_H4), u0, rtol=1e-14)


def test_zstar_like_column_with_many_vanished_bottom_layers():      # :170-179
    h0 = np.r_[np.full(44, 0.0), np.linspace(5, 20, 6)]
    u0 = np.r_[np.full(44, 12.0), np.linspace(12, 18, 6)]
    h1 = np.r_[np.full(44, 1e-3), np.linspace(5, 20, 6)]
    h1[-1] -= 44e-3
    for scheme in SCHEMES:
        u1 = _remap(h0, u0, h1, scheme)
        assert np.isfinite(u1).all()
        assert abs((h1 * u1).sum() - (h0 * u0).sum()) <= 1e-12 * (h0 * u0).sum()


def test_remap_columns_matches_single_column():                     # :182-195
    rng = np.random.default_rng(5)
    N, ny, nx = 8, 3, 4
    h0 = rng.uniform(0.5, 2.0, (N, ny, nx))
    f = rng.normal(10, 1, (N, ny, nx))
    h1 = rng.uniform(0.5, 2.0, (N, ny, nx))
    h1 *= h0.sum(0) / h1.sum(0)
    wet = np.ones((ny, nx), bool)
    wet[0, 0] = False
    out = P.remap_columns(h0, f, h1, P.PPM_H4, wet)
    np.testing.assert_array_equal(out, O.remap_columns(h0, f, h1, O.PPM_H4, wet))
    np.testing.assert_array_equal(out[:, 1, 2], _remap(h0[:, 1, 2], f[:, 1, 2], h1[:, 1, 2], P.PPM_H4))
    np.testing.assert_array_equal(out[:, 0, 0], f[:, 0, 0])


def test_ppm_interleaved_vanished_layers_many_columns():            # :205-216, the 200 columns in one call
    rng = np.random.default_rng(5)
    n, m = 50, 200
    h0 = np.empty((n, 1, m))
    u0 = np.empty((n, 1, m))
    h1 = np.empty((n, 1, m))
    for c in range(m):
        a = np.where(rng.random(n) < 0.85, rng.choice([0.0, 1e-10, 1e-3], n), rng.uniform(0.5, 50.0, n))
        u = rng.normal(15, 3, n)
        b = rng.uniform(0.1, 2.0, n)
        b *= a.sum() / b.sum()
        h0[:, 0, c], u0[:, 0, c], h1[:, 0, c] = a, u, b
    wet = np.ones((1, m), bool)
    u1 = P.remap_columns(h0, u0, h1, P.PPM_H4, wet)
    np.testing.assert_array_equal(u1, O.remap_columns(h0, u0, h1, O.PPM_H4, wet))
    assert np.isfinite(u1).all()
    tot0, tot1 = (h0 * u0).sum(0), (h1 * u1).sum(0)
    assert np.all(np.abs(tot1 - tot0) <= 1e-11 * np.abs(tot0))
