"""The neighbours of the tracer step on the GPU: z* / sigma / hybrid regrid with the remap, the velocity remap in
fraction space, the face fractions and the ALE diffusion — bit for bit against the reference's golden vectors and
the oracle, plus full-size cases against the oracle."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import case_periodic, load_golden, regrid_columns_args
import pyocean_b200 as P
from oracle import oracle as O
from pyocean_b200 import ALECoordinate, Periodic, diffuse_ale, face_fractions, remap_faces
from pyocean_b200 import workloads as W

pytestmark = pytest.mark.gpu
NB = load_golden("neighbours")


def _vc(rec):
    key = "dz_top" if str(rec["rule"]) == "zstar" else "dsigma"
    return ALECoordinate(rec["H"], rec["active"], str(rec["rule"]), {key: rec["coord"], "h_min": float(rec["h_min"])},
                         2)


@pytest.mark.parametrize("case", ["regrid_zstar", "regrid_sigma", "regrid_zstar_hmin"])
def test_regrid_remap_matches_reference_bitwise(case):
    rec = NB[case]
    h_new, (T1, S1) = _vc(rec).regrid_remap(rec["eta"], rec["h_src"], [rec["T"], rec["S"]], rec["T"], rec["S"])
    np.testing.assert_array_equal(h_new, rec["h_new"])
    np.testing.assert_array_equal(T1, rec["T1"])
    np.testing.assert_array_equal(S1, rec["S1"])


@pytest.mark.parametrize("case", ["regrid_zstar", "regrid_sigma"])
def test_regrid_alone_and_three_fields(case):
    rec = NB[case]
    vc = _vc(rec)
    np.testing.assert_array_equal(vc.regrid(rec["eta"], rec["h_src"], rec["T"]), rec["h_new"])
    U = rec["T"] * 0.5 + 1.0
    _, outs = vc.regrid_remap(rec["eta"], rec["h_src"], [rec["T"], rec["S"], U])   # a pair and an odd field
    wet = rec["active"] & (np.nan_to_num(rec["H"]) + rec["eta"] > 0) & (rec["h_src"].sum(0) > 0)
    np.testing.assert_array_equal(outs[2], O.remap_columns(rec["h_src"], U, rec["h_new"], 2, wet))


def test_zstar_regrid_raises_like_the_reference():
    rec = NB["regrid_zstar_bad"]
    with pytest.raises(ValueError, match="z\\* needs H > 0"):
        _vc(rec).regrid_remap(rec["eta"], rec["h_src"], [rec["T"]], rec["T"])


class _LinearEOS:
    """The linear equation of state the hybrid golden cases were made with."""
    linear = True

    @staticmethod
    def density(T, S):
        return 1027.0 * (1.0 - 2e-4 * (T - 10.0) + 7.6e-4 * (S - 35.0))


def _hybrid_params(rec) -> dict:
    return {"dz_top": rec["dz_top"], "rho_target": rec["rho_target"], "max_h_top": rec["max_h_top"],
            "dsigma": rec["dsigma"], "d_sigma": float(rec["d_sigma"]), "d_hybrid": float(rec["d_hybrid"]),
            "h_min": float(rec["h_min"]), "keep_isopycnal": bool(rec["keep"])}


@pytest.mark.parametrize("case", ["regrid_hybrid", "regrid_hybrid_window", "regrid_hybrid_nokeep"])
def test_hybrid_regrid_remap_matches_reference_bitwise(case):
    rec = NB[case]
    vc = ALECoordinate(rec["H"], rec["active"], "hybrid", _hybrid_params(rec), 2, eos=_LinearEOS)
    h_new, (T1, S1) = vc.regrid_remap(rec["eta"], rec["h_src"], [rec["T"], rec["S"]], rec["T"], rec["S"])
    np.testing.assert_array_equal(h_new, rec["h_new"])
    np.testing.assert_array_equal(T1, rec["T1"])
    np.testing.assert_array_equal(S1, rec["S1"])
    # the densities given directly, regrid alone
    np.testing.assert_array_equal(vc.regrid(rec["eta"], rec["h_src"], rho=rec["rho"]), rec["h_new"])


def test_hybrid_regrid_raises_like_the_reference():
    rec = NB["regrid_hybrid"]
    params = _hybrid_params(rec)
    H = rec["H"].copy()
    H[2, 3] = 0.0                                      # a wet column with H <= 0 and no sigma zone
    eta = rec["eta"].copy()
    eta[2, 3] = 0.5
    act = np.ones_like(rec["active"])
    with pytest.raises(ValueError, match="hybrid needs"):
        ALECoordinate(H, act, "hybrid", params, 2).regrid_remap(eta, rec["h_src"], [rec["T"]], rho=rec["rho"])
    rho = rec["rho"].copy()
    rho[1, 3, 3] = np.nan                              # non-finite density in a wet column
    with pytest.raises(ValueError, match="hybrid needs"):
        ALECoordinate(rec["H"], act, "hybrid", params, 2).regrid(rec["eta"], rec["h_src"], rho=rho)
    with pytest.raises(ValueError, match="rho_target"):
        ALECoordinate(rec["H"], rec["active"], "hybrid", {"dz_top": rec["dz_top"]}, 2).regrid(
            rec["eta"], rec["h_src"], rho=rec["rho"])


def test_full_size_hybrid_regrid_remap_against_oracle():
    # a stratified basin with density inversions and massless layers: isopycnal targets over the density range, a
    # z* floor, a shallow sigma window
    w = W.basin(seed=4, nx=192, ny=160, n=40)
    rng = np.random.default_rng(21)
    n = 40
    H = np.where(w.wet, w.h_tgt.sum(0), np.nan)
    eta = rng.uniform(-0.5, 0.5, H.shape)
    hs = w.h_src.copy()
    hs[rng.random(hs.shape) < 0.1] = 0.0
    z = np.cumsum(hs, axis=0) - 0.5 * hs                             # layer mid heights above the bed
    T = 4.0 + 16.0 * z / np.maximum(hs.sum(0), 1.0) + rng.normal(0.0, 0.3, hs.shape)
    S = 35.0 + rng.normal(0.0, 0.2, hs.shape)
    rho = _LinearEOS.density(T, S)
    lo, hi = float(rho[:, w.wet].min()), float(rho[:, w.wet].max())
    rho_t = np.r_[lo - 0.02, lo - 0.01, np.linspace(lo, hi, n - 1)]
    params = {"dz_top": np.linspace(2.0, 120.0, n), "rho_target": rho_t, "max_h_top": np.full(n, 400.0),
              "dsigma": np.full(n, 1.0 / n), "d_sigma": 1300.0, "d_hybrid": 1700.0, "h_min": 0.01}
    dev = torch.device("cuda", 0)
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                       # noqa: E731
    for keep in (True, False):
        p = dict(params, keep_isopycnal=keep)
        vc = ALECoordinate(H, w.wet, "hybrid", p, 2, eos=_LinearEOS)
        h_new, outs = vc.regrid_remap(g(eta), g(hs), [g(T), g(S)], g(T), g(S))
        ref_h, wet, bad = O.regrid_hybrid(H, eta, hs, w.wet, rho, p)
        assert bad == 0
        assert torch.equal(h_new.cpu(), torch.from_numpy(ref_h))
        for m, f in enumerate((T, S)):
            np.testing.assert_array_equal(outs[m].cpu().numpy(), O.remap_columns(hs, f, ref_h, 2, wet))


@pytest.mark.parametrize("case", ["faces_ppm_h4", "faces_plm", "faces_wgiven"])
def test_velocity_remap_matches_reference_bitwise(case):
    rec = NB[case]
    out = remap_faces(rec["vel"], rec["hf_src"], rec["hf_tgt"], int(rec["scheme"]), rec.get("w_tgt"))
    np.testing.assert_array_equal(out, rec["out"])


def test_face_fractions_match_reference_bitwise():
    rec = NB["fractions"]
    np.testing.assert_array_equal(face_fractions(rec["hf"]), rec["w"])


@pytest.mark.parametrize("case", ["diffuse_closed", "diffuse_per_x", "diffuse_per_xy"])
def test_diffusion_matches_reference_bitwise(case):
    rec = NB[case]
    per = Periodic(case_periodic(rec))
    out = diffuse_ale(rec["T"], rec["Tw"], rec["h"], rec["act"], rec["cx"], rec["cy"], rec["okx"], rec["oky"],
                      rec["V"], float(rec["kh"]), float(rec["dt"]), per)
    np.testing.assert_array_equal(out, rec["out"])


def test_diffusion_stack_equals_fields_one_by_one():
    rec = NB["diffuse_per_x"]
    per = Periodic(("x",))
    T2 = np.stack([rec["T"], rec["T"] * 1.5])
    Tw2 = np.stack([rec["Tw"], rec["Tw"] - 3.0])
    out = diffuse_ale(T2, Tw2, rec["h"], rec["act"], rec["cx"], rec["cy"], rec["okx"], rec["oky"], rec["V"],
                      float(rec["kh"]), float(rec["dt"]), per)
    for m in range(2):
        one = O.diffuse_ale(T2[m], Tw2[m], rec["h"], rec["act"], rec["cx"], rec["cy"], rec["okx"], rec["oky"],
                            rec["V"], float(rec["kh"]), float(rec["dt"]), O.Periodic(("x",)))
        np.testing.assert_array_equal(out[m], one)


def test_full_size_regrid_remap_and_diffusion_against_oracle():
    # the basin's bathymetry with z* and sigma targets, both tracers; the diffusion of T on the same grid
    w = W.basin(seed=2, nx=256, ny=192, n=30)
    rng = np.random.default_rng(9)
    H = w.h_tgt.sum(0)
    H = np.where(w.wet, H, np.nan)
    eta = rng.uniform(-0.5, 0.5, H.shape)
    dz = np.linspace(5.0, 300.0, 30)
    for rule, params in (("zstar", {"dz_top": dz}), ("sigma", {"dsigma": np.full(30, 1 / 30)})):
        vc = ALECoordinate(H, w.wet, rule, params, 2)
        dev = torch.device("cuda", 0)
        g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                   # noqa: E731
        h_new, outs = vc.regrid_remap(g(eta), g(w.h_src), g(w.C))
        coord = params["dz_top"] if rule == "zstar" else params["dsigma"]
        ref_h, ref = O.regrid_remap(rule, H, eta, w.h_src, w.wet, [w.C[0], w.C[1]], coord, 2)
        assert torch.equal(h_new.cpu(), torch.from_numpy(ref_h))
        for m in range(2):
            np.testing.assert_array_equal(outs[m].cpu().numpy(), ref[m])
    n, ny, nx = w.V0.shape
    act = w.wet
    h = np.where(act[None], w.h_tgt, 0.0)
    cx = rng.uniform(0.5, 2.0, (ny, nx + 1))
    cy = rng.uniform(0.5, 2.0, (ny + 1, nx))
    okx = rng.random((ny, nx + 1)) > 0.05
    oky = rng.random((ny + 1, nx)) > 0.05
    Tw = w.C[0] - 10.0
    out = diffuse_ale(w.C[0], Tw, h, act, cx, cy, okx, oky, w.V0, 100.0, 600.0)
    np.testing.assert_array_equal(out, O.diffuse_ale(w.C[0], Tw, h, act, cx, cy, okx, oky, w.V0, 100.0, 600.0))


RC = load_golden("regrid_columns")


@pytest.mark.parametrize("case", sorted(RC))
def test_regrid_columns_matches_reference_bitwise(case):
    rec = RC[case]
    args = regrid_columns_args(rec)
    zw = P.regrid_columns(*args)
    np.testing.assert_array_equal(zw, rec["zw"])
    dev = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda()   # noqa: E731
    rule, H, eta, h, rho, params, wet, n_out = args
    zd = P.regrid_columns(rule, dev(H), dev(eta), dev(h), dev(rho), params, dev(wet), n_out)
    assert zd.is_cuda
    np.testing.assert_array_equal(zd.cpu().numpy(), rec["zw"])


def test_regrid_columns_finer_source_against_oracle_and_errors():
    rng = np.random.default_rng(17)
    n, m, ny, nx = 90, 40, 96, 80
    H = rng.uniform(3.0, 500.0, (ny, nx))
    eta = rng.uniform(-0.4, 0.4, (ny, nx))
    wet = rng.random((ny, nx)) > 0.1
    D = H + eta
    w = rng.uniform(0.3, 1.7, (n, ny, nx))
    h = w / w.sum(0) * D[None]
    z = np.cumsum(h, axis=0) - 0.5 * h
    rho = 1030.0 - 6.0 * np.clip(z / 400.0, 0, 1) + rng.normal(0, 0.01, (n, ny, nx))
    rho_t = np.linspace(rho.min() - 0.5, rho.max() + 0.1, m + 1)
    params = dict(dz_top=np.full(m, 4.0), rho_target=rho_t, max_h_top=np.full(m, 50.0), h_min=0.05,
                  dsigma=np.full(m, 1.0 / m), d_sigma=5.0, d_hybrid=50.0)
    zw = P.regrid_columns("hybrid", H, eta, h, rho, params, wet, n_out=m)
    np.testing.assert_array_equal(zw, O.regrid_columns("hybrid", H, eta, h, rho, params, wet, n_out=m))
    assert zw.shape == (m + 1, ny, nx) and np.isnan(zw[:, ~wet]).all() and np.isfinite(zw[:, wet]).all()
    with pytest.raises(ValueError, match="only for rule 'hybrid'"):
        P.regrid_columns("zstar", H, eta, h, None, {"dz_top": np.ones(n)}, wet, n_out=m)
    bad = rho.copy()
    bad[3, 5, 5] = np.nan
    wet2 = wet.copy()
    wet2[5, 5] = True
    with pytest.raises(ValueError, match="non-finite density"):
        P.regrid_columns("hybrid", H, eta, h, bad, params, wet2, n_out=m)
