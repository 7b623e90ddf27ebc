"""
The CPU oracle (oracle/) against golden vectors produced by the reference itself (tests/golden/make_golden.py):
bit-for-bit equality, since both evaluate the same FP64 expressions in the same order without FMA contraction.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import case_open, case_periodic, load_golden, regrid_columns_args
from oracle import oracle as O

FCT = load_golden("fct")
RK3 = load_golden("rk3")
RK3X = load_golden("rk3_ext")
HLP = load_golden("helpers")
KER = load_golden("kernels")
REM = load_golden("remap")


def _adv(rec, cls=O.TracerAdvection):
    time = str(rec["time"]) if "time" in rec else "ssprk3"
    adv = cls(scheme=str(rec["scheme"]), time=time, dt=float(rec["dt"]), ob=O.OpenEdges(case_open(rec)))
    adv.per = O.Periodic(case_periodic(rec))
    return adv


@pytest.mark.parametrize("case", sorted(FCT))
def test_oracle_advect_fct_matches_reference_bitwise(case):
    rec = FCT[case]
    adv = _adv(rec)
    adv.record_open_flux = "open_flux" in rec
    fi = int(rec["flux_face_i"]) if "flux_face_i" in rec else None
    res = adv.advect_fct(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["ok"],
                         unlimited=bool(rec["unlimited"]), inflow=rec.get("inflow"), flux_face_i=fi)
    out, fx = (res if fi is not None else (res, None))
    np.testing.assert_array_equal(out, rec["out"])
    if fi is not None:
        np.testing.assert_array_equal(fx, rec["fx_i"])
    if "open_flux" in rec:
        np.testing.assert_allclose(adv.last_open_flux, rec["open_flux"], rtol=1e-13, atol=0)


@pytest.mark.parametrize("case", sorted(RK3))
def test_oracle_rk3_matches_reference_bitwise(case):
    rec = RK3[case]
    adv = _adv(rec)
    fi = int(rec["flux_face_i"]) if "flux_face_i" in rec else None
    res = adv.advect(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["Fz"], rec["ok"],
                     inflow=rec.get("inflow"), flux_face_i=fi)
    out, fx = (res if fi is not None else (res, None))
    np.testing.assert_array_equal(out, rec["out"])
    if fi is not None:
        np.testing.assert_array_equal(fx, rec["fx_i"])
    if not case_periodic(rec):
        np.testing.assert_array_equal(adv.rhs(rec["C"], rec["Qx"], rec["Qy"], rec["Fz"], rec["ok"]), rec["rhs"])


@pytest.mark.parametrize("case", sorted(RK3X))
def test_oracle_rk3_ext_matches_reference_bitwise(case):
    """The NumPy path's upwind-3/1 faces and the 'pc' time stepping."""
    rec = RK3X[case]
    adv = _adv(rec)
    fi = int(rec["flux_face_i"]) if "flux_face_i" in rec else None
    inflow = rec.get("inflow")
    res = adv.advect(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["Fz"], rec["ok"], inflow=inflow,
                     flux_face_i=fi)
    out, fx = (res if fi is not None else (res, None))
    np.testing.assert_array_equal(out, rec["out"])
    if fi is not None:
        np.testing.assert_array_equal(fx, rec["fx_i"])
    if "rhs" in rec:
        args = (rec["C"], rec["Qx"], rec["Qy"], rec["Fz"], rec["ok"])
        np.testing.assert_array_equal(adv.rhs(*args, centred=True, inflow=inflow), rec["rhs_centred"])
        np.testing.assert_array_equal(adv.rhs(*args, inflow=inflow), rec["rhs"])


@pytest.mark.parametrize("case", sorted(HLP))
def test_oracle_single_stage_helpers_match_reference_bitwise(case):
    """faces_h, upwind_faces_h, flux_x, rhs (and rhs_numpy where the oracle restates its faces)."""
    rec = HLP[case]
    adv = _adv(rec)
    C, Qx, Qy, Fz, ok, infl = rec["C"], rec["Qx"], rec["Qy"], rec["Fz"], rec["ok"], rec.get("inflow")
    okc = np.ascontiguousarray(np.broadcast_to(ok, C.shape[1:]))
    fx, fy = adv.faces_h(C, Qx, Qy, okc, inflow=infl)
    np.testing.assert_array_equal(fx, rec["faces_h_x"])
    np.testing.assert_array_equal(fy, rec["faces_h_y"])
    ux, uy = adv.upwind_faces_h(C, Qx, Qy, inflow=infl)
    np.testing.assert_array_equal(ux, rec["upwind_x"])
    np.testing.assert_array_equal(uy, rec["upwind_y"])
    np.testing.assert_array_equal(adv.flux_x(C, Qx, Qy, ok, inflow=infl), rec["flux_x"])
    np.testing.assert_array_equal(adv.flux_x(C, Qx, Qy, ok, centred=True, inflow=infl), rec["flux_x_centred"])
    np.testing.assert_array_equal(adv.rhs(C, Qx, Qy, Fz, ok, inflow=infl), rec["rhs"])
    np.testing.assert_array_equal(adv.rhs(C, Qx, Qy, Fz, ok, centred=True, inflow=infl), rec["rhs_centred"])
    if not str(rec["scheme"]).startswith("weno5"):
        np.testing.assert_array_equal(adv.rhs_numpy(C, Qx, Qy, Fz, ok, inflow=infl), rec["rhs_numpy"])


@pytest.mark.parametrize("variant", ["z", "js"])
def test_oracle_faces_match_reference_bitwise(variant):
    rec = KER["faces_" + variant]
    fx, fy = O.advect_faces_h(rec["c"], rec["Qx"], rec["Qy"], rec["ok"], rec["ext"], True, True, True, False,
                              variant == "z")
    np.testing.assert_array_equal(fx, rec["fx"])
    np.testing.assert_array_equal(fy, rec["fy"])


def test_oracle_fct_coefficients_match_reference_bitwise():
    rec = KER["coeff"]
    Cx, Cy = O.fct_coefficients(rec["c0"], rec["cL"], rec["V1"], rec["Ax"], rec["Ay"], rec["ok"], float(rec["dt"]))
    np.testing.assert_array_equal(Cx, rec["Cx"])
    np.testing.assert_array_equal(Cy, rec["Cy"])


@pytest.mark.parametrize("group", ["cols", "n0n1"])
@pytest.mark.parametrize("scheme", ["pcm", "plm", "ppm_h4"])
def test_oracle_remap_columns_match_reference_bitwise(group, scheme):
    rec = REM[group]
    out = O.remap_columns(rec["h_src"], rec["f_src"], rec["h_tgt"], O.SCHEMES[scheme], rec["wet"])
    np.testing.assert_array_equal(out, rec["out_" + scheme])


@pytest.mark.parametrize("case", sorted(c for c in REM if c.startswith("short")))
def test_oracle_short_columns_match_reference_bitwise(case):
    rec = REM[case]
    out = O.remap_column(rec["h_src"], rec["f_src"], rec["h_tgt"], int(rec["scheme"]))
    np.testing.assert_array_equal(out, rec["out"])


@pytest.mark.parametrize("case", ["coef_plm", "coef_ppm_h4"])
def test_oracle_reconstruction_matches_reference_bitwise(case):
    rec = REM[case]
    np.testing.assert_array_equal(O.reconstruct(rec["h"], rec["u"], int(rec["scheme"])), rec["coef"])


def test_oracle_plm_is_exact_for_a_linear_profile_interior():
    # tests/test_vertical_remap.py:83-93: u = 2 + 3 z as cell means on a non-uniform grid
    h = np.array([1.0, 0.5, 2.0, 1.0, 1.5])
    z = np.concatenate([[0.0], np.cumsum(h)])
    u = 2 + 3 * 0.5 * (z[1:] + z[:-1])
    coef = O.reconstruct(h, u, O.PLM)
    for k in (1, 2, 3):
        np.testing.assert_allclose(coef[k, 0], 2 + 3 * z[k], rtol=1e-12)
        np.testing.assert_allclose(coef[k, 0] + coef[k, 1], 2 + 3 * z[k + 1], rtol=1e-12)
    np.testing.assert_allclose(coef[[0, 4], 1], 0.0)


def test_oracle_ppm_is_exact_for_a_quadratic_interior():
    # tests/test_vertical_remap.py:124-135: cell means of 1 + z + z^2 (monotonic, no limiter action)
    h = np.array([1.0, 0.7, 1.3, 0.9, 1.1, 0.8, 1.2])
    z = np.concatenate([[0.0], np.cumsum(h)]) + 1.0
    F = lambda x: x + x ** 2 / 2 + x ** 3 / 3                                   # noqa: E731
    u = (F(z[1:]) - F(z[:-1])) / h
    coef = O.reconstruct(h, u, O.PPM_H4)
    for k in range(2, 5):
        np.testing.assert_allclose(coef[k, 0], 1 + z[k] + z[k] ** 2, rtol=1e-10)
        np.testing.assert_allclose(coef[k].sum(), 1 + z[k + 1] + z[k + 1] ** 2, rtol=1e-10)


def test_oracle_thread_count_does_not_change_results():
    rec = FCT["open4_inflow"]
    adv = _adv(rec)
    n0 = O.num_threads()
    try:
        O.set_threads(1)
        a = adv.advect_fct(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["ok"], inflow=rec["inflow"])
        O.set_threads(max(2, n0))
        b = adv.advect_fct(rec["C"], rec["V0"], rec["V1"], rec["Qx"], rec["Qy"], rec["ok"], inflow=rec["inflow"])
    finally:
        O.set_threads(n0)
    np.testing.assert_array_equal(a, b)


NB = load_golden("neighbours")


@pytest.mark.parametrize("case", ["regrid_zstar", "regrid_sigma", "regrid_zstar_hmin"])
def test_oracle_regrid_remap_matches_reference_bitwise(case):
    rec = NB[case]
    h_new, (T1, S1) = O.regrid_remap(str(rec["rule"]), rec["H"], rec["eta"], rec["h_src"], rec["active"],
                                     [rec["T"], rec["S"]], rec["coord"], O.PPM_H4, float(rec["h_min"]))
    np.testing.assert_array_equal(h_new, rec["h_new"])
    np.testing.assert_array_equal(T1, rec["T1"])
    np.testing.assert_array_equal(S1, rec["S1"])


def test_oracle_zstar_regrid_refuses_a_wet_column_without_depth():
    rec = NB["regrid_zstar_bad"]
    with pytest.raises(ValueError, match="z\\* needs H > 0"):
        O.regrid_remap("zstar", rec["H"], rec["eta"], rec["h_src"], rec["active"], [rec["T"]], rec["coord"],
                       O.PPM_H4, float(rec["h_min"]))


@pytest.mark.parametrize("case", ["regrid_hybrid", "regrid_hybrid_window", "regrid_hybrid_nokeep"])
def test_oracle_hybrid_regrid_remap_matches_reference_bitwise(case):
    rec = NB[case]
    params = {k: rec[k] for k in ("dz_top", "rho_target", "max_h_top", "dsigma")}
    params.update(d_sigma=float(rec["d_sigma"]), d_hybrid=float(rec["d_hybrid"]), h_min=float(rec["h_min"]),
                  keep_isopycnal=bool(rec["keep"]))
    h_new, wet, bad = O.regrid_hybrid(rec["H"], rec["eta"], rec["h_src"], rec["active"], rec["rho"], params)
    assert bad == 0
    np.testing.assert_array_equal(h_new, rec["h_new"])
    for f, ref in (("T", "T1"), ("S", "S1")):
        np.testing.assert_array_equal(O.remap_columns(rec["h_src"], rec[f], h_new, O.PPM_H4, wet), rec[ref])


@pytest.mark.parametrize("case", ["diffuse_closed", "diffuse_per_x", "diffuse_per_xy"])
def test_oracle_diffusion_matches_reference_bitwise(case):
    rec = NB[case]
    out = O.diffuse_ale(rec["T"], rec["Tw"], rec["h"], rec["act"], rec["cx"], rec["cy"], rec["okx"], rec["oky"],
                        rec["V"], float(rec["kh"]), float(rec["dt"]), O.Periodic(case_periodic(rec)))
    np.testing.assert_array_equal(out, rec["out"])


@pytest.mark.parametrize("case", ["faces_ppm_h4", "faces_plm", "faces_wgiven"])
def test_oracle_velocity_remap_matches_reference_bitwise(case):
    rec = NB[case]
    out = O.remap_faces(rec["vel"], rec["hf_src"], rec["hf_tgt"], int(rec["scheme"]), rec.get("w_tgt"))
    np.testing.assert_array_equal(out, rec["out"])


def test_oracle_face_fractions_match_reference_bitwise():
    rec = NB["fractions"]
    np.testing.assert_array_equal(O.face_fractions(rec["hf"]), rec["w"])


PR = load_golden("producers")


@pytest.mark.parametrize("case", ["ftt_clip", "ftt_noclip"])
def test_oracle_face_transport_thickness_matches_reference_bitwise(case):
    rec = PR[case]
    q_e, q_w = O.face_transport_thickness(rec["h"], rec["H"], rec["active"], bool(rec["clip"]))
    np.testing.assert_array_equal(q_e, rec["q_e"])
    np.testing.assert_array_equal(q_w, rec["q_w"])


def test_oracle_transport_velocity_matches_reference_bitwise():
    rec = PR["tvel"]
    ut, Qb = O.transport_velocity(rec["u_new"], rec["u_old"], rec["last_wet"], rec["w"], rec["L"], rec["D"],
                                  float(rec["theta"]), float(rec["theta_bc"]))
    np.testing.assert_array_equal(ut, rec["ut"])
    np.testing.assert_array_equal(Qb, rec["Qb"])


def test_oracle_ppm_edges_match_reference_bitwise():
    rec = PR["ppm_edges"]
    h_w, h_e = O.ppm_edges_x(rec["h"], rec["active"])
    np.testing.assert_array_equal(h_w, rec["h_w"])
    np.testing.assert_array_equal(h_e, rec["h_e"])


@pytest.mark.parametrize("case", ["ppm_transport_it20", "ppm_transport_it1"])
def test_oracle_ppm_transport_matches_reference_bitwise(case):
    rec = PR[case]
    out = O.ppm_transport_x(rec["h"], rec["ut"], rec["L"], rec["Q_bt"], rec["q_e"], rec["q_w"], rec["active"],
                            float(rec["dt"]), rec["dx"], int(rec["max_iter"]))
    np.testing.assert_array_equal(out, rec["Qx"])


@pytest.mark.parametrize("case", sorted(c for c in PR if c.startswith("limit_")))
def test_oracle_limit_outflow_matches_reference_bitwise(case):
    rec = PR[case]
    args = (rec["h"], rec["Qx"], rec["Qy"], rec["area"], float(rec["dt"]), rec["active"])
    per = tuple(bool(x) for x in rec["periodic"])
    if str(rec["status"]) == "raised":
        with pytest.raises(RuntimeError):
            O.limit_outflow(*args, periodic=per)
        return
    Qx, Qy, nl = O.limit_outflow(*args, periodic=per)
    assert nl == int(rec["n_limited"])
    np.testing.assert_array_equal(Qx, rec["Qx_out"])
    np.testing.assert_array_equal(Qy, rec["Qy_out"])


@pytest.mark.parametrize("case", ["lagrangian_calm", "lagrangian_limited", "lagrangian_strong"])
def test_oracle_lagrangian_thickness_matches_reference_bitwise(case):
    rec = PR[case]
    args = (rec["h"], rec["divq"], float(rec["dt"]), rec["area"])
    if bool(rec["raises"]):
        with pytest.raises(RuntimeError, match="emptied in the Lagrangian step"):
            O.lagrangian_thickness(*args)
        return
    np.testing.assert_array_equal(O.lagrangian_thickness(*args), rec["h_dag"])


LT = load_golden("layer_transport")


@pytest.mark.parametrize("case", ["upwind", "upwind_empty"])
def test_oracle_upwind_transport_matches_reference_bitwise(case):
    rec = LT[case]
    np.testing.assert_array_equal(O.upwind_transport_x(rec["q_e"], rec["q_w"], rec["ut"], rec["L"], rec["Q_bt"]),
                                  rec["Q"])


@pytest.mark.parametrize("case", ["fw_thickness", "fw_volume"])
def test_oracle_freshwater_volumes_match_reference_bitwise(case):
    rec = LT[case]
    V, nl = O.freshwater_volumes(rec["V"], rec["dV"], rec["floor"])
    np.testing.assert_array_equal(V, rec["V_new"])
    assert nl == int(rec["n_limited"])


def test_oracle_lagrangian_thickness_signed_zero_matches_reference():
    rec = LT["lagrangian_negzero"]
    out = O.lagrangian_thickness(rec["h"], rec["divq"], float(rec["dt"]), rec["area"])
    np.testing.assert_array_equal(out, rec["h_dag"])
    assert not np.signbit(out).any() and not np.signbit(rec["h_dag"]).any()


def layer_transport_args(rec) -> dict:
    return dict(h=rec["h"], u_old=rec["u"], v_old=rec["v"], u_new=rec["u_new"], v_new=rec["v_new"],
                wet_u=rec["wet_u"], wet_v=rec["wet_v"], wu=rec["wu"], wv=rec["wv"], Lu=rec["Lu"], Lv=rec["Lv"],
                Du=rec["Du"], Dv=rec["Dv"], qe=rec["qe"], qw=rec["qw"], qn=rec["qn"], qs=rec["qs"],
                active=rec["active"], area=rec["area"], dx_t=rec["dx_t"], dy_t=rec["dy_t"], dt=float(rec["dt"]),
                theta=float(rec["theta"]), theta_bc=float(rec["theta_bc"]),
                thickness_flux=str(rec["thickness_flux"]),
                periodic=("x" in list(rec["periodic"]), "y" in list(rec["periodic"])), fw=rec.get("fw"),
                open_=tuple(str(e) for e in rec["open"]) if "open" in rec else (), open_Du=rec.get("open_Du"),
                open_Dv=rec.get("open_Dv"), open_Qu=rec.get("open_Qu"), open_Qv=rec.get("open_Qv"))


@pytest.mark.parametrize("case", ["lt_ppm", "lt_upwind", "lt_ppm_fw", "lt_upwind_perx", "lt_ppm_strong",
                                  "lt_upwind_strong"])
def test_oracle_layer_transport_step_matches_reference_bitwise(case):
    rec = LT[case]
    out = O.ale_layer_transport(**layer_transport_args(rec))
    for key in ("Qx", "Qy", "V0", "V1", "ok", "h_dagger") + (("h_fw", "V_fw") if "fw" in rec else ()):
        np.testing.assert_array_equal(out[key], rec[key], err_msg=key)
    assert out["n_limited"] == int(rec["n_limited"])


LTX = load_golden("layer_transport_ext")


@pytest.mark.parametrize("case", sorted(LTX))
def test_oracle_layer_transport_periodic_ppm_and_open_edges_match_reference_bitwise(case):
    rec = LTX[case]
    out = O.ale_layer_transport(**layer_transport_args(rec))
    for key in ("Qx", "Qy", "V0", "V1", "ok", "h_dagger"):
        np.testing.assert_array_equal(out[key], rec[key], err_msg=key)
    assert out["n_limited"] == int(rec["n_limited"])


RC = load_golden("regrid_columns")


@pytest.mark.parametrize("case", sorted(RC))
def test_oracle_regrid_columns_matches_reference_bitwise(case):
    rec = RC[case]
    zw = O.regrid_columns(*regrid_columns_args(rec))
    np.testing.assert_array_equal(zw, rec["zw"])


def test_oracle_regrid_columns_raises_where_the_reference_does():
    rec = RC["rc_zstar"]
    with pytest.raises(ValueError, match="only for rule 'hybrid'"):
        O.regrid_columns("zstar", rec["H"], rec["eta"], rec["h"], None, {"dz_top": rec["dz_top"]}, rec["wet"], 5)
    with pytest.raises(ValueError, match="needs params"):
        O.regrid_columns("sigma", rec["H"], rec["eta"], rec["h"], None, {}, rec["wet"])
