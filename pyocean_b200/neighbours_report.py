"""
Timing of the neighbours of the tracer step at the benchmark size (512 x 512 x 50 basin, T and S):

* the z* regrid + PPM_H4 remap of both tracers in one call (``pocean_regrid_remap_f64``), and the regrid alone;
* the same with the hybrid (HYCOM1) rule on a stratified column (``pocean_regrid_hybrid_remap_f64``);
* the ALE horizontal diffusion of the T/S stack, with its compulsory HBM bytes (T, Tw in and out per tracer; h, V
  per cell; the 2-D masks and metrics once) against the measured HBM peak;
* the velocity remap in fraction space of the u-faces (512 x 513 x 50);
* the producers of the step's inputs on the u-faces: face transport thickness, transport velocity, PPM layer
  transport with the barotropic Newton correction, the outflow limiter's check (nothing to limit, its common case)
  and the Lagrangian thickness;
* the whole layer-transport step (``producers.ALELayerTransport``) with the PPM and the donor-cell flux, and the
  whole ALE tracer step on device tensors (layer transport, advect_fct, regrid and remap);
* the unlimited RK3 step ``TracerAdvection.advect`` with a vertical transport (the secondary path).

    python -m pyocean_b200.neighbours_report
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

from . import _lib
from . import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _hbm_peak() -> float:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"])
    return 6650.0


def _time(fn, reps: int = 20, warm: int = 3) -> float:
    for _ in range(warm):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def neighbours_report(device=None) -> dict:
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    L = _lib.lib()
    w = W.basin()
    nt, n, ny, nx = w.C.shape
    plane = ny * nx
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                       # noqa: E731
    st = lambda: torch.cuda.current_stream(dev).cuda_stream                                # noqa: E731
    H = w.h_tgt.sum(0)
    Hd, etad = g(np.where(w.wet, H, np.nan)), g(np.zeros((ny, nx)))
    hs, C = g(w.h_src), g(w.C)
    act = g(w.wet.astype(np.uint8))
    dz = g(np.full(n, 4000.0 / n))
    h_new, wet = torch.empty_like(hs), torch.empty((ny, nx), dtype=torch.uint8, device=dev)
    out, out2 = torch.empty_like(C), torch.empty_like(C)

    def fused():
        _lib.check(L.pocean_regrid_remap_f64(0, Hd.data_ptr(), etad.data_ptr(), hs.data_ptr(), act.data_ptr(),
                                             dz.data_ptr(), 1e-3, C.data_ptr(), n, ny, nx, nt, 2, h_new.data_ptr(),
                                             wet.data_ptr(), out.data_ptr(), None, st()), "regrid_remap")

    def separate():
        _lib.check(L.pocean_regrid_remap_f64(0, Hd.data_ptr(), etad.data_ptr(), hs.data_ptr(), act.data_ptr(),
                                             dz.data_ptr(), 1e-3, None, n, ny, nx, 0, 2, h_new.data_ptr(),
                                             wet.data_ptr(), None, None, st()), "regrid")
        _lib.check(L.pocean_remap_columns_f64(hs.data_ptr(), C.data_ptr(), h_new.data_ptr(), wet.data_ptr(), n, n,
                                              ny, nx, nt, 2, out2.data_ptr(), st()), "remap_columns")

    def regrid_only():
        _lib.check(L.pocean_regrid_remap_f64(0, Hd.data_ptr(), etad.data_ptr(), hs.data_ptr(), act.data_ptr(),
                                             dz.data_ptr(), 1e-3, None, n, ny, nx, 0, 2, h_new.data_ptr(),
                                             wet.data_ptr(), None, None, st()), "regrid")

    t_fused, t_sep, t_regrid = _time(fused), _time(separate), _time(regrid_only)
    torch.cuda.synchronize()
    same = bool(torch.equal(out, out2))

    # hybrid rule: densities of a stratified column (linear EOS), isopycnal targets over their range, a z* floor and
    # a sigma window over the shallower part of the basin (1300-1700 m)
    rng = np.random.default_rng(3)
    zmid = np.cumsum(w.h_src, axis=0) - 0.5 * w.h_src
    T = 4.0 + 16.0 * zmid / np.maximum(w.h_src.sum(0), 1.0) + rng.normal(0.0, 0.3, w.h_src.shape)
    rho_np = 1027.0 * (1.0 - 2e-4 * (T - 10.0))
    lo, hi = float(rho_np[:, w.wet].min()), float(rho_np[:, w.wet].max())
    rho = g(rho_np)
    rho_t = g(np.r_[lo - 0.02, lo - 0.01, np.linspace(lo, hi, n - 1)])
    dzh, mht, dsg = g(np.linspace(2.0, 120.0, n)), g(np.full(n, 400.0)), g(np.full(n, 1.0 / n))

    def hybrid(nf):
        _lib.check(L.pocean_regrid_hybrid_remap_f64(Hd.data_ptr(), etad.data_ptr(), hs.data_ptr(), act.data_ptr(),
                                                    rho.data_ptr(), rho_t.data_ptr(), dzh.data_ptr(), mht.data_ptr(),
                                                    dsg.data_ptr(), 1300.0, 1700.0, 1e-2, 1,
                                                    C.data_ptr() if nf else None, n, ny, nx, nf, 2,
                                                    h_new.data_ptr(), wet.data_ptr(),
                                                    out.data_ptr() if nf else None, None, st()), "regrid_hybrid")

    t_hyb, t_hyb_regrid = _time(lambda: hybrid(nt), reps=10), _time(lambda: hybrid(0), reps=10)

    # diffusion of the stack
    rng = np.random.default_rng(1)
    h = g(np.where(w.wet[None], w.h_tgt, 0.0))
    V = g(w.V0)
    cx, cy = g(rng.uniform(0.5, 2.0, (ny, nx + 1))), g(rng.uniform(0.5, 2.0, (ny + 1, nx)))
    okx = g((rng.random((ny, nx + 1)) > 0.05).astype(np.uint8))
    oky = g((rng.random((ny + 1, nx)) > 0.05).astype(np.uint8))
    Tw = C - 10.0
    dout = torch.empty_like(C)

    def diffuse():
        _lib.check(L.pocean_diffuse_ale_f64(C.data_ptr(), Tw.data_ptr(), h.data_ptr(), act.data_ptr(), cx.data_ptr(),
                                            cy.data_ptr(), okx.data_ptr(), oky.data_ptr(), V.data_ptr(), nt, n, ny,
                                            nx, 0, 100.0, 600.0, dout.data_ptr(), st()), "diffuse_ale")

    t_diff = _time(diffuse)
    diff_bytes = n * plane * (24 * nt + 16) + plane * (1 + 2 * 9)
    # velocity remap of the u-faces
    nf = nx + 1
    hu_src = g(np.abs(rng.normal(5.0, 2.0, (n, ny, nf))))
    hu_tgt = g(np.abs(rng.normal(5.0, 2.0, (n, ny, nf))))
    vel = g(rng.normal(0.0, 0.3, (n, ny, nf)))
    vout = torch.empty_like(vel)

    def faces():
        _lib.check(L.pocean_remap_faces_f64(vel.data_ptr(), hu_src.data_ptr(), hu_tgt.data_ptr(), None, n, ny, nf, 1,
                                            2, vout.data_ptr(), st()), "remap_faces")

    t_faces = _time(faces)

    # producers (u-faces)
    Hd0 = g(H)
    u8 = lambda a: g(a.astype(np.uint8))                                                   # noqa: E731
    hx = g(np.where(w.wet[None], w.h_src, 0.0))
    q_e, q_w = torch.empty_like(vel), torch.empty_like(vel)
    ut, Qb = torch.empty_like(vel), torch.empty((ny, nf), dtype=torch.float64, device=dev)
    Lf, Df = g(rng.uniform(1800.0, 2200.0, (ny, nf))), g(rng.uniform(20.0, 400.0, (ny, nf)))
    lw = u8(rng.random((ny, nf)) > 0.05)
    wf = torch.full_like(vel, 1.0 / n)
    u1, u0 = g(rng.normal(0.0, 0.3, (n, ny, nf))), g(rng.normal(0.0, 0.3, (n, ny, nf)))
    dxt = g(np.full((ny, nx), 2000.0))
    Qx = torch.empty_like(vel)
    nbytes = L.pocean_ppm_transport_workspace_bytes(n, ny, nx, 20)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)

    def ftt():
        _lib.check(L.pocean_face_transport_thickness_f64(hx.data_ptr(), Hd0.data_ptr(), act.data_ptr(), n, ny, nx, 1,
                                                         q_e.data_ptr(), q_w.data_ptr(), st()), "ftt")

    def tvel():
        _lib.check(L.pocean_transport_velocity_f64(u1.data_ptr(), u0.data_ptr(), lw.data_ptr(), wf.data_ptr(),
                                                   Lf.data_ptr(), Df.data_ptr(), n, ny, nf, 0.6, 0.5, ut.data_ptr(),
                                                   Qb.data_ptr(), st()), "tvel")

    def ppm():
        _lib.check(L.pocean_ppm_transport_f64(hx.data_ptr(), ut.data_ptr(), Lf.data_ptr(), Qb.data_ptr(),
                                              q_e.data_ptr(), q_w.data_ptr(), act.data_ptr(), dxt.data_ptr(), n, ny,
                                              nx, 300.0, 20, Qx.data_ptr(), ws.data_ptr(), nbytes, st()), "ppm")

    t_ftt, t_tvel = _time(ftt), _time(tvel)
    t_ppm = _time(ppm, reps=5)
    t_lt = _layer_transport_ms(w, dev, rng)
    t_rk3 = _advect_rk3_ms(w, dev)
    peak = _hbm_peak()
    return dict(workload=w.name,
                regrid_remap_zstar=dict(call_ms=t_fused, regrid_ms=t_regrid, regrid_then_remap_columns_ms=t_sep,
                                        equal=same, fields=nt),
                regrid_remap_hybrid=dict(call_ms=t_hyb, regrid_ms=t_hyb_regrid, fields=nt),
                diffuse_ale=dict(ms=t_diff, algorithmic_bytes=diff_bytes, gbs=diff_bytes / t_diff / 1e6,
                                 frac_of_measured_hbm=diff_bytes / t_diff / 1e6 / peak, fields=nt),
                remap_faces_u=dict(ms=t_faces, faces=n * ny * nf),
                producers_u=dict(face_transport_thickness_ms=t_ftt, transport_velocity_ms=t_tvel,
                                 ppm_transport_ms=t_ppm, faces=n * ny * nf),
                layer_transport_step=t_lt, advect_rk3=t_rk3)


def _advect_rk3_ms(w, dev) -> dict:
    """``TracerAdvection.advect`` (SSP-RK3 without limiter, WENO5 in x, y and z) of the basin's stack with a
    vertical transport through the interfaces, on device tensors."""
    from .step import ALETracerStep  # noqa: F401  (library loaded)
    from .tracers import TracerAdvection
    from .periodic import Periodic
    nt, n, ny, nx = w.C.shape
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                       # noqa: E731
    rng = np.random.default_rng(4)
    Fz = np.zeros((n + 1, ny, nx))
    Fz[1:-1] = rng.normal(0.0, 1.0, (n - 1, ny, nx)) * 1e2 * w.wet
    adv = TracerAdvection(scheme=w.scheme, time="ssprk3", dt=w.dt)
    adv.per = Periodic(w.periodic)
    args = [g(a) for a in (w.C, w.V0, w.V1, w.Qx, w.Qy, Fz, w.ok)]
    out = adv.advect(*args)
    torch.cuda.synchronize()
    ms = _time(lambda: adv.advect(*args), reps=10)
    return dict(ms=ms, cell_steps_per_s=w.tracer_cells / (ms / 1e3),
                what="advect (RK3, no limiter, vertical WENO) of the 512 x 512 x 50 T/S stack", finite=bool(
                    torch.isfinite(out).all()))


def _layer_transport_ms(w, dev, rng) -> dict:
    """The whole ALE layer-transport step (``producers.ALELayerTransport``: both face axes, PPM or donor-cell
    fluxes, limiter, h-dagger, volumes) on device tensors, warm, mean of a few calls."""
    from types import SimpleNamespace as NS

    from . import producers as P
    n, ny, nx = w.h_src.shape
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)                       # noqa: E731
    act = w.wet
    h = np.where(act[None], w.h_src, 0.0)
    H = h.sum(0)
    wet_u = np.zeros((ny, nx + 1), bool)
    wet_u[:, 1:-1] = act[:, 1:] & act[:, :-1]
    wet_v = np.zeros((ny + 1, nx), bool)
    wet_v[1:-1] = act[1:] & act[:-1]
    Du, Dv = np.zeros((ny, nx + 1)), np.zeros((ny + 1, nx))
    Du[:, 1:-1] = np.minimum(H[:, 1:], H[:, :-1])
    Dv[1:-1] = np.minimum(H[1:], H[:-1])
    hd, Hd = g(h), g(H)
    qe, qw = P.face_transport_thickness(hd, Hd, g(act), True)
    qn, qs = P.face_transport_thickness(hd.transpose(1, 2).contiguous(), Hd.T.contiguous(), g(act.T), True)
    from .vertical import face_fractions
    wu = face_fractions(0.5 * (qe + qw))
    wv = face_fractions(0.5 * (qn + qs)).transpose(1, 2).contiguous()
    u = [g(rng.normal(0.0, 0.2, (n, ny, nx + 1)) * wet_u) for _ in range(2)]
    v = [g(rng.normal(0.0, 0.2, (n, ny + 1, nx)) * wet_v) for _ in range(2)]
    area = g(np.full((ny, nx), 4e6))
    fs = NS(theta=0.6, active=g(act), Lu=g(np.full((ny, nx + 1), 2000.0)), Lv=g(np.full((ny + 1, nx), 2000.0)))
    geom = {"dx_t": g(np.full((ny, nx), 2000.0)), "dy_t": g(np.full((ny, nx), 2000.0))}
    fl = NS(wet_u=g(wet_u), wet_v=g(wet_v), Du=g(Du), Dv=g(Dv), fw=None)
    st = NS(h=hd, u=u[0], v=v[0], eta=None)
    out = {}
    for flux in ("ppm", "upwind"):
        lt = P.ALELayerTransport(fs=fs, H=Hd, area=area, dt=300.0, thickness_flux=flux, vi_geom=geom)
        run = lambda: lt(st, None, u[1], v[1], fl, 0.5, (), wu, wv, qe, qw, qn, qs)            # noqa: E731
        run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            lf = run()
        e1.record()
        e1.synchronize()
        out[flux + "_ms"] = e0.elapsed_time(e1) / 3
        out[flux + "_n_limited"] = lf.n_limited
    out["what"] = "ALELayerTransport on device tensors, both face axes, 512 x 512 x 50 basin layers, dt 300 s"

    # the whole ALE tracer step on the device: the layer transport (PPM), advect_fct of the T/S stack on its
    # fluxes and volumes, then the z* regrid of the Lagrangian thicknesses and the PPM_H4 remap of the stack; no
    # array leaves HBM between the three
    from .tracers import TracerAdvection
    L = _lib.lib()
    nt = w.C.shape[0]
    lt = P.ALELayerTransport(fs=fs, H=Hd, area=area, dt=300.0, thickness_flux="ppm", vi_geom=geom)
    adv = TracerAdvection(scheme="weno5", time="ssprk3", dt=300.0)
    C = g(w.C)
    Hn, eta0, actd = g(np.where(act, H, np.nan)), g(np.zeros((ny, nx))), g(act.astype(np.uint8))
    dz = g(np.full(n, 4000.0 / n))
    h_new, wet_new, C_new = torch.empty_like(hd), torch.empty((ny, nx), dtype=torch.uint8, device=dev), torch.empty_like(C)

    def whole():
        lf = lt(st, None, u[1], v[1], fl, 0.5, (), wu, wv, qe, qw, qn, qs)
        A = adv.advect_fct(C, lf.V0, lf.V1, lf.Qx, lf.Qy, lf.ok)
        _lib.check(L.pocean_regrid_remap_f64(0, Hn.data_ptr(), eta0.data_ptr(), lf.h_dagger.data_ptr(),
                                             actd.data_ptr(), dz.data_ptr(), 1e-3, A.data_ptr(), n, ny, nx, nt, 2,
                                             h_new.data_ptr(), wet_new.data_ptr(), C_new.data_ptr(), None,
                                             torch.cuda.current_stream(dev).cuda_stream), "regrid_remap")
        return A

    whole()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        whole()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / 3
    out["whole_ale_step"] = dict(ms=ms, tracer_cell_steps_per_s=nt * n * ny * nx / (ms / 1e3),
                                 finite=bool(torch.isfinite(C_new).all()),
                                 what="layer transport (PPM) + advect_fct of T and S + z* regrid and PPM_H4 remap, "
                                      "all on device tensors")
    return out


if __name__ == "__main__":
    print(json.dumps(neighbours_report()))
