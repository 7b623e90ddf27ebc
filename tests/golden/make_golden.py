"""
Generate the golden vectors of tests/golden/ by running the reference pyOCEAN code itself.

Run where a checkout of the reference (read-only) is available, giving its path::

    python tests/golden/make_golden.py REFERENCE [case-group ...]

It imports the reference's own modules (``core.components.tracers``, ``core.dynamics.sigma_baroclinic``,
``core.vertical.remap``) with a stub ``xarray`` (the hot-path modules use it only in annotations and helpers that
are not called here), keeps Numba's cache and Python's bytecode out of the reference tree, feeds seeded synthetic
inputs through the reference's public calls and stores inputs and outputs as compressed ``.npz`` files next to this
script.  The tests never import the reference: they read these files.
"""
from __future__ import annotations

import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
if len(sys.argv) < 2 or not os.path.isdir(sys.argv[1]):
    sys.exit("usage: python tests/golden/make_golden.py REFERENCE [case-group ...]  (REFERENCE: path of the "
             "reference pyOCEAN checkout)")
REFERENCE = sys.argv[1]

os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/pocean_golden_numba_cache")
os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
sys.dont_write_bytecode = True
_xr = types.ModuleType("xarray")


class _Placeholder:                                   # annotations only
    pass


_xr.Dataset = _xr.DataArray = _Placeholder
sys.modules.setdefault("xarray", _xr)
sys.path.insert(0, REFERENCE)

import numpy as np                                     # noqa: E402

from core.components.tracers import TracerAdvection    # noqa: E402
from core.dynamics import sigma_baroclinic as sb       # noqa: E402
from core.model import threads                         # noqa: E402
from core.model.periodic import Periodic               # noqa: E402
from core.vertical import remap as rm                  # noqa: E402
from core.vertical import regrid as rg                 # noqa: E402
from core.vertical import ale                          # noqa: E402
from core.vertical.ale import face_fractions           # noqa: E402
from core.components.vertical_coordinate import ALECoordinate   # noqa: E402


class _OB:
    def __init__(self, open_=()):
        self.open = tuple(open_)


def transports(rng, nt, n, ny, nx, dt, open_=(), land=0.1, thin=True, periodic=()):
    """Seeded layer volumes and transports: V0, V1 = V0 − Δt ∇·Q, ok = active & V1 > 0 (as the ALE step)."""
    h = rng.uniform(1.0, 5.0, (n, ny, nx))
    if thin:
        h[min(2, n - 1), ny // 2, nx // 2] = 1e-3
    area = rng.uniform(0.9, 1.1, (ny, nx)) * 1e6
    active = rng.random((ny, nx)) > land
    V0 = area * h * active
    hx = np.concatenate([h[..., :1], h], axis=-1)
    hy = np.concatenate([h[:, :1], h], axis=1)
    Qx = rng.uniform(-0.4, 0.4, (n, ny, nx + 1)) * 1e3 * hx
    Qy = rng.uniform(-0.4, 0.4, (n, ny + 1, nx)) * 1e3 * hy
    ax = np.zeros((ny, nx + 1), bool)
    ax[:, 1:-1] = active[:, 1:] & active[:, :-1]
    ay = np.zeros((ny + 1, nx), bool)
    ay[1:-1] = active[1:] & active[:-1]
    if "west" in open_:
        ax[:, 0] = active[:, 0]
    if "east" in open_:
        ax[:, -1] = active[:, -1]
    if "south" in open_:
        ay[0] = active[0]
    if "north" in open_:
        ay[-1] = active[-1]
    if "x" in periodic:
        ax[:, 0] = ax[:, -1] = active[:, 0] & active[:, -1]
    if "y" in periodic:
        ay[0] = ay[-1] = active[0] & active[-1]
    Qx *= ax
    Qy *= ay
    if "x" in periodic:
        Qx[..., -1] = Qx[..., 0]
    if "y" in periodic:
        Qy[:, -1] = Qy[:, 0]
    V1 = V0 - dt * (Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:] - Qy[:, :-1])
    ok = active[None] & (V1 > 0)
    return V0, V1, Qx, Qy, ok


def fct_cases():
    out = {}
    specs = [
        # name, nt, n, ny, nx, open, inflow, scheme, periodic, dt, extras
        ("closed", 2, 4, 12, 14, (), False, "weno5", (), 30.0, {}),
        ("open4_inflow", 2, 4, 12, 14, ("west", "east", "south", "north"), True, "weno5", (), 30.0, {}),
        ("open3_noinflow", 2, 3, 10, 13, ("west", "east", "south"), False, "weno5", (), 30.0, {}),
        ("js", 2, 4, 11, 12, ("west",), True, "weno5js", (), 30.0, {}),
        ("periodic_x", 1, 5, 16, 16, (), False, "weno5", ("x",), 30.0, {}),
        ("periodic_xy", 2, 3, 12, 10, (), False, "weno5", ("x", "y"), 30.0, {}),
        ("periodic_x_open_sn", 1, 3, 12, 9, ("south", "north"), True, "weno5", ("x",), 30.0, {}),
        ("tef_budget", 2, 3, 9, 11, ("west", "east", "north"), True, "weno5", (), 30.0,
         {"flux_face_i": 4, "record": True}),
        ("unlimited", 2, 3, 9, 11, ("west",), True, "weno5", (), 30.0, {"unlimited": True}),
        ("unlimited_tef", 1, 3, 8, 10, (), False, "weno5", (), 30.0, {"unlimited": True, "flux_face_i": 3}),
        ("tiny_1x1", 1, 2, 1, 1, (), False, "weno5", (), 30.0, {}),
        ("thin_row", 1, 2, 1, 9, ("west", "east"), True, "weno5", (), 30.0, {}),
    ]
    for seed, (name, nt, n, ny, nx, open_, infl, scheme, per, dt, extras) in enumerate(specs):
        rng = np.random.default_rng(100 + seed)
        V0, V1, Qx, Qy, ok = transports(rng, nt, n, ny, nx, dt, open_, periodic=per)
        T = 7.0 + rng.normal(0, 1, (n, ny, nx))
        C = np.stack([T, T ** 2][:nt]) if nt <= 2 else rng.normal(0, 1, (nt, n, ny, nx))
        inflow = np.stack([np.full(T.shape, 9.0), np.full(T.shape, 81.0)][:nt]) if infl else None
        adv = TracerAdvection(scheme=scheme, time="ssprk3", dt=dt, ob=_OB(open_))
        adv.per = Periodic(per)
        adv.record_open_flux = bool(extras.get("record"))
        res = adv.advect_fct(C, V0, V1, Qx, Qy, ok, unlimited=bool(extras.get("unlimited")), inflow=inflow,
                             flux_face_i=extras.get("flux_face_i"))
        rec = dict(C=C, V0=V0, V1=V1, Qx=Qx, Qy=Qy, ok=ok, dt=dt, scheme=scheme, open=np.array(open_, dtype="U5"),
                   periodic=np.array(per, dtype="U1"), unlimited=bool(extras.get("unlimited")))
        if inflow is not None:
            rec["inflow"] = inflow
        if "flux_face_i" in extras:
            rec["flux_face_i"] = extras["flux_face_i"]
            rec["out"], rec["fx_i"] = res
        else:
            rec["out"] = res
        if adv.record_open_flux:
            rec["open_flux"] = adv.last_open_flux
        out[name] = rec
    # the two-cell pulse at Courant 0.5 of tests/test_sigma_ale.py:1308-1325 (1-D, 4 layers, dx = 1 km)
    nx, n, dt, dx = 60, 4, 30.0, 1000.0
    h = np.full((n, 1, nx), 5.0)
    V = h * dx * dx
    Qx = np.zeros((n, 1, nx + 1))
    Qx[:, :, 1:-1] = 0.5 * dx / dt * h[:, :, 1:] * dx
    Qx[:, :, -2:] = 0.0
    Qy = np.zeros((n, 2, nx))
    V1 = V - dt * (Qx[..., 1:] - Qx[..., :-1])
    ok = V1 > 0
    T = np.where((np.arange(nx) >= 20) & (np.arange(nx) < 22), 1.0, 0.0)[None, None, :].repeat(n, 0)[None]
    adv = TracerAdvection(scheme="weno5", time="ssprk3", dt=dt, ob=_OB())
    out["pulse"] = dict(C=T, V0=V, V1=V1, Qx=Qx, Qy=Qy, ok=ok, dt=dt, scheme="weno5", open=np.array((), "U5"),
                        periodic=np.array((), "U1"), unlimited=False, out=adv.advect_fct(T, V, V1, Qx, Qy, ok))
    return out


def rk3_cases():
    out = {}
    specs = [("open_vert", 2, 6, 9, 13, ("west", "east", "south"), True, "weno5", ()),
             ("closed_js_vert", 1, 5, 8, 10, (), False, "weno5js", ()),
             ("periodic_x_novert", 2, 4, 10, 12, (), False, "weno5", ("x",)),
             ("tef", 1, 4, 7, 9, ("east",), False, "weno5", ()),
             ("open_inflow_vert", 2, 5, 8, 11, ("west", "east", "south", "north"), True, "weno5", ())]
    for seed, (name, nt, n, ny, nx, open_, vert, scheme, per) in enumerate(specs):
        rng = np.random.default_rng(200 + seed)
        dt = 10.0
        V0, V1, Qx, Qy, ok = transports(rng, nt, n, ny, nx, dt, open_, periodic=per)
        Fz = rng.normal(size=(n + 1, ny, nx)) * 1e2 if vert else np.zeros((n + 1, ny, nx))
        Fz[0] = Fz[-1] = 0.0
        C = rng.normal(10.0, 1.0, (nt, n, ny, nx))
        inflow = rng.normal(11.0, 1.0, C.shape) if "inflow" in name else None
        adv = TracerAdvection(scheme=scheme, time="ssprk3", dt=dt, ob=_OB(open_))
        adv.per = Periodic(per)
        fi = 3 if name == "tef" else None
        res = adv.advect(C, V0, V1, Qx, Qy, Fz, ok, inflow=inflow, flux_face_i=fi)
        rec = dict(C=C, V0=V0, V1=V1, Qx=Qx, Qy=Qy, Fz=Fz, ok=ok, dt=dt, scheme=scheme,
                   open=np.array(open_, dtype="U5"), periodic=np.array(per, dtype="U1"))
        if inflow is not None:
            rec["inflow"] = inflow
        if fi is None:
            rec["out"] = res
        else:
            rec["flux_face_i"] = fi
            rec["out"], rec["fx_i"] = res
        # the RHS alone (_advect_div) for the kernel-level check
        rec["rhs"] = adv.rhs(C, Qx, Qy, Fz, ok) if not per else adv.rhs(C[..., :], Qx, Qy, Fz, ok)
        out[name] = rec
    return out


def rk3_ext_cases():
    """``advect`` with the NumPy path's face schemes (upwind3, upwind1) and the 'pc' predictor-corrector time
    stepping (tracers.py:110-151, 303-375)."""
    out = {}
    specs = [("up3_open_vert_inflow", 2, 6, 9, 13, ("west", "east", "south"), True, "upwind3", "ssprk3", ()),
             ("up1_closed_vert", 1, 5, 8, 10, (), True, "upwind1", "ssprk3", ()),
             ("up3_periodic_xy_tef", 2, 4, 10, 12, (), False, "upwind3", "ssprk3", ("x", "y")),
             ("pc_weno5_open_vert", 2, 7, 9, 11, ("west", "north"), True, "weno5", "pc", ()),
             ("pc_weno5js_periodic_x_tef", 1, 5, 8, 12, ("south",), True, "weno5js", "pc", ("x",)),
             ("pc_up3_inflow_vert", 2, 6, 8, 11, ("west", "east", "south", "north"), True, "upwind3", "pc", ()),
             ("pc_up1_novert_tef", 1, 4, 7, 9, ("east",), False, "upwind1", "pc", ())]
    for seed, (name, nt, n, ny, nx, open_, vert, scheme, time, per) in enumerate(specs):
        rng = np.random.default_rng(900 + seed)
        dt = 10.0
        V0, V1, Qx, Qy, ok = transports(rng, nt, n, ny, nx, dt, open_, periodic=per)
        Fz = rng.normal(size=(n + 1, ny, nx)) * 1e2 if vert else np.zeros((n + 1, ny, nx))
        Fz[0] = Fz[-1] = 0.0
        C = rng.normal(10.0, 1.0, (nt, n, ny, nx))
        inflow = rng.normal(11.0, 1.0, C.shape) if "inflow" in name else None
        adv = TracerAdvection(scheme=scheme, time=time, dt=dt, ob=_OB(open_))
        adv.per = Periodic(per)
        fi = 4 if name.endswith("tef") else None
        res = adv.advect(C, V0, V1, Qx, Qy, Fz, ok, inflow=inflow, flux_face_i=fi)
        rec = dict(C=C, V0=V0, V1=V1, Qx=Qx, Qy=Qy, Fz=Fz, ok=ok, dt=dt, scheme=scheme, time=time,
                   open=np.array(open_, dtype="U5"), periodic=np.array(per, dtype="U1"))
        if inflow is not None:
            rec["inflow"] = inflow
        if fi is None:
            rec["out"] = res
        else:
            rec["flux_face_i"] = fi
            rec["out"], rec["fx_i"] = res
        if not per:
            # the NumPy RHS alone: centred (the predictor's) and with the scheme's own faces
            rec["rhs_centred"] = adv.rhs(C, Qx, Qy, Fz, ok, centred=True, inflow=inflow)
            rec["rhs"] = adv.rhs(C, Qx, Qy, Fz, ok, inflow=inflow)
        out[name] = rec
    return out


def helper_cases():
    """The single-stage helpers of TracerAdvection (tracers.py:139-206) on unpadded arrays: faces_h, upwind_faces_h,
    flux_x (scheme and centred faces), rhs (fused WENO5 or the NumPy path; centred) and rhs_numpy."""
    out = {}
    specs = [("weno5_open_inflow_vert", 2, 5, 9, 12, ("west", "east", "south"), True, "weno5"),
             ("weno5js_closed", 1, 4, 8, 10, (), False, "weno5js"),
             ("up3_open_vert", 2, 5, 8, 11, ("west", "north"), True, "upwind3"),
             ("up1_inflow", 1, 4, 7, 9, ("east", "south"), True, "upwind1")]
    for seed, (name, nt, n, ny, nx, open_, vert, scheme) in enumerate(specs):
        rng = np.random.default_rng(700 + seed)
        dt = 10.0
        V0, V1, Qx, Qy, ok = transports(rng, nt, n, ny, nx, dt, open_)
        Fz = rng.normal(size=(n + 1, ny, nx)) * 1e2 if vert else np.zeros((n + 1, ny, nx))
        Fz[0] = Fz[-1] = 0.0
        C = rng.normal(10.0, 1.0, (nt, n, ny, nx))
        inflow = rng.normal(11.0, 1.0, C.shape) if "inflow" in name else None
        adv = TracerAdvection(scheme=scheme, time="ssprk3", dt=dt, ob=_OB(open_))
        okc = np.ascontiguousarray(np.broadcast_to(ok, C.shape[1:]))
        rec = dict(C=C, Qx=Qx, Qy=Qy, Fz=Fz, ok=ok, dt=dt, scheme=scheme, open=np.array(open_, dtype="U5"),
                   periodic=np.array((), dtype="U1"))
        if inflow is not None:
            rec["inflow"] = inflow
        rec["faces_h_x"], rec["faces_h_y"] = adv.faces_h(C, Qx, Qy, okc, inflow=inflow)
        rec["upwind_x"], rec["upwind_y"] = adv.upwind_faces_h(C, Qx, Qy, inflow=inflow)
        rec["flux_x"] = adv.flux_x(C, Qx, Qy, ok, inflow=inflow)
        rec["flux_x_centred"] = adv.flux_x(C, Qx, Qy, ok, centred=True, inflow=inflow)
        rec["rhs"] = adv.rhs(C, Qx, Qy, Fz, ok, inflow=inflow)
        rec["rhs_centred"] = adv.rhs(C, Qx, Qy, Fz, ok, centred=True, inflow=inflow)
        rec["rhs_numpy"] = adv.rhs_numpy(C, Qx, Qy, Fz, ok, inflow=inflow)
        out[name] = rec
    return out


def kernel_cases():
    """Single kernels: faces_h and the FCT coefficients (tests/test_sigma_ale.py:1396-1429 inputs)."""
    out = {}
    rng = np.random.default_rng(3)
    nt, n, ny, nx = 2, 3, 4, 5
    c0 = rng.uniform(0, 1, (nt, n, ny, nx)); cL = rng.uniform(0, 1, (nt, n, ny, nx))
    V1 = rng.uniform(0.5, 2, (n, ny, nx)) * 1e6
    Ax = rng.normal(0, 1e4, (nt, n, ny, nx + 1)); Ax[..., [0, -1]] = 0
    Ay = rng.normal(0, 1e4, (nt, n, ny + 1, nx)); Ay[..., [0, -1], :] = 0
    ok = rng.uniform(0, 1, (n, ny, nx)) > 0.1
    Cx, Cy = sb._fct_coeff_kernel(c0, cL, V1, Ax, Ay, ok, 30.0)
    out["coeff"] = dict(c0=c0, cL=cL, V1=V1, Ax=Ax, Ay=Ay, ok=ok, dt=30.0, Cx=Cx, Cy=Cy)
    rng = np.random.default_rng(11)
    nt, n, ny, nx = 2, 3, 9, 11
    c = rng.normal(10.0, 1.0, (nt, n, ny, nx))
    Qx = rng.normal(size=(n, ny, nx + 1)); Qx[rng.random(Qx.shape) < 0.1] = 0.0
    Qy = rng.normal(size=(n, ny + 1, nx)); Qy[rng.random(Qy.shape) < 0.1] = 0.0
    ok = rng.random((n, ny, nx)) > 0.15
    ext = rng.normal(12.0, 1.0, c.shape)
    for z in (True, False):
        fx, fy = sb._advect_faces_h(c, Qx, Qy, ok, ext, True, True, True, False, z)
        out["faces_" + ("z" if z else "js")] = dict(c=c, Qx=Qx, Qy=Qy, ok=ok, ext=ext, fx=fx, fy=fy)
    return out


def remap_cases():
    out = {}
    rng = np.random.default_rng(5)
    # many columns: random thicknesses with vanished layers at random places, n0 = n1 = 50
    N, ny, nx = 50, 8, 25
    h0 = np.where(rng.random((N, ny, nx)) < 0.3, rng.choice([0.0, 1e-10, 1e-3], (N, ny, nx)),
                  rng.uniform(0.5, 50.0, (N, ny, nx)))
    f = rng.normal(15, 3, (N, ny, nx))
    h1 = rng.uniform(0.1, 2.0, (N, ny, nx))
    h1 *= h0.sum(0) / h1.sum(0)
    h1[:, 0, :5] = h0[:, 0, :5]                        # identity columns
    h1[:, 1, :3] = 0.0                                 # vanished targets (whole column)
    h1[3:9, 2, :] = 0.0                                # a band of vanished targets
    h1[:, 2, :] *= h0[:, 2, :].sum(0) / np.where(h1[:, 2, :].sum(0) > 0, h1[:, 2, :].sum(0), 1.0)
    h1[-1, 3, :4] += 1e-9                              # target thicker than source
    h0[-1, 3, 4:8] += 1e-9                             # source thicker than target
    h0[:, 4, :2] = 0.0                                 # dry-by-thickness columns (wet flag True)
    wet = rng.random((ny, nx)) > 0.1
    wet[4, :2] = True
    out["cols"] = dict(h_src=h0, f_src=f, h_tgt=h1, wet=wet)
    for name, scheme in (("pcm", rm.PCM), ("plm", rm.PLM), ("ppm_h4", rm.PPM_H4)):
        out["cols"]["out_" + name] = rm.remap_columns(h0, f, h1, scheme, wet)
    # n0 != n1 (with dry columns -> NaN), z*-like columns with many vanished bottom layers
    N0, N1 = 30, 20
    h0 = rng.uniform(0.0, 4.0, (N0, 6, 7)); h0[rng.random(h0.shape) < 0.2] = 0.0
    h0[:22, 5, :] = 0.0
    f = rng.normal(12, 2, (N0, 6, 7))
    h1 = rng.uniform(0.1, 2.0, (N1, 6, 7)); h1 *= h0.sum(0) / h1.sum(0)
    wet = np.ones((6, 7), bool); wet[0, 0] = False; wet[2, 3] = False
    out["n0n1"] = dict(h_src=h0, f_src=f, h_tgt=h1, wet=wet)
    for name, scheme in (("pcm", rm.PCM), ("plm", rm.PLM), ("ppm_h4", rm.PPM_H4)):
        out["n0n1"]["out_" + name] = rm.remap_columns(h0, f, h1, scheme, wet)
    # short columns (n = 1 … 5) in every scheme, single-column API
    for n in (1, 2, 3, 4, 5):
        hs = rng.uniform(0.2, 2.0, n); us = rng.normal(10, 2, n)
        ht = rng.uniform(0.2, 2.0, n + 1); ht *= hs.sum() / ht.sum()
        for name, scheme in (("pcm", rm.PCM), ("plm", rm.PLM), ("ppm_h4", rm.PPM_H4)):
            u1 = np.empty(n + 1)
            rm.remap_column(hs, us, ht, scheme, u1)
            out[f"short{n}_{name}"] = dict(h_src=hs, f_src=us, h_tgt=ht, scheme=scheme, out=u1)
    # reconstruction coefficients of a few columns
    for name, scheme in (("plm", rm.PLM), ("ppm_h4", rm.PPM_H4)):
        h = np.array([1.0, 0.7, 0.0, 1.3, 0.9, 1e-12, 1.1, 0.8, 1.2, 2.0])
        u = rng.normal(10, 2, h.size)
        coef = np.empty((h.size, 3))
        rm.reconstruct(h, u, scheme, rm.H_NEGLECT, rm.H_NEGLECT_EDGE, coef)
        out["coef_" + name] = dict(h=h, u=u, scheme=scheme, coef=coef)
    return out


class _Vertical:
    """The attributes of an ALECoordinate that regrid_remap / regrid / remap_faces read, with the reference's own
    methods (core/components/vertical_coordinate.py:69-153)."""
    regrid_remap = ALECoordinate.regrid_remap
    regrid = ALECoordinate.regrid
    regrid_density = ALECoordinate.regrid_density
    remap_faces = ALECoordinate.remap_faces

    def __init__(self, H, active, rule, params, remap_code):
        self.H, self.active, self.regrid_rule = H, active, rule
        self.regrid_params, self.remap_code = params, remap_code


def neighbour_cases():
    """The z*/sigma/hybrid regrid + remap, the ALE diffusion kernel and the velocity remap in fraction space."""
    out = {}
    rng = np.random.default_rng(21)
    n, ny, nx = 12, 7, 9
    H = rng.uniform(20.0, 400.0, (ny, nx))
    H[0, :3] = rng.uniform(0.5, 3.0, 3)                       # shallower than the nominal levels: collapsed layers
    H[1, 0] = np.nan                                         # land depth NaN (nan_to_num -> 0, not wet)
    active = rng.random((ny, nx)) > 0.1
    active[1, 0] = True
    eta = rng.uniform(-1.0, 1.0, (ny, nx))
    eta[1, 0] = -0.5                                         # the NaN-depth column is dry (D <= 0)
    h_src = rng.uniform(0.5, 40.0, (n, ny, nx))
    h_src[rng.random(h_src.shape) < 0.1] = 0.0
    h_src[:, 2, 2] = 0.0                                     # no water: not wet
    T = rng.normal(12.0, 3.0, (n, ny, nx))
    S = rng.normal(35.0, 0.3, (n, ny, nx))
    dz_top = np.linspace(2.0, 30.0, n)                       # nominal z* levels, surface first
    dsigma = rng.uniform(0.5, 1.5, n)
    dsigma /= dsigma.sum()
    for rule, params in (("zstar", {"dz_top": dz_top}), ("sigma", {"dsigma": dsigma}),
                         ("zstar_hmin", {"dz_top": dz_top, "h_min": 0.25})):
        Hc = H.copy()
        if rule == "sigma":
            Hc[3, 4] = -0.5                                   # flooded land: sigma at any depth (D > 0 with eta)
        etac = eta.copy()
        etac[3, 4] = 1.0
        r = rule.split("_")[0]
        vc = _Vertical(Hc, active, r, params, rm.PPM_H4)
        h_new, (T1, S1) = vc.regrid_remap(etac, h_src, [T, S], T, S)
        coord = params["dz_top"] if r == "zstar" else params["dsigma"]
        out["regrid_" + rule] = dict(rule=r, H=Hc, eta=etac, h_src=h_src, active=active, coord=coord,
                                     h_min=params.get("h_min", rg.H_MIN), T=T, S=S, h_new=h_new, T1=T1, S1=S1)
    # z* with a wet column of H <= 0: the reference raises ValueError
    Hb = H.copy()
    Hb[4, 4] = 0.0
    eb = eta.copy()
    eb[4, 4] = 0.5
    try:
        _Vertical(Hb, active | True, "zstar", {"dz_top": dz_top}, rm.PPM_H4).regrid_remap(eb, h_src, [T], T)
        raised = False
    except ValueError:
        raised = True
    assert raised
    out["regrid_zstar_bad"] = dict(rule="zstar", H=Hb, eta=eb, h_src=h_src, active=active | True, coord=dz_top,
                                   h_min=rg.H_MIN, T=T, raises=True)

    # the hybrid (HYCOM1) rule with a linear equation of state: isopycnal targets, a z* floor, a maximum top
    # thickness, and (second case) a shallow sigma zone with flooded land
    class _EOS:
        linear = True

        @staticmethod
        def density(T, S):
            return 1027.0 * (1.0 - 2e-4 * (T - 10.0) + 7.6e-4 * (S - 35.0))

    rho_col = _EOS.density(T, S)
    rho_t = rg.target_densities(rho_col[::-1, 3, 3], n, n_light=2)
    base = {"dz_top": dz_top, "rho_target": rho_t, "max_h_top": np.full(n, 80.0), "h_min": 0.05}
    for name, extra in (("hybrid", {}), ("hybrid_window", {"dsigma": dsigma, "d_sigma": 5.0, "d_hybrid": 60.0}),
                        ("hybrid_nokeep", {"keep_isopycnal": False})):
        params = dict(base, **extra)
        Hc, etac = H.copy(), eta.copy()
        if "d_hybrid" in extra:
            Hc[3, 4], etac[3, 4] = -0.5, 1.0                          # flooded land: sigma at any depth
        vc = _Vertical(Hc, active, "hybrid", params, rm.PPM_H4)
        vc.eos = _EOS
        h_new, (T1, S1) = vc.regrid_remap(etac, h_src, [T, S], T, S)
        out["regrid_" + name] = dict(rule="hybrid", H=Hc, eta=etac, h_src=h_src, active=active, rho=rho_col,
                                     rho_target=rho_t, dz_top=dz_top, max_h_top=params["max_h_top"],
                                     dsigma=params.get("dsigma", np.full(n, 1.0 / n)),
                                     d_sigma=params.get("d_sigma", 0.0), d_hybrid=params.get("d_hybrid", 0.0),
                                     h_min=params["h_min"], keep=params.get("keep_isopycnal", True), T=T, S=S,
                                     h_new=h_new, T1=T1, S1=S1)

    # ALE diffusion kernel (tracers.py:436-447): closed, periodic x, periodic x and y
    n, ny, nx = 4, 9, 11
    for name, axes in (("closed", ()), ("per_x", ("x",)), ("per_xy", ("x", "y"))):
        Tf = rng.normal(15.0, 2.0, (n, ny, nx))
        Tw = Tf - rng.normal(14.0, 0.5, (n, 1, 1))
        act = rng.random((ny, nx)) > 0.1
        h = np.where(act[None], rng.uniform(0.0, 20.0, (n, ny, nx)), 0.0)
        h[1, 3, 3] = 0.0
        cx = rng.uniform(0.5, 2.0, (ny, nx + 1))
        cy = rng.uniform(0.5, 2.0, (ny + 1, nx))
        okx = rng.random((ny, nx + 1)) > 0.1
        oky = rng.random((ny + 1, nx)) > 0.1
        if "x" in axes:
            cx[:, -1] = cx[:, 0]
            okx[:, -1] = okx[:, 0]
        if "y" in axes:
            cy[-1] = cy[0]
            oky[-1] = oky[0]
        V = np.where(act[None], rng.uniform(1e5, 1e7, (n, ny, nx)), 0.0)
        kh, dt = 50.0, 300.0

        def run(T, Tw, h, act, cx, cy, okx, oky, V):
            o = np.empty(np.shape(T))
            c = np.ascontiguousarray
            sb._diffuse_ale_kernel(c(T, dtype=float), c(Tw, dtype=float), c(h, dtype=float), c(act),
                                   c(cx, dtype=float), c(cy, dtype=float), c(okx), c(oky), c(V, dtype=float), kh, dt,
                                   o)
            return o
        args = (Tf, Tw, h, act, cx, cy, okx, oky, V)
        if axes:
            res = Periodic(axes).apply(run, args, ("c", "c", "c", "c", "u", "v", "u", "v", "c"), "c", 1)
        else:
            res = run(*args)
        out["diffuse_" + name] = dict(T=Tf, Tw=Tw, h=h, act=act, cx=cx, cy=cy, okx=okx, oky=oky, V=V, kh=kh,
                                      dt=dt, periodic=np.array(axes, dtype=str), out=res)

    # velocity remap in fraction space and the fractions themselves (u-faces (N, ny, nx+1))
    n, ny, nxf = 10, 6, 9
    vel = rng.normal(0.0, 0.3, (n, ny, nxf))
    hf_src = rng.uniform(0.0, 8.0, (n, ny, nxf))
    hf_src[rng.random(hf_src.shape) < 0.15] = 0.0
    hf_src[:, 0, 0] = 0.0                                    # a face without water
    hf_tgt = rng.uniform(0.1, 6.0, (n, ny, nxf))
    hf_tgt[:4, 1, :] = 0.0
    for code, name in ((rm.PPM_H4, "ppm_h4"), (rm.PLM, "plm")):
        vc = _Vertical(None, None, "zstar", {}, code)
        out["faces_" + name] = dict(vel=vel, hf_src=hf_src, hf_tgt=hf_tgt, scheme=code,
                                    out=vc.remap_faces(vel, hf_src, hf_tgt))
    w_given = face_fractions(hf_tgt)
    out["faces_wgiven"] = dict(vel=vel, hf_src=hf_src, hf_tgt=hf_tgt, w_tgt=w_given, scheme=rm.PPM_H4,
                               out=_Vertical(None, None, "zstar", {}, rm.PPM_H4).remap_faces(vel, hf_src, hf_tgt,
                                                                                              w_given))
    out["fractions"] = dict(hf=hf_src, w=face_fractions(hf_src))
    return out


def _producer_state(rng, n, ny, nx, land=0.12):
    """A basin of layers for the producer cases: depth, active mask, layer thicknesses (bed first, z*-like with a
    shallow shelf), face lengths, metrics and a velocity field."""
    H = rng.uniform(30.0, 300.0, (ny, nx))
    H[:, : nx // 4] = rng.uniform(5.0, 20.0, (ny, nx // 4))            # shelf: thin / vanished bed layers
    active = rng.random((ny, nx)) > land
    h = np.empty((n, ny, nx))
    for k in range(n):
        h[k] = H / n * rng.uniform(0.6, 1.4, (ny, nx))
    h[0, :, : nx // 4] = 0.0                                           # vanished bed layer on the shelf
    h[:, ~active] = np.nan
    dx = rng.uniform(900.0, 1100.0, (ny, nx))
    Lu = rng.uniform(900.0, 1100.0, (ny, nx + 1))
    return H, active, h, dx, Lu


def producer_cases():
    """The producers of the step's inputs: face transport thicknesses, transport velocity, PPM layer transport
    with its barotropic correction, the outflow limiter (fast and limiting paths) and the Lagrangian thickness."""
    out = {}
    rng = np.random.default_rng(33)
    n, ny, nx = 6, 9, 14
    H, active, h, dx, Lu = _producer_state(rng, n, ny, nx)
    for clip in (True, False):
        q_e, q_w = ale.face_transport_thickness(h, H, active, clip)
        out["ftt_" + ("clip" if clip else "noclip")] = dict(h=h, H=H, active=active, clip=clip, q_e=q_e, q_w=q_w)
    q_e, q_w = ale.face_transport_thickness(h, H, active, True)
    # transport velocity (fractions of the face layers, half the faces wet in the last step)
    u_new = rng.normal(0.0, 0.4, (n, ny, nx + 1))
    u_old = rng.normal(0.0, 0.4, (n, ny, nx + 1))
    last_wet = rng.random((ny, nx + 1)) > 0.2
    w = face_fractions(0.5 * (q_e + q_w))
    D = rng.uniform(5.0, 300.0, (ny, nx + 1))
    ut, Qb = ale.transport_velocity(u_new, u_old, last_wet, w, Lu, D, 0.6, 0.5)
    out["tvel"] = dict(u_new=u_new, u_old=u_old, last_wet=last_wet, w=w, L=Lu, D=D, theta=0.6, theta_bc=0.5, ut=ut,
                       Qb=Qb)
    # PPM edges and layer transport (Courant up to ~0.4, a barotropic target that needs correcting)
    dt = 600.0
    hc = np.where(active[None], np.nan_to_num(h), 0.0)
    h_w, h_e = ale.ppm_edges_x(hc, active)
    out["ppm_edges"] = dict(h=h, active=active, h_w=h_w, h_e=h_e)
    Q_bt = Qb * rng.uniform(0.8, 1.2, Qb.shape)
    for it in (20, 1):
        Qx = ale.ppm_transport_x(h, ut, Lu, Q_bt, q_e, q_w, active, dt, dx, it)
        out[f"ppm_transport_it{it}"] = dict(h=h, ut=ut, L=Lu, Q_bt=Q_bt, q_e=q_e, q_w=q_w, active=active, dt=dt,
                                            dx=dx, max_iter=it, Qx=Qx)
    # outflow limiter: a calm case (nothing to limit) and one with strong outflow from thin layers
    area = dx * rng.uniform(900.0, 1100.0, (ny, nx))
    hz = np.where(active[None], np.nan_to_num(h), 0.0)
    for name, amp in (("calm", 0.02), ("limited", 0.2), ("heavy", 0.3), ("strong", 3.0)):
        Qx = rng.normal(0.0, 1.0, (n, ny, nx + 1)) * amp * 1e3 * np.concatenate([hz[..., :1], hz], axis=-1)
        Qy = rng.normal(0.0, 1.0, (n, ny + 1, nx)) * amp * 1e3 * np.concatenate([hz[:, :1], hz], axis=1)
        fx = np.zeros((ny, nx + 1), bool)
        fx[:, 1:-1] = active[:, 1:] & active[:, :-1]
        fy = np.zeros((ny + 1, nx), bool)
        fy[1:-1] = active[1:] & active[:-1]
        Qx *= fx
        Qy *= fy
        for per in ((False, False), (True, False)):
            Qxp, Qyp = Qx.copy(), Qy.copy()
            if per[0]:                                         # flow through the wrap face (cells nx-1 and 0)
                wrapf = active[:, 0] & active[:, -1]
                wq = rng.normal(0.0, 1.0, (n, ny)) * amp * 1e3 * np.minimum(hz[..., 0], hz[..., -1]) * wrapf
                Qxp[..., 0] = Qxp[..., -1] = wq
            try:
                Lx, Ly, nl = ale.limit_outflow(hz, Qxp, Qyp, area, dt, active, periodic=per)
                status = "ok"
            except RuntimeError:
                Lx, Ly, nl, status = Qxp, Qyp, -1, "raised"
            out[f"limit_{name}" + ("_perx" if per[0] else "")] = dict(
                h=hz, Qx=Qxp, Qy=Qyp, area=area, dt=dt, active=active, periodic=np.array(per), Qx_out=Lx,
                Qy_out=Ly, n_limited=nl, status=status)
    # Lagrangian thickness of the limited fluxes (where the limiter finished), and a step too long for the outflow
    Aw = np.where(active, area, 0.0)
    for name in ("limit_calm", "limit_limited", "limit_strong"):
        rec = out[name]
        div = rec["Qx_out"][..., 1:] - rec["Qx_out"][..., :-1] + rec["Qy_out"][:, 1:] - rec["Qy_out"][:, :-1]
        try:
            out["lagrangian_" + name[6:]] = dict(h=hz, divq=div, dt=dt, area=Aw,
                                                  h_dag=ale.lagrangian_thickness(hz, div, dt, Aw), raises=False)
        except RuntimeError:
            out["lagrangian_" + name[6:]] = dict(h=hz, divq=div, dt=dt, area=Aw, raises=True)
    for k, v in out.items():
        if k.startswith(("limit", "lagr")):
            print(k, v.get("status"), v.get("n_limited"), v.get("raises"))
    return out


def layer_transport_cases():
    """The donor-cell layer transport, the freshwater volumes, the Lagrangian thickness at a signed-zero tie and the
    whole ALE layer-transport step (ALELayerTransport.__call__ without open faces; PPM and donor-cell thickness
    fluxes, with and without freshwater, donor cell on a periodic x axis)."""
    from types import SimpleNamespace as NS
    from core.components.freshwater import freshwater_volumes
    from core.components.layer_transport import ALELayerTransport
    out = {}
    rng = np.random.default_rng(71)
    n, ny, nx = 6, 9, 14
    H, active, h, dx, Lu = _producer_state(rng, n, ny, nx)
    q_e, q_w = ale.face_transport_thickness(h, H, active, True)
    ut = rng.normal(0.0, 0.4, (n, ny, nx + 1))
    Q_bt = rng.normal(0.0, 1.0, (ny, nx + 1)) * 5e4
    qe2, qw2 = q_e.copy(), q_w.copy()
    qe2[:, 2, :6] = 0.0                                                   # one side empty: the other side takes R
    qw2[:, 3, 4:9] = 0.0
    qe2[:, 4, 1:3] = qw2[:, 4, 1:3] = 0.0                                 # both empty: R added to nothing
    for name, (a_, b_) in (("upwind", (q_e, q_w)), ("upwind_empty", (qe2, qw2))):
        out[name] = dict(q_e=a_, q_w=b_, ut=ut, L=Lu, Q_bt=Q_bt, Q=ale.upwind_transport_x(a_, b_, ut, Lu, Q_bt))
    # freshwater volumes: thicknesses with the scalar floor (ALE), volumes with a per-column floor (sigma)
    dt = 600.0
    hz = np.where(active[None], np.nan_to_num(h), 0.0)
    area = dx * rng.uniform(900.0, 1100.0, (ny, nx))
    dh = rng.normal(0.0, 0.3, (ny, nx)) * 1e-3 * dt
    dh[1, 2:8] = -hz[-1, 1, 2:8] - rng.uniform(0.0, 2.0, 6)                # evaporation beyond the top layer
    dh[5, 3:6] = -hz[:, 5, 3:6].sum(0) - 1.0                               # more than the whole column
    dh[6, 7] = -hz[-1, 6, 7]                                               # exactly the top layer
    for name, (V, dv, fl) in (("fw_thickness", (hz, dh, ale.DZ_FLOOR)),
                              ("fw_volume", (hz * area[None], dh * area, ale.DZ_FLOOR * area))):
        Vn, nl = freshwater_volumes(V, dv, fl)
        out[name] = dict(V=V, dV=dv, floor=np.broadcast_to(fl, (ny, nx)).copy(), V_new=Vn, n_limited=nl)
    # Lagrangian thickness of a layer that is -0.0 with no divergence (numpy.maximum(-0.0, 0.0) is +0.0)
    Aw = np.where(active, area, 0.0)
    hn = hz.copy()
    hn[2] = -0.0
    div = rng.normal(0.0, 1.0, hz.shape) * 1e-3 * hz * area[None] / dt
    div[2] = 0.0
    out["lagrangian_negzero"] = dict(h=hn, divq=div, dt=dt, area=Aw, h_dag=ale.lagrangian_thickness(hn, div, dt, Aw))
    # the whole ALE layer-transport step
    Lv = rng.uniform(900.0, 1100.0, (ny + 1, nx))
    dy = rng.uniform(900.0, 1100.0, (ny, nx))
    eta, eta_new = rng.uniform(-0.3, 0.3, (ny, nx)), rng.uniform(-0.3, 0.3, (ny, nx))
    u_old, u_new = rng.normal(0.0, 0.1, (n, ny, nx + 1)), rng.normal(0.0, 0.1, (n, ny, nx + 1))
    v_old, v_new = rng.normal(0.0, 0.1, (n, ny + 1, nx)), rng.normal(0.0, 0.1, (n, ny + 1, nx))
    wet_u = np.zeros((ny, nx + 1), bool)
    wet_u[:, 1:-1] = active[:, 1:] & active[:, :-1]
    wet_v = np.zeros((ny + 1, nx), bool)
    wet_v[1:-1] = active[1:] & active[:-1]
    u_old *= wet_u
    u_new *= wet_u
    v_old *= wet_v
    v_new *= wet_v
    Dc = hz.sum(0)                                                         # face depths of the columns' water
    Du = np.zeros((ny, nx + 1))
    Du[:, 1:-1] = np.minimum(Dc[:, 1:], Dc[:, :-1])
    Du *= wet_u
    Dv = np.zeros((ny + 1, nx))
    Dv[1:-1] = np.minimum(Dc[1:], Dc[:-1])
    Dv *= wet_v
    qn, qs = ale.face_transport_thickness(hz.swapaxes(1, 2), H.T, active.T, True)
    wu = face_fractions(0.5 * (q_e + q_w))
    wv = face_fractions(0.5 * (qn + qs)).swapaxes(1, 2)
    fw = rng.normal(0.0, 1.0, (ny, nx)) * 2e-6
    for name, flux, per, with_fw, amp in (("lt_ppm", "ppm", (), False, 1.0), ("lt_upwind", "upwind", (), False, 1.0),
                                          ("lt_ppm_fw", "ppm", (), True, 1.0),
                                          ("lt_upwind_perx", "upwind", ("x",), False, 1.0),
                                          ("lt_ppm_strong", "ppm", (), False, 6.0),
                                          ("lt_upwind_strong", "upwind", (), False, 6.0)):
        fs = NS(theta=0.6, active=active, Lu=Lu, Lv=Lv)
        lt = ALELayerTransport(fs=fs, H=H, area=area, dt=dt, thickness_flux=flux, vi_geom={"dx_t": dx, "dy_t": dy},
                               layer_volumes=lambda e, hh: hh * area[None], ob=None)
        Lu_p, u_o, u_n, wet_up, Du_p, qe_p, qw_p, wu_p = Lu, u_old, u_new, wet_u, Du, q_e, q_w, wu
        if per:
            lt.per = Periodic(per)
            Lu_p = Lu.copy()
            Lu_p[:, -1] = Lu_p[:, 0]                                          # face nx is face 0
            wrap = active[:, 0] & active[:, -1]
            wet_up = wet_u.copy()
            wet_up[:, 0] = wet_up[:, -1] = wrap
            u_o, u_n = u_old.copy(), u_new.copy()
            u_o[..., 0] = u_o[..., -1] = rng.normal(0.0, 0.1, (n, ny)) * wrap
            u_n[..., 0] = u_n[..., -1] = rng.normal(0.0, 0.1, (n, ny)) * wrap
            Du_p = Du.copy()
            Du_p[:, 0] = Du_p[:, -1] = np.minimum(Dc[:, 0], Dc[:, -1]) * wrap
            pe = np.concatenate([hz[..., -1:], hz], axis=-1)
            pw = np.concatenate([hz, hz[..., :1]], axis=-1)
            qe_p, qw_p = q_e.copy(), q_w.copy()
            qe_p[..., 0] = qe_p[..., -1] = (pe[..., 0] * wrap)
            qw_p[..., 0] = qw_p[..., -1] = (pw[..., -1] * wrap)
            wu_p = face_fractions(0.5 * (qe_p + qw_p))
            fs.Lu = Lu_p
        u_o, u_n, v_o, v_n = u_o * amp, u_n * amp, v_old * amp, v_new * amp
        st = NS(h=hz, u=u_o, v=v_o, eta=eta)
        fluxes = NS(wet_u=wet_up, wet_v=wet_v, Du=Du_p, Dv=Dv, fw=fw if with_fw else None)
        lf = lt(st, eta_new, u_n, v_n, fluxes, 0.5, (), wu_p, wv, qe_p, qw_p, qn, qs)
        rec = dict(thickness_flux=flux, periodic=np.array(per, dtype=str), theta=0.6, theta_bc=0.5, dt=dt, H=H,
                   area=area, active=active, Lu=Lu_p, Lv=Lv, dx_t=dx, dy_t=dy, h=hz, u=u_o, v=v_o, eta=eta,
                   eta_new=eta_new, u_new=u_n, v_new=v_n, wet_u=wet_up, wet_v=wet_v, Du=Du_p, Dv=Dv, wu=wu_p,
                   wv=wv, qe=qe_p, qw=qw_p, qn=qn, qs=qs, Qx=lf.Qx, Qy=lf.Qy, V0=lf.V0, V1=lf.V1, ok=lf.ok,
                   h_dagger=lf.h_dagger, n_limited=lf.n_limited)
        if with_fw:
            rec.update(fw=fw, V_fw=lf.V_fw, h_fw=lf.h_fw)
        out[name] = rec
        print(name, "limited", lf.n_limited)
    return out


def regrid_columns_cases():
    """``regrid_columns`` itself (regrid.py:345-395): the z*, sigma and hybrid rules on a given wet mask (NaN in the
    other columns), and the hybrid rule on a source of another layer count (``n_out``: the finer data levels of an
    initial state, and a coarser source), with and without the shallow sigma window."""
    out = {}
    rng = np.random.default_rng(91)
    ny, nx = 7, 9

    class _EOS:
        @staticmethod
        def density(T, S):
            return 1027.0 * (1.0 - 2e-4 * (T - 10.0) + 7.6e-4 * (S - 35.0))

    H = rng.uniform(20.0, 400.0, (ny, nx))
    H[1, 2] = 3.0                                                     # shallower than the sigma zone
    eta = rng.uniform(-0.5, 0.5, (ny, nx))
    wet = rng.random((ny, nx)) > 0.15
    for name, n_src, m in (("rc_hybrid_fine", 40, 12), ("rc_hybrid_coarse", 8, 15), ("rc_hybrid_same", 12, 12)):
        D = H + eta
        # source layers: thicker towards the bed, a few nearly massless, T warm at the surface with a jump
        w = rng.uniform(0.5, 1.5, (n_src, ny, nx))
        w[rng.random((n_src, ny, nx)) < 0.08] = 1e-4
        h = w / w.sum(0) * D[None]
        z = np.cumsum(h, axis=0) - 0.5 * h                                  # height above the bed
        T = 4.0 + 18.0 * np.clip(z / 300.0, 0, 1) + np.where(z > 0.6 * D[None], 2.0, 0.0)
        S = 35.0 - 0.5 * np.clip(z / 300.0, 0, 1)
        rho = _EOS.density(T, S)
        rho_t = rg.target_densities(rho[::-1, 3, 3], m, n_light=2)
        dz_top = np.concatenate([np.full(m // 2, 5.0), np.full(m - m // 2, 30.0)])
        dsigma = np.full(m, 1.0 / m)
        for variant, extra in (("", {}), ("_window", {"dsigma": dsigma, "d_sigma": 5.0, "d_hybrid": 60.0})):
            params = {"dz_top": dz_top, "rho_target": rho_t, "max_h_top": np.full(m, 60.0), "h_min": 0.05, **extra}
            zw = rg.regrid_columns("hybrid", H, eta, h, rho, params, wet, n_out=m)
            out[name + variant] = dict(rule="hybrid", H=H, eta=eta, h=h, rho=rho, wet=wet, n_out=m,
                                       dz_top=dz_top, rho_target=rho_t, max_h_top=params["max_h_top"],
                                       dsigma=params.get("dsigma", np.full(m, 1.0 / m)),
                                       d_sigma=params.get("d_sigma", 0.0), d_hybrid=params.get("d_hybrid", 0.0),
                                       h_min=params["h_min"], keep=True, zw=zw)
    n = 10
    h = rng.uniform(1.0, 10.0, (n, ny, nx))
    for rule, params in (("zstar", {"dz_top": rng.uniform(2.0, 20.0, n)}),
                         ("sigma", {"dsigma": rng.dirichlet(np.ones(n))})):
        zw = rg.regrid_columns(rule, H, eta, h, None, params, wet)
        out["rc_" + rule] = dict(rule=rule, H=H, eta=eta, h=h, wet=wet, zw=zw, **params)
    return out


def layer_transport_ext_cases():
    """The whole ALE layer-transport step with the PPM thickness flux on a periodic x axis and on periodic x and y
    axes (the reference pads its inputs by four wrapped cells and crops), and with open edges (the Flather split of
    OpenBoundary.open_face_transports, PPM and donor cell)."""
    from types import SimpleNamespace as NS
    from core.components.layer_transport import ALELayerTransport
    from core.components.open_boundary import OpenBoundary
    out = {}
    rng = np.random.default_rng(83)
    n, ny, nx = 6, 11, 14
    H, active, h, dx, Lu = _producer_state(rng, n, ny, nx)
    hz = np.where(active[None], np.nan_to_num(h), 0.0)
    dt = 600.0
    area = dx * rng.uniform(900.0, 1100.0, (ny, nx))
    Lv = rng.uniform(900.0, 1100.0, (ny + 1, nx))
    dy = rng.uniform(900.0, 1100.0, (ny, nx))
    eta, eta_new = rng.uniform(-0.3, 0.3, (ny, nx)), rng.uniform(-0.3, 0.3, (ny, nx))
    Dc = hz.sum(0)
    for name, flux, per, open_ in (("lt_ppm_perx", "ppm", ("x",), ()), ("lt_ppm_perxy", "ppm", ("x", "y"), ()),
                                   ("lt_ppm_open", "ppm", (), ("west", "north")),
                                   ("lt_upwind_open", "upwind", (), ("east", "south")),
                                   ("lt_ppm_perx_open_sn", "ppm", ("x",), ("south", "north"))):
        px, py = "x" in per, "y" in per
        wrapx = active[:, 0] & active[:, -1]
        wrapy = active[0, :] & active[-1, :]
        wet_u = np.zeros((ny, nx + 1), bool)
        wet_u[:, 1:-1] = active[:, 1:] & active[:, :-1]
        wet_v = np.zeros((ny + 1, nx), bool)
        wet_v[1:-1] = active[1:] & active[:-1]
        if px:
            wet_u[:, 0] = wet_u[:, -1] = wrapx
        if py:
            wet_v[0] = wet_v[-1] = wrapy
        u_old, u_new = rng.normal(0.0, 0.1, (n, ny, nx + 1)), rng.normal(0.0, 0.1, (n, ny, nx + 1))
        v_old, v_new = rng.normal(0.0, 0.1, (n, ny + 1, nx)), rng.normal(0.0, 0.1, (n, ny + 1, nx))
        if px:
            u_old[..., -1], u_new[..., -1] = u_old[..., 0], u_new[..., 0]
        if py:
            v_old[:, -1], v_new[:, -1] = v_old[:, 0], v_new[:, 0]
        u_old *= wet_u
        u_new *= wet_u
        v_old *= wet_v
        v_new *= wet_v
        Du = np.zeros((ny, nx + 1))
        Du[:, 1:-1] = np.minimum(Dc[:, 1:], Dc[:, :-1])
        Dv = np.zeros((ny + 1, nx))
        Dv[1:-1] = np.minimum(Dc[1:], Dc[:-1])
        if px:
            Du[:, 0] = Du[:, -1] = np.minimum(Dc[:, 0], Dc[:, -1])
        if py:
            Dv[0] = Dv[-1] = np.minimum(Dc[0], Dc[-1])
        Du *= wet_u
        Dv *= wet_v
        Lu_p, Lv_p = Lu.copy(), Lv.copy()
        if px:
            Lu_p[:, -1] = Lu_p[:, 0]                                          # face nx is face 0
        if py:
            Lv_p[-1] = Lv_p[0]
        q_e, q_w = ale.face_transport_thickness(hz, H, active, True)
        qn, qs = ale.face_transport_thickness(hz.swapaxes(1, 2), H.T, active.T, True)
        if px:
            pe = np.concatenate([hz[..., -1:], hz], axis=-1)
            pw = np.concatenate([hz, hz[..., :1]], axis=-1)
            q_e[..., 0] = q_e[..., -1] = pe[..., 0] * wrapx
            q_w[..., 0] = q_w[..., -1] = pw[..., -1] * wrapx
        if py:
            hzt = hz.swapaxes(1, 2)
            pn = np.concatenate([hzt[..., -1:], hzt], axis=-1)
            ps = np.concatenate([hzt, hzt[..., :1]], axis=-1)
            qn[..., 0] = qn[..., -1] = pn[..., 0] * wrapy
            qs[..., 0] = qs[..., -1] = ps[..., -1] * wrapy
        qn, qs = np.ascontiguousarray(qn), np.ascontiguousarray(qs)
        wu = face_fractions(0.5 * (q_e + q_w))
        wv = face_fractions(0.5 * (qn + qs)).swapaxes(1, 2)
        fs = NS(theta=0.6, active=active, Lu=Lu_p, Lv=Lv_p)
        ob = None
        fluxes = NS(wet_u=wet_u, wet_v=wet_v, Du=Du, Dv=Dv, fw=None)
        rec_open = {}
        if open_:
            ob = OpenBoundary()
            ob.open, ob.fs, ob.theta_bc = tuple(open_), fs, 0.5
            # open face depths and Flather volume fluxes of the free surface on the edge faces
            oDu, oDv = np.zeros((ny, nx + 1)), np.zeros((ny + 1, nx))
            oQu, oQv = np.zeros((ny, nx + 1)), np.zeros((ny + 1, nx))
            oDu[:, 0], oDu[:, -1] = Dc[:, 0] * active[:, 0], Dc[:, -1] * active[:, -1]
            oDv[0], oDv[-1] = Dc[0] * active[0], Dc[-1] * active[-1]
            oQu[:, [0, -1]] = rng.normal(0.0, 1.0, (ny, 2)) * 2e3 * (oDu[:, [0, -1]] > 0)
            oQv[[0, -1]] = rng.normal(0.0, 1.0, (2, nx)) * 2e3 * (oDv[[0, -1]] > 0)
            # interior-cell velocities on the open faces (the wet flag is False there)
            for e in open_:
                if e == "west":
                    u_new[..., 0] = rng.normal(0.0, 0.1, (n, ny)) * active[:, 0]
                    u_old[..., 0] = rng.normal(0.0, 0.1, (n, ny)) * active[:, 0]
                elif e == "east":
                    u_new[..., -1] = rng.normal(0.0, 0.1, (n, ny)) * active[:, -1]
                    u_old[..., -1] = rng.normal(0.0, 0.1, (n, ny)) * active[:, -1]
                elif e == "south":
                    v_new[:, 0] = rng.normal(0.0, 0.1, (n, nx)) * active[0]
                    v_old[:, 0] = rng.normal(0.0, 0.1, (n, nx)) * active[0]
                else:
                    v_new[:, -1] = rng.normal(0.0, 0.1, (n, nx)) * active[-1]
                    v_old[:, -1] = rng.normal(0.0, 0.1, (n, nx)) * active[-1]
            fluxes = NS(wet_u=wet_u, wet_v=wet_v, Du=Du, Dv=Dv, fw=None, open_Du=oDu, open_Dv=oDv, open_Qu=oQu,
                        open_Qv=oQv)
            rec_open = dict(open=np.array(open_, dtype=str), open_Du=oDu, open_Dv=oDv, open_Qu=oQu, open_Qv=oQv)
        lt = ALELayerTransport(fs=fs, H=H, area=area, dt=dt, thickness_flux=flux, vi_geom={"dx_t": dx, "dy_t": dy},
                               layer_volumes=lambda e, hh: hh * area[None], ob=ob)
        if per:
            lt.per = Periodic(per)
        st = NS(h=hz, u=u_old, v=v_old, eta=eta)
        lf = lt(st, eta_new, u_new, v_new, fluxes, 0.5, tuple(open_), wu, wv, q_e, q_w, qn, qs)
        rec = dict(thickness_flux=flux, periodic=np.array(per, dtype=str), theta=0.6, theta_bc=0.5, dt=dt, H=H,
                   area=area, active=active, Lu=Lu_p, Lv=Lv_p, dx_t=dx, dy_t=dy, h=hz, u=u_old, v=v_old, eta=eta,
                   eta_new=eta_new, u_new=u_new, v_new=v_new, wet_u=wet_u, wet_v=wet_v, Du=Du, Dv=Dv, wu=wu,
                   wv=wv, qe=q_e, qw=q_w, qn=qn, qs=qs, Qx=lf.Qx, Qy=lf.Qy, V0=lf.V0, V1=lf.V1, ok=lf.ok,
                   h_dagger=lf.h_dagger, n_limited=lf.n_limited, **rec_open)
        out[name] = rec
        print(name, "limited", lf.n_limited)
    return out


def save(name, cases):
    flat = {}
    for case, rec in cases.items():
        for k, v in rec.items():
            flat[f"{case}/{k}"] = np.asarray(v)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **flat)
    print(f"{path}: {len(cases)} cases, {os.path.getsize(path) / 1e3:.0f} kB")


if __name__ == "__main__":
    threads.set_threads(1)
    which = sys.argv[2:] or ["fct", "rk3", "rk3_ext", "helpers", "kernels", "remap", "neighbours", "producers",
                             "layer_transport",
                             "layer_transport_ext", "regrid_columns"]
    makers = {"fct": fct_cases, "rk3": rk3_cases, "rk3_ext": rk3_ext_cases, "helpers": helper_cases,
              "kernels": kernel_cases, "remap": remap_cases,
              "neighbours": neighbour_cases, "producers": producer_cases, "layer_transport": layer_transport_cases,
              "layer_transport_ext": layer_transport_ext_cases, "regrid_columns": regrid_columns_cases}
    for name in which:
        save(name, makers[name]())
