"""
The vertical-coordinate neighbours of the tracer step, with the reference's interface, computed on the GPU.

``ALECoordinate`` mirrors the part of ``core.components.vertical_coordinate.ALECoordinate`` that the ALE tracer
step calls (vertical_coordinate.py:69-111, 142-153): ``regrid_remap`` (regrid to the z* or sigma target, then the
conservative remap of every field: a regrid launch writes the target thicknesses, the column remap follows),
``regrid`` and ``remap_faces`` (the velocity remap in fraction space), for the rules 'zstar', 'sigma' and 'hybrid'
(HYCOM1 with isopycnal targets, a z* floor and an optional shallow sigma window).  ``face_fractions`` is
``core.vertical.ale.face_fractions``.  Arrays are NumPy (copied in and out) or CUDA torch tensors (results stay on
the device).  The hybrid rule's layer densities come from the model's equation of state (``eos``, the reference's
EOS component, outside this path) or are given directly (``rho=``).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._device import Converter, shape_of

H_MIN = 1e-3                                    # core/vertical/regrid.py:41
RULES = {"zstar": _lib.REGRID_ZSTAR, "sigma": _lib.REGRID_SIGMA}
P_REF = 2e7                                     # vertical_coordinate.py:37, reference pressure of the hybrid density


class ALECoordinate:
    """z* / sigma regrid + remap and the velocity remap of an ALE vertical coordinate, on B200.

    ``H`` (ny, nx) depth [m] (NaN on land reads as 0), ``active`` (ny, nx) water mask, ``regrid_rule`` 'zstar',
    'sigma' or 'hybrid', ``regrid_params`` as ``core.vertical.regrid.regrid_columns`` takes them (``dz_top``
    surface first, ``dsigma`` bed first, ``rho_target`` surface first, ``max_h_top``, ``d_sigma``, ``d_hybrid``,
    ``h_min``, ``keep_isopycnal``), ``remap_code`` 0 / 1 / 2 (PCM / PLM / PPM_H4), and for 'hybrid' the equation of
    state ``eos`` (``linear``, ``density(T, S)``, ``potential_density(T, S, p_ref)``) with ``p_ref`` — the attributes
    of the reference's component."""

    def __init__(self, H, active, regrid_rule: str, regrid_params: dict, remap_code: int = _lib.PPM_H4, eos=None,
                 p_ref: float = P_REF) -> None:
        if regrid_rule not in ("zstar", "sigma", "hybrid"):
            raise ValueError(f"unknown rule {regrid_rule!r}; use 'zstar', 'sigma' or 'hybrid'")
        self.H, self.active = H, active
        self.regrid_rule, self.regrid_params, self.remap_code = regrid_rule, dict(regrid_params), int(remap_code)
        self.eos, self.p_ref = eos, float(p_ref)

    @classmethod
    def like(cls, ref) -> "ALECoordinate":
        """The GPU coordinate of a reference ALECoordinate instance (reads H, active, rule, params, remap code, eos)."""
        return cls(ref.H, ref.active, ref.regrid_rule, ref.regrid_params, ref.remap_code, getattr(ref, "eos", None),
                   getattr(ref, "p_ref", P_REF))

    def _param(self, key: str, n: int, default=None) -> np.ndarray:
        if key not in self.regrid_params and default is None:
            raise ValueError(f"regrid_columns({self.regrid_rule!r}) needs params[{key!r}]")
        v = np.ascontiguousarray(self.regrid_params.get(key, default), dtype=np.float64)
        if v.shape != (n,):
            raise ValueError(f"{key} must have {n} entries, got {v.shape}")
        return v

    def regrid_density(self, T, S=None):
        """Layer density the hybrid rule follows (vertical_coordinate.py:80-94): the equation of state's density for
        a linear EOS, the potential density at ``p_ref`` otherwise; computed by the given ``eos``."""
        if self.eos is None:
            raise ValueError("the hybrid rule needs the layer densities: give eos= or rho=")
        if self.eos.linear:
            return self.eos.density(T, S)
        return self.eos.potential_density(T, S, self.p_ref)

    def regrid_remap(self, eta, h_src, fields, T=None, S=None, rho=None):
        """(h_new, [remap_columns(h_src, f, h_new, remap_code, wet) for f in fields]) with the rule's target grid
        (vertical_coordinate.py:69-78); ``fields`` a list of (N, ny, nx) arrays or one (nf, N, ny, nx) stack.
        'hybrid': the densities ``rho`` (N, ny, nx, bed first), else ``regrid_density(T, S)``."""
        stacked = not isinstance(fields, (list, tuple))
        h_new, outs = self._run(eta, h_src, fields if stacked else list(fields), T, S, rho)
        return h_new, (outs if stacked else list(outs))

    def regrid(self, eta, h, T=None, wet=None, S=None, rho=None):
        """New layer thicknesses of the rule where wet (active, D > 0, water in the column), else h
        (vertical_coordinate.py:96-111; ``wet`` is always the reference's default mask)."""
        if wet is not None:
            raise NotImplementedError("regrid with a caller-given wet mask; the GPU regrid derives it as the "
                                      "reference's default")
        return self._run(eta, h, None, T, S, rho)[0]

    def _run(self, eta, h_src, fields, T=None, S=None, rho=None):
        n, ny, nx = shape_of(h_src)
        hybrid = self.regrid_rule == "hybrid"
        if hybrid:
            d_hybrid = float(self.regrid_params.get("d_hybrid", 0.0))
            coords = (self._param("rho_target", n + 1), self._param("dz_top", n),
                      self._param("max_h_top", n, np.full(n, np.inf)),
                      self._param("dsigma", n, None if d_hybrid > 0.0 else np.full(n, 1.0 / n)))
            if rho is None:
                if T is None:
                    raise ValueError("regrid_columns('hybrid') needs the layer densities rho")
                rho = self.regrid_density(T, S)
        else:
            coords = (self._param("dz_top" if self.regrid_rule == "zstar" else "dsigma", n),)
        if fields is None:
            arrays = ()
        elif isinstance(fields, list):
            arrays = tuple(fields)
        else:
            arrays = (fields,)
        cv = Converter(h_src, eta, self.H, *arrays, *((rho,) if hybrid else ()))
        hsd = cv.f64(h_src)
        Hd = cv.f64(self.H, (ny, nx))
        ed = cv.f64(eta, (ny, nx))
        act = cv.u8(self.active, (ny, nx))
        cds = [cv.f64(c) for c in coords]
        if fields is None:
            nf, fd = 0, None
        elif isinstance(fields, list):
            nf = len(fields)
            fd = torch.stack([cv.f64(f, (n, ny, nx)) for f in fields]) if nf else None
        else:
            fd = cv.f64(fields)
            nf = fd.shape[0]
        h_new = cv.empty((n, ny, nx))
        wet = torch.empty((ny, nx), dtype=torch.uint8, device=cv.device)
        out = cv.empty((nf, n, ny, nx)) if nf else None
        bad = torch.zeros(1, dtype=torch.int32, device=cv.device)
        h_min = float(self.regrid_params.get("h_min", H_MIN))
        tail = (None if fd is None else fd.data_ptr(), n, ny, nx, nf, self.remap_code, h_new.data_ptr(),
                wet.data_ptr(), None if out is None else out.data_ptr(), bad.data_ptr(), cv.stream())
        if hybrid:
            rd = cv.f64(rho, (n, ny, nx))
            rc = _lib.lib().pocean_regrid_hybrid_remap_f64(
                Hd.data_ptr(), ed.data_ptr(), hsd.data_ptr(), act.data_ptr(), rd.data_ptr(),
                *(c.data_ptr() for c in cds), float(self.regrid_params.get("d_sigma", 0.0)), d_hybrid, h_min,
                int(bool(self.regrid_params.get("keep_isopycnal", True))), *tail)
        else:
            rc = _lib.lib().pocean_regrid_remap_f64(RULES[self.regrid_rule], Hd.data_ptr(), ed.data_ptr(),
                                                    hsd.data_ptr(), act.data_ptr(), cds[0].data_ptr(), h_min, *tail)
        _lib.check(rc, "regrid_remap")
        if int(bad.item()):
            if hybrid:
                raise ValueError("hybrid needs finite densities in wet columns and H > 0 unless it has a shallow "
                                 "sigma zone (d_hybrid > 0)")
            raise ValueError("z* needs H > 0 in every wet column (cells that can dry: sigma, or hybrid with "
                             "d_hybrid > 0)")
        if out is None:
            return cv.out(h_new), None
        if isinstance(fields, list):
            return cv.out(h_new), [cv.out(out[m]) for m in range(nf)]
        return cv.out(h_new), cv.out(out)

    def remap_faces(self, vel, hf_src, hf_tgt, w_tgt=None):
        """Face velocities remapped from the face layers hf_src to hf_tgt in fraction space (Σ w u conserved,
        vertical_coordinate.py:142-153).  ``vel`` (N, ny, nf) or a stack (m, N, ny, nf)."""
        return remap_faces(vel, hf_src, hf_tgt, self.remap_code, w_tgt)


def regrid_columns(rule: str, H, eta, h, rho, params: dict, wet, n_out: int | None = None):
    """Target interface heights zw (N+1, ny, nx), bed first, of the rule 'zstar', 'sigma' or 'hybrid'
    (core/vertical/regrid.py:345-395, same arguments): N = n_out, by default the source layer count; the hybrid
    rule may regrid a source of another count (the data levels of an initial state).  NaN in the columns that are
    not wet.  Raises ValueError where the reference does."""
    if rule not in ("zstar", "sigma", "hybrid"):
        raise ValueError(f"unknown rule {rule!r}; use 'zstar', 'sigma' or 'hybrid'")
    required = {"zstar": ("dz_top",), "sigma": ("dsigma",), "hybrid": ("dz_top", "rho_target")}[rule]
    if rule == "hybrid" and float(params.get("d_hybrid", 0.0)) > 0.0:
        required += ("dsigma",)
    for key in required:
        if key not in params:
            raise ValueError(f"regrid_columns({rule!r}) needs params[{key!r}]")
    if rule == "hybrid" and rho is None:
        raise ValueError("regrid_columns('hybrid') needs the layer densities rho")
    n, ny, nx = shape_of(h)
    m = n if n_out is None else int(n_out)
    if m != n and rule != "hybrid":
        raise ValueError("n_out != the source layer count is only for rule 'hybrid'")
    cv = Converter(H, eta, h, wet, *(() if rho is None else (rho,)))
    Hd, ed, hd, wd = cv.f64(H, (ny, nx)), cv.f64(eta, (ny, nx)), cv.f64(h), cv.u8(wet, (ny, nx))
    w = wd.bool()
    Hw, Dw = Hd[w], (Hd + ed)[w]
    if not bool(torch.isfinite(Hw).all() & torch.isfinite(Dw).all() & (Dw > 0).all()):
        raise ValueError("wet columns need finite H and D = H + eta > 0")
    if rule == "zstar" and not bool((Hw > 0).all()):
        raise ValueError("z* needs H > 0 in every wet column (cells that can dry: sigma, or hybrid with d_hybrid > 0)")
    rd = None
    if rule == "hybrid":
        if float(params.get("d_hybrid", 0.0)) <= 0 and bool((Hw <= 0).any()):
            raise ValueError("hybrid needs H > 0 unless it has a shallow sigma zone (d_hybrid > 0); columns with "
                             "H <= 0 then stay sigma at any depth")
        rd = cv.f64(rho, (n, ny, nx))
        if not bool(torch.isfinite(rd[:, w]).all()):
            raise ValueError("non-finite density in a wet column")
    f = lambda key, default, size: cv.f64(np.asarray(params.get(key, default), float), (size,))   # noqa: E731
    dz = f("dz_top", np.ones(m), m)
    ds = f("dsigma", np.full(m, 1.0 / m), m)
    rt = f("rho_target", np.zeros(m + 1), m + 1)
    mx = f("max_h_top", np.full(m, np.inf), m)
    zw = cv.empty((m + 1, ny, nx))
    code = {"zstar": 0, "sigma": 1, "hybrid": 2}[rule]
    _lib.check(_lib.lib().pocean_regrid_columns_f64(
        code, Hd.data_ptr(), ed.data_ptr(), hd.data_ptr(), None if rd is None else rd.data_ptr(), wd.data_ptr(),
        dz.data_ptr(), ds.data_ptr(), rt.data_ptr(), mx.data_ptr(), float(params.get("d_sigma", 0.0)),
        float(params.get("d_hybrid", 0.0)), float(params.get("h_min", H_MIN)),
        int(bool(params.get("keep_isopycnal", True))), n, m, ny, nx, zw.data_ptr(), cv.stream()), "regrid_columns")
    return cv.out(zw)


def remap_faces(vel, hf_src, hf_tgt, scheme: int, w_tgt=None):
    vs, hs = shape_of(vel), shape_of(hf_src)
    if len(hs) != 3 or vs[-3:] != hs or len(vs) not in (3, 4) or shape_of(hf_tgt) != hs:
        raise ValueError(f"face arrays must share (N, ny, nf): vel {vs}, hf_src {hs}, hf_tgt {shape_of(hf_tgt)}")
    n, ny, nf = hs
    m = vs[0] if len(vs) == 4 else 1
    cv = Converter(vel, hf_src, hf_tgt, w_tgt)
    vd, hsd, htd = cv.f64(vel), cv.f64(hf_src), cv.f64(hf_tgt)
    wd = None if w_tgt is None else cv.f64(w_tgt, hs)
    out = cv.empty(vs)
    rc = _lib.lib().pocean_remap_faces_f64(vd.data_ptr(), hsd.data_ptr(), htd.data_ptr(),
                                           None if wd is None else wd.data_ptr(), n, ny, nf, m, int(scheme),
                                           out.data_ptr(), cv.stream())
    _lib.check(rc, "remap_faces")
    return cv.out(out)


def face_fractions(hf):
    """w_k = h_k,f / Σ_k h_k,f, uniform 1/N on faces with no water (core/vertical/ale.py:895-902)."""
    if len(shape_of(hf)) != 3:
        raise ValueError("face_fractions expects (N, ny, nf) face thicknesses")
    n, ny, nf = shape_of(hf)
    cv = Converter(hf)
    hd = cv.f64(hf)
    w = cv.empty((n, ny, nf))
    _lib.check(_lib.lib().pocean_face_fractions_f64(hd.data_ptr(), n, ny, nf, w.data_ptr(), cv.stream()),
               "face_fractions")
    return cv.out(w)
