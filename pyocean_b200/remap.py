"""
Conservative vertical remap with the reference's interface (core/vertical/remap.py:306-427), computed on the GPU.

``remap_columns(h_src, f_src, h_tgt, scheme, wet)`` is the drop-in for ``core.vertical.remap.remap_columns``: every
wet column of f_src (N0, ny, nx) goes from thicknesses h_src to h_tgt (N1, ny, nx); dry columns are copied when
N0 == N1, else NaN.  It also takes a stack of fields (nf, N0, ny, nx) remapped in one launch (the ALE step remaps
every tracer of the stack with the same thicknesses).  ``remap_column`` is the single-column form, ``reconstruct``
the per-cell polynomials of one column or of many.  Pinned host tensors are remapped in row blocks with the copies
overlapping the kernels (``_pipeline``).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import _pipeline as _pl
from ._device import Converter, shape_of

PCM, PLM, PPM_H4 = _lib.PCM, _lib.PLM, _lib.PPM_H4
SCHEMES = {"pcm": PCM, "plm": PLM, "ppm_h4": PPM_H4}
MAX_LAYERS = 256
H_NEGLECT = 1e-30          # remap.py:42-43, the negligible thicknesses the kernels are built with
H_NEGLECT_EDGE = 1e-10


def remap_columns(h_src, f_src, h_tgt, scheme: int, wet):
    """Remap every wet column of f_src (N0, ny, nx) or (nf, N0, ny, nx) from h_src to h_tgt [m]."""
    hs, ht, fs = shape_of(h_src), shape_of(h_tgt), shape_of(f_src)
    if len(hs) != 3 or len(ht) != 3 or hs[1:] != ht[1:]:
        raise ValueError(f"thicknesses must be (N0, ny, nx) and (N1, ny, nx), got {hs} and {ht}")
    stacked = len(fs) == 4
    if fs[-3:] != hs or len(fs) not in (3, 4):
        raise ValueError(f"field shape {fs} does not match the source thicknesses {hs}")
    n0, ny, nx = hs
    n1 = ht[0]
    nf = fs[0] if stacked else 1
    if _pl.pinned(h_src, f_src, h_tgt) and _wet_pinned(wet, ny, nx) and \
            all(a.dtype == torch.float64 for a in (h_src, f_src, h_tgt)) and \
            8 * nf * (n0 + n1) * ny * nx >= _pl.MIN_BYTES and ny >= 8:
        return _remap_pipelined(h_src, f_src, h_tgt, wet, n0, n1, ny, nx, nf, int(scheme), stacked)
    cv = Converter(h_src, f_src, h_tgt, wet)
    hsd, fsd, htd = cv.f64(h_src), cv.f64(f_src), cv.f64(h_tgt)
    wd = cv.u8(wet, (ny, nx))
    out = cv.empty((nf, n1, ny, nx) if stacked else (n1, ny, nx))
    rc = _lib.lib().pocean_remap_columns_f64(hsd.data_ptr(), fsd.data_ptr(), htd.data_ptr(), wd.data_ptr(), n0, n1,
                                             ny, nx, nf, int(scheme), out.data_ptr(), cv.stream())
    _lib.check(rc, "remap_columns")
    return cv.out(out)


def _wet_pinned(wet, ny: int, nx: int) -> bool:
    return (isinstance(wet, torch.Tensor) and not wet.is_cuda and wet.is_pinned() and wet.is_contiguous() and
            tuple(wet.shape) == (ny, nx) and wet.dtype in (torch.bool, torch.uint8))


def _remap_pipelined(h_src, f_src, h_tgt, wet, n0, n1, ny, nx, nf, scheme, stacked, f_dev=None, blocks=None):
    """remap_columns of pinned host tensors in row blocks of columns: block b's thicknesses and fields go to the
    device on one stream while block b-1 is remapped on another and block b-2's result comes back on a third.
    ``f_dev``: the fields are already on the device (nf, n0, ny, nx), made by work ordered on the compute stream;
    their rows are copied there instead of uploaded (``f_src`` unused).  ``blocks``: (full blocks, tail), default
    ``_pipeline.REMAP_BLOCKS``."""
    dev = _pl.device_now()
    s_in, s_cmp, s_out = _pl.streams(dev)
    s_in.wait_stream(torch.cuda.current_stream(dev))
    out = torch.empty((nf, n1, ny, nx) if stacked else (n1, ny, nx), dtype=torch.float64, pin_memory=True)
    L, row, keep = _lib.lib(), 8 * nx, []
    for j0, j1 in _pl.row_blocks(ny, *(blocks or _pl.REMAP_BLOCKS)):
        r = j1 - j0
        with torch.cuda.stream(s_in):
            hs = torch.empty((n0, r, nx), dtype=torch.float64, device=dev)
            ht = torch.empty((n1, r, nx), dtype=torch.float64, device=dev)
            fc = torch.empty((nf, n0, r, nx), dtype=torch.float64, device=dev)
            wc = torch.empty((r, nx), dtype=torch.uint8, device=dev)
        _pl.copy2d(hs.data_ptr(), r * row, h_src.data_ptr() + j0 * row, ny * row, r * row, n0, s_in)
        _pl.copy2d(ht.data_ptr(), r * row, h_tgt.data_ptr() + j0 * row, ny * row, r * row, n1, s_in)
        if f_dev is None:
            _pl.copy2d(fc.data_ptr(), r * row, f_src.data_ptr() + j0 * row, ny * row, r * row, nf * n0, s_in)
        _pl.copy2d(wc.data_ptr(), r * nx, wet.data_ptr() + j0 * nx, ny * nx, r * nx, 1, s_in)
        ev = torch.cuda.Event()
        ev.record(s_in)
        s_cmp.wait_event(ev)
        if f_dev is not None:
            fc.record_stream(s_cmp)
            _pl.copy2d(fc.data_ptr(), r * row, f_dev.data_ptr() + j0 * row, ny * row, r * row, nf * n0, s_cmp)
        with torch.cuda.stream(s_cmp):
            oc = torch.empty((nf, n1, r, nx), dtype=torch.float64, device=dev)
        _lib.check(L.pocean_remap_columns_f64(hs.data_ptr(), fc.data_ptr(), ht.data_ptr(), wc.data_ptr(), n0, n1, r,
                                              nx, nf, scheme, oc.data_ptr(), s_cmp.cuda_stream), "remap_columns")
        ev = torch.cuda.Event()
        ev.record(s_cmp)
        s_out.wait_event(ev)
        _pl.copy2d(out.data_ptr() + j0 * row, ny * row, oc.data_ptr(), r * row, r * row, nf * n1, s_out)
        keep += [hs, ht, fc, wc, oc]
    s_out.synchronize()
    if f_dev is not None:
        keep.append(f_dev)
    return out


def remap_column(h_src, u_src, h_tgt, scheme: int, u_tgt=None):
    """Conservative remap of one column (remap.py:306): returns u_tgt (and fills it when given)."""
    n0, n1 = len(h_src), len(h_tgt)
    res = remap_columns(np.reshape(np.asarray(h_src, float), (n0, 1, 1)),
                        np.reshape(np.asarray(u_src, float), (n0, 1, 1)),
                        np.reshape(np.asarray(h_tgt, float), (n1, 1, 1)), scheme, np.ones((1, 1), bool))
    res = np.asarray(res).reshape(n1)
    if u_tgt is not None:
        u_tgt[...] = res
    return res


def reconstruct(h, u, scheme: int, h_neglect: float = H_NEGLECT, h_neglect_edge: float = H_NEGLECT_EDGE,
                coef=None):
    """The polynomial p(xi) = c0 + c1 xi + c2 xi^2 of every cell (remap.py:234-294): h, u of one column (n,) or of
    many (n, ...) give coef (n, 3) or (n, ..., 3); ``coef``, when given, is filled as the reference fills it.  The
    kernels carry the reference's default negligible thicknesses; other values are refused."""
    if h_neglect != H_NEGLECT or h_neglect_edge != H_NEGLECT_EDGE:
        raise ValueError("reconstruct: only the default h_neglect / h_neglect_edge (remap.py:42-43) are built")
    shp = tuple(shape_of(h))
    if tuple(shape_of(u)) != shp or len(shp) < 1:
        raise ValueError(f"reconstruct: h {shp} and u {tuple(shape_of(u))} must have the same shape (n, ...)")
    n = shp[0]
    ncols = int(np.prod(shp[1:])) if len(shp) > 1 else 1
    if n > MAX_LAYERS:
        raise ValueError(f"reconstruct: at most {MAX_LAYERS} cells per column, got {n}")
    if int(scheme) not in (PCM, PLM, PPM_H4):
        raise ValueError(f"reconstruct: unknown scheme {scheme}")
    cv = Converter(h, u)
    hd, ud = cv.f64(h), cv.f64(u)
    out = cv.empty(shp + (3,))
    _lib.check(_lib.lib().pocean_reconstruct_f64(hd.data_ptr(), ud.data_ptr(), n, ncols, int(scheme),
                                                 out.data_ptr(), cv.stream()), "reconstruct")
    res = cv.out(out)
    if coef is not None:
        coef[...] = res
    return res
