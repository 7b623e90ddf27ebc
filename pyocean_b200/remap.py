"""
Conservative vertical remap with the reference's interface (core/vertical/remap.py:306-427), computed on the GPU.

``remap_columns(h_src, f_src, h_tgt, scheme, wet)`` is the drop-in for ``core.vertical.remap.remap_columns``: every
wet column of f_src (N0, ny, nx) goes from thicknesses h_src to h_tgt (N1, ny, nx); dry columns are copied when
N0 == N1, else NaN.  It also takes a stack of fields (nf, N0, ny, nx) remapped in one launch (the ALE step remaps
every tracer of the stack with the same thicknesses).  ``remap_column`` is the single-column form.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._device import Converter, shape_of

PCM, PLM, PPM_H4 = _lib.PCM, _lib.PLM, _lib.PPM_H4
SCHEMES = {"pcm": PCM, "plm": PLM, "ppm_h4": PPM_H4}
MAX_LAYERS = 256


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
    cv = Converter(h_src, f_src, h_tgt, wet)
    hsd, fsd, htd = cv.f64(h_src), cv.f64(f_src), cv.f64(h_tgt)
    wd = cv.u8(wet, (ny, nx))
    out = cv.empty((nf, n1, ny, nx) if stacked else (n1, ny, nx))
    rc = _lib.lib().pocean_remap_columns_f64(hsd.data_ptr(), fsd.data_ptr(), htd.data_ptr(), wd.data_ptr(), n0, n1,
                                             ny, nx, nf, int(scheme), out.data_ptr(), cv.stream())
    _lib.check(rc, "remap_columns")
    return cv.out(out)


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
