"""
A resident ALE tracer step on one GPU: ``advect_fct`` of the stack followed by the remap of every member, with
every buffer allocated once.

This is the device-resident form of the reference's phases 7 and 8 (core/model/driver.py:888-985: the tracer
advection of the stack, then ``ALECoordinate.regrid_remap`` remapping each stack member,
core/components/vertical_coordinate.py:69-78).  All arrays are CUDA tensors; calls are stream-ordered and never
synchronise, so a sequence of steps can be timed with events or captured in a CUDA graph.
"""
from __future__ import annotations

import torch

from . import _lib


class ALETracerStep:
    """advect_fct + PPM_H4 (or PCM / PLM) remap of a (nt, N, ny, nx) stack with preallocated buffers."""

    def __init__(self, nt: int, n: int, ny: int, nx: int, dt: float, flags: int = 0, remap_scheme: int = 2,
                 n_tgt: int | None = None, device=None, mixed: bool = False) -> None:
        self.nt, self.n, self.ny, self.nx = nt, n, ny, nx
        self.n1 = n if n_tgt is None else n_tgt
        self.dt, self.flags, self.remap_scheme = float(dt), int(flags), int(remap_scheme)
        self.mixed = bool(mixed)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        L = _lib.lib()
        self.ws_bytes = L.pocean_advect_fct_workspace_bytes(nt, n, ny, nx)
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
        self.adv_out = torch.empty((nt, n, ny, nx), dtype=torch.float64, device=self.device)
        # 7 FCT passes (face + cell for stages 1 and 2, the stage-3 face pass, coefficients, final); the remap:
        # field pairs (nt >= 2), the odd field (nt odd), the general-column fixup
        self.launches_per_step = 7 + (nt >= 2) + (nt % 2) + 1

    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def advect(self, C, V0, V1, Qx, Qy, ok, out=None, inflow=None) -> torch.Tensor:
        out = self.adv_out if out is None else out
        L = _lib.lib()
        fn = L.pocean_advect_fct_mixed if self.mixed else L.pocean_advect_fct_f64
        rc = fn(C.data_ptr(), V0.data_ptr(), V1.data_ptr(), Qx.data_ptr(),
                                              Qy.data_ptr(), ok.data_ptr(),
                                              None if inflow is None else inflow.data_ptr(), self.nt, self.n,
                                              self.ny, self.nx, self.flags, self.dt, out.data_ptr(), 0, None, None,
                                              self.ws.data_ptr(), self.ws_bytes, self.stream())
        _lib.check(rc, "advect_fct")
        return out

    def remap(self, h_src, f, h_tgt, wet, out) -> torch.Tensor:
        rc = _lib.lib().pocean_remap_columns_f64(h_src.data_ptr(), f.data_ptr(), h_tgt.data_ptr(), wet.data_ptr(),
                                                 self.n, self.n1, self.ny, self.nx, self.nt, self.remap_scheme,
                                                 out.data_ptr(), self.stream())
        _lib.check(rc, "remap_columns")
        return out

    def step(self, C, V0, V1, Qx, Qy, ok, h_src, h_tgt, wet, out) -> torch.Tensor:
        """out = remap(advect_fct(C)); ``out`` must not alias ``C``."""
        return self.remap(h_src, self.advect(C, V0, V1, Qx, Qy, ok), h_tgt, wet, out)


def ale_tracer_step(adv, C, V0, V1, Qx, Qy, ok, h_src, h_tgt, scheme: int, wet):
    """One ALE tracer step as the reference's driver runs it (core/model/driver.py:888-985, phases 7 and 8):
    ``adv.advect_fct`` of the stack (``adv`` a ``TracerAdvection``), then ``remap_columns`` of every member from
    h_src onto h_tgt, in one call, so the advected stack never leaves the device.  Results equal the two calls made
    one after the other, bit for bit.  Host arrays (NumPy, or pinned torch tensors: then the uploads of layer blocks,
    the FCT passes, the uploads of the thicknesses' row blocks, the remap and the downloads overlap) give the
    remapped stack on the host; CUDA tensors give a CUDA tensor."""
    from . import _pipeline as _pl
    from .remap import _remap_pipelined, _wet_pinned, remap_columns
    nt, n, ny, nx = tuple(C.shape)
    n1 = tuple(h_tgt.shape)[0]
    if (nt >= 2 and _pl.pinned(C, V0, V1, Qx, Qy, ok, h_src, h_tgt) and _wet_pinned(wet, ny, nx)
            and all(a.dtype == torch.float64 for a in (C, V0, V1, Qx, Qy, h_src, h_tgt))
            and ok.dtype in (torch.bool, torch.uint8) and tuple(ok.shape) in ((n, ny, nx), (ny, nx))
            and 8 * nt * n * ny * nx >= _pl.MIN_BYTES and ny >= 8 and not adv.record_open_flux):
        A = adv._advect_fct_layered(C, V0, V1, Qx, Qy, ok, download=False, blocks=_pl.FUSED_FCT_BLOCKS)
        return _remap_pipelined(h_src, None, h_tgt, wet, n, n1, ny, nx, nt, int(scheme), True, f_dev=A,
                                blocks=_pl.FUSED_REMAP_BLOCKS)
    host = not (isinstance(C, torch.Tensor) and C.is_cuda)
    if host:
        from ._device import Converter
        cv = Converter(C, V0, V1, Qx, Qy, ok, h_src, h_tgt, wet)
        A = adv.advect_fct(cv.f64(C), cv.f64(V0), cv.f64(V1), cv.f64(Qx), cv.f64(Qy), cv.u8(ok, tuple(ok.shape)))
        return cv.out(remap_columns(cv.f64(h_src), A, cv.f64(h_tgt), scheme, cv.u8(wet, (ny, nx))))
    return remap_columns(h_src, adv.advect_fct(C, V0, V1, Qx, Qy, ok), h_tgt, scheme, wet)
