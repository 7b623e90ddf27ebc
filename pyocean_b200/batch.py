"""
Batched ALE tracer steps of many independent, unevenly sized domains on one GPU.

One step of every domain is ``advect_fct`` of its stack followed by the remap of every stack member onto its target
grid (the reference's phases 7 and 8, core/model/driver.py:888-985, run once per domain).  Instead of 10-11 kernel
launches per domain and step, each pass of the step is ONE launch over all domains: the CTAs of a launch are split
into per-domain ranges by a CTA-offset table and every CTA finds its domain by binary search, so small domains share
the GPU instead of each leaving most of the 148 SMs idle.  A step sequence only enqueues kernels and is captured in
a CUDA graph (``capture``); the tile shapes come from ``autotune``.

Results of each domain are bit for bit those of ``pocean_advect_fct_f64`` (or ``_mixed``) followed by
``pocean_remap_columns_f64`` on that domain alone, whatever the tile shape.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Iterable, Sequence

import numpy as np
import torch

from . import _lib


class _Domain(ctypes.Structure):
    """Mirror of ``pocean_domain`` (include/pocean_b200.h)."""
    _fields_ = [("C", ctypes.c_void_p), ("V0", ctypes.c_void_p), ("V1", ctypes.c_void_p), ("Qx", ctypes.c_void_p),
                ("Qy", ctypes.c_void_p), ("ok", ctypes.c_void_p), ("inflow", ctypes.c_void_p),
                ("nt", ctypes.c_int), ("nz", ctypes.c_int), ("ny", ctypes.c_int), ("nx", ctypes.c_int),
                ("flags", ctypes.c_uint), ("dt", ctypes.c_double), ("C_adv", ctypes.c_void_p),
                ("workspace", ctypes.c_void_p), ("workspace_bytes", ctypes.c_size_t), ("h_src", ctypes.c_void_p),
                ("h_tgt", ctypes.c_void_p), ("wet", ctypes.c_void_p), ("remap_scheme", ctypes.c_int),
                ("C_next", ctypes.c_void_p)]


@dataclass
class Domain:
    """Device-resident state of one domain: geometry and transports (read only) and its ping-pong stacks."""
    C: torch.Tensor            # (nt, nz, ny, nx) state at parity 0
    C_next: torch.Tensor       # state at parity 1
    C_adv: torch.Tensor        # advected stack (before the remap)
    V0: torch.Tensor
    V1: torch.Tensor
    Qx: torch.Tensor
    Qy: torch.Tensor
    ok: torch.Tensor           # uint8
    h_src: torch.Tensor
    h_tgt: torch.Tensor
    wet: torch.Tensor          # uint8
    workspace: torch.Tensor
    flags: int
    dt: float
    remap_scheme: int
    inflow: torch.Tensor | None = None

    @property
    def shape(self) -> tuple:
        return tuple(self.C.shape)

    @property
    def cells(self) -> int:
        return int(self.C.numel())

    @classmethod
    def from_workload(cls, w, device, flags: int | None = None) -> "Domain":
        """Copies a ``workloads.Workload`` to the device (flags from its periodic axes and scheme by default)."""
        g = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a if dt is None else a.astype(dt))).to(device)  # noqa: E731
        if flags is None:
            flags = (_lib.PERIODIC_X if "x" in w.periodic else 0) | (_lib.PERIODIC_Y if "y" in w.periodic else 0)
            flags |= 0 if w.scheme == "weno5" else _lib.WENO_JS
            for e, f in (("west", _lib.OPEN_W), ("east", _lib.OPEN_E), ("south", _lib.OPEN_S), ("north", _lib.OPEN_N)):
                flags |= f if e in w.open else 0
        return cls.from_tensors(g(w.C), g(w.V0), g(w.V1), g(w.Qx), g(w.Qy), g(w.ok, np.uint8), g(w.h_src),
                                g(w.h_tgt), g(w.wet, np.uint8), flags, w.dt, w.remap_scheme)

    @classmethod
    def from_tensors(cls, C, V0, V1, Qx, Qy, ok, h_src, h_tgt, wet, flags, dt, remap_scheme, inflow=None) -> "Domain":
        nt, n, ny, nx = C.shape
        nbytes = _lib.lib().pocean_advect_fct_workspace_bytes(nt, n, ny, nx)
        dev = C.device
        return cls(C=C.contiguous().clone(), C_next=torch.empty_like(C), C_adv=torch.empty_like(C),
                   V0=V0.contiguous(), V1=V1.contiguous(), Qx=Qx.contiguous(), Qy=Qy.contiguous(),
                   ok=ok.contiguous(), h_src=h_src.contiguous(), h_tgt=h_tgt.contiguous(), wet=wet.contiguous(),
                   workspace=torch.empty(nbytes, dtype=torch.uint8, device=dev), flags=int(flags), dt=float(dt),
                   remap_scheme=int(remap_scheme), inflow=None if inflow is None else inflow.contiguous())

    def as_struct(self, swapped: bool = False) -> _Domain:
        """The C descriptor; ``swapped``: the current state is in C_next (parity 0 of the plan reads C_next)."""
        nt, n, ny, nx = self.shape
        p = lambda t: None if t is None else t.data_ptr()                              # noqa: E731
        cur, nxt = (self.C_next, self.C) if swapped else (self.C, self.C_next)
        return _Domain(p(cur), p(self.V0), p(self.V1), p(self.Qx), p(self.Qy), p(self.ok), p(self.inflow),
                       nt, n, ny, nx, self.flags, self.dt, p(self.C_adv), p(self.workspace), self.workspace.numel(),
                       p(self.h_src), p(self.h_tgt), p(self.wet), self.remap_scheme, p(nxt))


class _Plan:
    """A ``pocean_batch`` plan and the device buffer holding its descriptors (``buf``: reuse a buffer of an earlier
    plan — the new descriptors are written in stream order, after the steps already enqueued)."""

    def __init__(self, structs, tile_rows: int, device, buf: torch.Tensor | None = None,
                 stream: int | None = None) -> None:
        L = _lib.lib()
        n = len(structs)
        need = L.pocean_batch_device_bytes(n)
        if buf is None or buf.numel() < need:
            buf = torch.empty(need, dtype=torch.uint8, device=device)
        self.buf = buf
        arr = (_Domain * n)(*structs)
        h = ctypes.c_void_p()
        st = torch.cuda.current_stream(device).cuda_stream if stream is None else stream
        _lib.check(L.pocean_batch_create(ctypes.cast(arr, ctypes.c_void_p), n, tile_rows, self.buf.data_ptr(),
                                         self.buf.numel(), ctypes.byref(h), st), "batch_create")
        self.handle = h
        self.tile_rows = tile_rows

    def step(self, parity: int, remap_nf: int, mixed: bool, stream: int) -> None:
        _lib.check(_lib.lib().pocean_batch_step(self.handle, parity, remap_nf, int(mixed), stream), "batch_step")

    def __del__(self) -> None:
        h = getattr(self, "handle", None)
        L = getattr(_lib, "_LIB", None)           # None once the interpreter is shutting down
        if h is not None and h.value and L is not None:
            L.pocean_batch_destroy(h)
            self.handle = None


class DomainBatch:
    """Many independent domains stepped together: every pass of a step is one launch over all of them."""

    TILE_ROWS = (4, 8, 16)
    REMAP_NF = (1, 2)

    def __init__(self, domains: Iterable[Domain], tile_rows: int = 8, remap_nf: int = 2, mixed: bool = False) -> None:
        self.domains = list(domains)
        if not self.domains:
            raise ValueError("a batch needs at least one domain")
        self.device = self.domains[0].C.device
        self.mixed = bool(mixed)
        self.remap_nf = int(remap_nf)
        self.parity = 0
        self._structs = [d.as_struct() for d in self.domains]
        self._plans: dict[int, _Plan] = {}
        self.plan = self._plan(tile_rows)

    @property
    def launches_per_step(self) -> int:
        """3 face and 2 cell passes, the limiter coefficients, the final update, then the remap: one pass over
        field pairs and one over the odd fields (or one over all fields) and the general-column fixup."""
        nts = [d.shape[0] for d in self.domains]
        if self.remap_nf == 2:
            return 7 + any(n >= 2 for n in nts) + any(n % 2 for n in nts) + 1
        return 7 + 2

    def _plan(self, tile_rows: int) -> _Plan:
        if tile_rows not in self._plans:
            self._plans[tile_rows] = _Plan(self._structs, tile_rows, self.device)
        return self._plans[tile_rows]

    @property
    def cells(self) -> int:
        """Tracer cells of one step of the whole batch."""
        return sum(d.cells for d in self.domains)

    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def state(self, i: int) -> torch.Tensor:
        """Current stack of domain i."""
        d = self.domains[i]
        return d.C if self.parity == 0 else d.C_next

    def step(self, steps: int = 1) -> None:
        for _ in range(steps):
            self.plan.step(self.parity, self.remap_nf, self.mixed, self.stream())
            self.parity ^= 1

    def capture(self, steps: int) -> torch.cuda.CUDAGraph:
        """A CUDA graph of ``steps`` steps from the current parity (even ``steps``: replays chain).  Capturing
        enqueues nothing; each replay advances the state by ``steps`` steps."""
        if steps < 2 or steps % 2:
            raise ValueError("capture an even number of steps so that replays start from the same parity")
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        p0 = self.parity
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.step(steps)
        torch.cuda.current_stream(self.device).wait_stream(s)
        self.parity = p0
        return g

    def autotune(self, steps: int = 2, tile_rows: Sequence[int] | None = None,
                 nfs: Sequence[int] | None = None) -> dict:
        """Times every (tile rows of the stage passes, remap fields per thread) on the batch itself and keeps the
        fastest.  The state is saved before and restored after, so tuning does not advance the domains."""
        rows = tuple(tile_rows or self.TILE_ROWS)
        nfs = tuple(nfs or self.REMAP_NF)
        saved = [self.state(i).clone() for i in range(len(self.domains))]
        p0 = self.parity
        times = {}
        for sl in rows:
            self.plan = self._plan(sl)
            for nf in nfs:
                self.remap_nf = nf
                self.step(2)                                        # warm-up
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                self.step(2 * steps)
                e1.record()
                e1.synchronize()
                times[(sl, nf)] = e0.elapsed_time(e1) / (2 * steps)
        best = min(times, key=times.get)
        self.plan = self._plan(best[0])
        self.remap_nf = best[1]
        self._plans = {best[0]: self.plan}
        self.parity = p0
        for i, s in enumerate(saved):
            self.state(i).copy_(s)
        return dict(tile_rows=best[0], remap_nf=best[1],
                    ms_per_step={f"{k[0]}/{k[1]}": v for k, v in times.items()})


def sequential_launches(domains: Sequence[Domain]) -> int:
    """Kernel launches of one ``sequential_step``: 7 FCT passes, then per domain the remap of field pairs (if any),
    of the odd field (if any) and the general-column fixup."""
    return sum(7 + (d.shape[0] >= 2) + (d.shape[0] % 2) + 1 for d in domains)


def sequential_step(domains: Sequence[Domain], parity: int, mixed: bool = False, stream: int | None = None) -> None:
    """One step of every domain with the single-domain entry points, one domain after another (7-8 plain launches
    per domain), on the same buffers as the batch: the form a batch replaces."""
    L = _lib.lib()
    fn = L.pocean_advect_fct_mixed if mixed else L.pocean_advect_fct_f64
    for d in domains:
        nt, n, ny, nx = d.shape
        src, dst = (d.C, d.C_next) if parity == 0 else (d.C_next, d.C)
        st = torch.cuda.current_stream(d.C.device).cuda_stream if stream is None else stream
        _lib.check(fn(src.data_ptr(), d.V0.data_ptr(), d.V1.data_ptr(), d.Qx.data_ptr(), d.Qy.data_ptr(),
                      d.ok.data_ptr(), None if d.inflow is None else d.inflow.data_ptr(), nt, n, ny, nx, d.flags,
                      d.dt, d.C_adv.data_ptr(), 0, None, None, d.workspace.data_ptr(), d.workspace.numel(), st),
                   "advect_fct")
        _lib.check(L.pocean_remap_columns_f64(d.h_src.data_ptr(), d.C_adv.data_ptr(), d.h_tgt.data_ptr(),
                                              d.wet.data_ptr(), n, n, ny, nx, nt, d.remap_scheme, dst.data_ptr(), st),
                   "remap_columns")
