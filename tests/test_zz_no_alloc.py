"""
pocean_advect_fct_f64_noalloc: the FCT step for callers that cannot allocate device memory (a host model that
reaches the GPU only through the C ABI with no device allocator of its own, or one whose device memory belongs to a
pool that forbids side allocations).  It runs on a fixed scratch array inside the library instead of a caller
workspace.

Checked through the C ABI against pocean_advect_fct_f64 (caller workspace) on two different calls in a row, so a
second call cannot pass on what the first left in the shared scratch.  Both entry points run the same kernels on the
same inputs, so the results must be equal bit for bit.  The refusal of shapes beyond the fixed array is a CPU test
(tests/test_abi.py): it needs no device and hands the library no device pointers.  This file is collected last so
that a stop-at-first-failure run has run every other test before it.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from pyocean_b200 import _lib

pytestmark = pytest.mark.gpu


def _case(seed, nt, n, ny, nx, open_edges):
    rng = np.random.default_rng(seed)
    h = rng.uniform(1.0, 5.0, (n, ny, nx))
    active = rng.random((ny, nx)) > 0.1
    V0 = 1e6 * h * active
    Qx = rng.uniform(-0.4, 0.4, (n, ny, nx + 1)) * 1e3 * np.concatenate([h[..., :1], h], -1)
    Qy = rng.uniform(-0.4, 0.4, (n, ny + 1, nx)) * 1e3 * np.concatenate([h[:, :1], h], 1)
    ax = np.zeros((ny, nx + 1), bool)
    ax[:, 1:-1] = active[:, 1:] & active[:, :-1]
    ay = np.zeros((ny + 1, nx), bool)
    ay[1:-1] = active[1:] & active[:-1]
    if open_edges:
        ax[:, 0], ax[:, -1], ay[0], ay[-1] = active[:, 0], active[:, -1], active[0], active[-1]
    Qx *= ax
    Qy *= ay
    dt = 30.0
    V1 = V0 - dt * (Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:] - Qy[:, :-1])
    ok = (active[None] & (V1 > 0)).astype(np.uint8)
    T = 7.0 + rng.normal(0, 1, (n, ny, nx))
    C = np.stack([T, T ** 2, rng.uniform(0, 1, T.shape)][:nt])
    inflow = np.stack([np.full(T.shape, 9.0), np.full(T.shape, 81.0), np.full(T.shape, 0.5)][:nt])
    flags = (_lib.OPEN_W | _lib.OPEN_E | _lib.OPEN_S | _lib.OPEN_N) if open_edges else 0
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()                    # noqa: E731
    return dict(C=dev(C), V0=dev(V0), V1=dev(V1), Qx=dev(Qx), Qy=dev(Qy), ok=dev(ok),
                inflow=dev(inflow) if open_edges else None, shape=(nt, n, ny, nx), flags=flags, dt=dt)


def _outputs(k):
    nt, n, ny, nx = k["shape"]
    return (torch.full((nt, n, ny, nx), np.nan, dtype=torch.float64, device="cuda"),
            torch.full((nt, n, ny), np.nan, dtype=torch.float64, device="cuda"),
            torch.full((nt,), np.nan, dtype=torch.float64, device="cuda"))


def _common(k):
    nt, n, ny, nx = k["shape"]
    return (k["C"].data_ptr(), k["V0"].data_ptr(), k["V1"].data_ptr(), k["Qx"].data_ptr(), k["Qy"].data_ptr(),
            k["ok"].data_ptr(), None if k["inflow"] is None else k["inflow"].data_ptr(), nt, n, ny, nx, k["flags"],
            k["dt"])


def _run_noalloc(k, face_i):
    L = _lib.lib()
    out, fx, of = _outputs(k)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.pocean_advect_fct_f64_noalloc(*_common(k), out.data_ptr(), face_i, fx.data_ptr(),
                                         of.data_ptr() if k["inflow"] is not None else None, stream)
    assert rc == 0, L.pocean_last_error()
    return out, fx, of


def _run_workspace(k, face_i):
    L = _lib.lib()
    nt, n, ny, nx = k["shape"]
    out, fx, of = _outputs(k)
    nbytes = L.pocean_advect_fct_workspace_bytes(nt, n, ny, nx)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.pocean_advect_fct_f64(*_common(k), out.data_ptr(), face_i, fx.data_ptr(),
                                 of.data_ptr() if k["inflow"] is not None else None, ws.data_ptr(), nbytes, stream)
    assert rc == 0, L.pocean_last_error()
    return out, fx, of


def _equal(got, ref):
    assert got.shape == ref.shape
    assert torch.equal(got, ref), f"max |diff| = {float((got - ref).abs().max())}"


def test_noalloc_matches_workspace_entry_point_on_two_calls_in_a_row():
    first = _case(21, 2, 5, 37, 70, open_edges=True)
    second = _case(22, 3, 4, 29, 45, open_edges=False)
    a = _run_noalloc(first, 11)
    b = _run_noalloc(second, 7)          # reuses the scratch the first call left behind
    torch.cuda.synchronize()
    ref_a = _run_workspace(first, 11)
    for got, ref in zip(a, ref_a):       # C_out, the TEF face column and the open-edge budget
        _equal(got, ref)
    ref_b = _run_workspace(second, 7)
    _equal(b[0], ref_b[0])               # the closed case asks for no open-edge budget
    _equal(b[1], ref_b[1])
    assert torch.isfinite(b[0]).all() and torch.isfinite(a[2]).all()
