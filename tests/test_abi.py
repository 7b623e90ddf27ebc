"""The C ABI (include/pocean_b200.h) without a GPU: the library loads, exports every declared symbol, sizes its
workspaces and rejects bad arguments before touching a device.

The argument-error tests hand the entry points made-up pointers (1, 8, 256 ...) that the argument checks must
refuse before any launch.  They run only in a process that sees no GPU: where one is visible (a plain `pytest` on a
GPU machine), `test_fake_pointer_checks_run_without_a_gpu` re-runs them in a child process with
CUDA_VISIBLE_DEVICES set empty, so a regression in the checks can never launch a kernel on a made-up address."""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import sys

import pytest

from conftest import ROOT
from pyocean_b200 import _lib

HEADER = os.path.join(ROOT, "include", "pocean_b200.h")


def _gpu_visible() -> bool:
    import torch
    return torch.cuda.is_available()


GPU_VISIBLE = _gpu_visible()
# tests that pass made-up device pointers: only where no GPU is visible
fake_pointers = pytest.mark.skipif(GPU_VISIBLE, reason="made-up pointers: run by "
                                   "test_fake_pointer_checks_run_without_a_gpu in a child process without a GPU")


@pytest.mark.skipif(not GPU_VISIBLE, reason="no GPU visible: the made-up-pointer tests run in this process")
def test_fake_pointer_checks_run_without_a_gpu():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", "-m", "not gpu",
                        os.path.abspath(__file__)], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and " failed" not in r.stdout, r.stdout[-2000:]


def declared_functions() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pocean_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert "pocean_advect_fct_f64" in names and "pocean_remap_columns_f64" in names
    for name in names:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature in pyocean_b200._lib"


def test_version_and_workspace_sizes():
    L = _lib.lib()
    assert L.pocean_version() >= 100
    nt, n, ny, nx = 2, 50, 512, 512
    cells = nt * n * ny * nx * 8
    fct = L.pocean_advect_fct_workspace_bytes(nt, n, ny, nx)
    # 3 cell stacks and 4 face stacks (u- and v-faces, twice)
    assert 7 * cells <= fct <= 7 * cells + 4 * nt * n * (ny + nx) * 8 + 7 * 256
    assert L.pocean_advect_fct_workspace_bytes(0, n, ny, nx) == 0
    assert L.pocean_advect_rk3_workspace_bytes(nt, n, ny, nx) >= 4 * cells


def _fct_call(**over):
    L = _lib.lib()
    args = dict(C=1, V0=1, V1=1, Qx=1, Qy=1, ok=1, inflow=None, nt=1, nz=2, ny=3, nx=4, flags=0, dt=1.0, out=1,
                face_i=0, fx=None, of=None, ws=256, wsb=1 << 20, stream=None)
    args.update(over)
    return L.pocean_advect_fct_f64(*args.values())


@fake_pointers
def test_argument_errors_are_reported_before_any_device_work():
    L = _lib.lib()
    assert _fct_call(nx=0) == 1
    assert b"sizes" in L.pocean_last_error()
    assert _fct_call(C=None) == 1
    assert _fct_call(flags=0x100) == 1                          # advect's face-scheme flags are not the FCT's
    rk3 = lambda flags: L.pocean_advect_rk3_f64(1, 1, 1, 1, 1, None, 1, None, 1, 2, 3, 4, flags, 1.0, 1, 0,  # noqa
                                                None, 256, 1 << 20, None)
    assert rk3(_lib.FACES_UP3 | _lib.FACES_UP1) == 1
    assert b"exclusive" in L.pocean_last_error()
    assert rk3(0x800) == 1
    assert _fct_call(fx=8, face_i=5) == 1                       # face_i > nx
    assert _fct_call(ws=None) == 2
    assert _fct_call(wsb=16) == 2
    assert _fct_call(ws=264) == 2                               # misaligned workspace
    assert _fct_call(nt=2, nz=40000) == 1                       # nt * nz planes > 65535 (one launch's grid)
    assert b"65535" in L.pocean_last_error()
    assert _fct_call(nz=512, ny=2047, nx=2047) == 1             # a field of 2^31 entries (32-bit offsets)
    assert b"2^31" in L.pocean_last_error()
    assert L.pocean_remap_columns_f64(1, 1, 1, 1, 300, 10, 2, 2, 1, 2, 1, None) == 1
    assert L.pocean_remap_columns_f64(1, 1, 1, 1, 10, 10, 2, 2, 1, 7, 1, None) == 1
    with pytest.raises(ValueError):
        _lib.check(1, "x")


def test_package_has_no_cpu_fallback(monkeypatch):
    # the product path refuses to run without the CUDA library instead of computing on the host
    monkeypatch.setattr(_lib, "_LIB", None)
    monkeypatch.setattr(_lib, "LIB_PATH", os.path.join(ROOT, "does-not-exist.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.lib()


def test_batch_domain_struct_layout_matches_ctypes(tmp_path):
    # the ctypes mirror of pocean_domain must agree with the C compiler's layout field by field
    import subprocess
    from pyocean_b200.batch import _Domain
    names = [f[0] for f in _Domain._fields_]
    src = tmp_path / "layout.c"
    body = "".join(f'    printf("%s %zu\\n", "{n}", offsetof(pocean_domain, {n}));\n' for n in names)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "pocean_b200.h"\nint main(void) {\n'
                   f'    printf("sizeof %zu\\n", sizeof(pocean_domain));\n{body}    return 0;\n}}\n')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = dict(line.split() for line in subprocess.check_output([str(exe)], text=True).splitlines())
    assert int(got["sizeof"]) == ctypes.sizeof(_Domain)
    for n in names:
        assert int(got[n]) == getattr(_Domain, n).offset, n


@fake_pointers
def test_batch_argument_errors():
    L = _lib.lib()
    assert L.pocean_batch_device_bytes(0) == 0
    assert L.pocean_batch_device_bytes(64) > L.pocean_batch_device_bytes(1) > 0
    h = ctypes.c_void_p()
    assert L.pocean_batch_create(8, 1, 8, 256, 1 << 20, None, None) == 1             # no output handle
    assert L.pocean_batch_create(None, 1, 8, 256, 1 << 20, ctypes.byref(h), None) == 1
    assert L.pocean_batch_create(8, 0, 8, 256, 1 << 20, ctypes.byref(h), None) == 1
    assert L.pocean_batch_create(8, 1, 5, 256, 1 << 20, ctypes.byref(h), None) == 1   # tile rows
    assert L.pocean_batch_create(8, 1, 8, 256, 16, ctypes.byref(h), None) == 2       # plan buffer too small
    assert L.pocean_batch_create(8, 1, 8, 264, 1 << 20, ctypes.byref(h), None) == 2   # misaligned
    assert h.value is None
    assert L.pocean_batch_step(None, 0, 2, 0, None) == 1


@fake_pointers
def test_layer_range_fct_argument_errors():
    L = _lib.lib()
    ws = 256 * 1024 * 1024
    call = lambda k0, k1, part, flags=0: L.pocean_advect_fct_layers(                           # noqa: E731
        0, 8, 8, 8, 8, 8, 8, None, 1, 4, 3, 3, flags, 1.0, 8, 256, ws, k0, k1, part, None)
    assert call(0, 5, 0) == 1 and call(2, 2, 0) == 1 and call(-1, 2, 1) == 1      # layer range
    assert call(0, 4, 2) == 1                                                     # part
    assert call(0, 4, 0, _lib.FCT_UNLIMITED) == 1                                 # unlimited refused


@fake_pointers
def test_neighbour_argument_errors():
    L = _lib.lib()
    # unknown rule, too many layers, null pointers, bad scheme
    assert L.pocean_regrid_remap_f64(2, 8, 8, 8, 8, 8, 1e-3, 8, 4, 3, 3, 1, 2, 8, 8, 8, None, None) == 1
    assert L.pocean_regrid_remap_f64(0, 8, 8, 8, 8, 8, 1e-3, 8, 300, 3, 3, 1, 2, 8, 8, 8, None, None) == 1
    assert L.pocean_regrid_remap_f64(0, 8, 8, 8, 8, None, 1e-3, 8, 4, 3, 3, 1, 2, 8, 8, 8, None, None) == 1
    assert L.pocean_regrid_remap_f64(0, 8, 8, 8, 8, 8, 1e-3, 8, 4, 3, 3, 1, 9, 8, 8, 8, None, None) == 1
    # hybrid: too many layers, null density, bad scheme
    hyb = lambda nz, rho, scheme: L.pocean_regrid_hybrid_remap_f64(                      # noqa: E731
        8, 8, 8, 8, rho, 8, 8, 8, 8, 0.0, 0.0, 1e-3, 1, 8, nz, 3, 3, 1, scheme, 8, 8, 8, None, None)
    assert hyb(300, 8, 2) == 1 and hyb(4, None, 2) == 1 and hyb(4, 8, 7) == 1
    assert L.pocean_face_fractions_f64(None, 4, 3, 3, 8, None) == 1
    assert L.pocean_remap_faces_f64(8, 8, None, None, 4, 3, 3, 1, 2, 8, None) == 1
    assert L.pocean_remap_faces_f64(8, 8, 8, None, 4, 3, 3, 0, 2, 8, None) == 1
    assert L.pocean_diffuse_ale_f64(8, 8, 8, 8, 8, 8, 8, 8, 8, 1, 2, 3, 4, 0x1, 1.0, 1.0, 8, None) == 1   # open flag
    assert L.pocean_diffuse_ale_f64(8, 8, 8, 8, 8, 8, 8, 8, None, 1, 2, 3, 4, 0, 1.0, 1.0, 8, None) == 1


@fake_pointers
def test_producer_argument_errors_and_workspaces():
    L = _lib.lib()
    assert L.pocean_upwind_transport_f64(8, 8, 8, 8, 8, 0, 3, 4, 8, None) == 1
    assert L.pocean_upwind_transport_f64(8, None, 8, 8, 8, 2, 3, 4, 8, None) == 1
    assert L.pocean_freshwater_volumes_f64(8, 8, None, 1e-6, 2, 3, 4, 8, None, None) == 1   # V_new aliases V
    assert L.pocean_freshwater_volumes_f64(8, None, None, 1e-6, 2, 3, 4, 16, None, None) == 1
    assert L.pocean_flux_divergence_f64(8, None, 2, 3, 4, 8, None) == 1
    assert L.pocean_layer_volumes_f64(8, 8, None, 2, 3, 4, 8, 8, None) == 1                 # ok without active
    assert L.pocean_ppm_transport_workspace_bytes(4, 8, 9, 20) >= 2 * 4 * 8 * 9 * 8 + 5 * 8 * 10 * 8
    assert L.pocean_limit_outflow_workspace_bytes(4, 8, 9) >= 3 * 4 * 8 * 9 * 8
    assert L.pocean_face_transport_thickness_f64(None, 8, 8, 2, 3, 4, 1, 8, 8, None) == 1
    assert L.pocean_ppm_transport_f64(8, 8, 8, 8, 8, 8, 8, 8, 2, 3, 4, 1.0, 20, 8, 256, 16, None) == 2
    assert L.pocean_ppm_transport_f64(8, 8, 8, 8, 8, 8, 8, 8, 2, 3, 4, 1.0, -1, 8, 256, 1 << 20, None) == 1
    # the PPM kernels index a field with 32-bit offsets: fields of 2^31 entries or more are refused
    assert L.pocean_ppm_edges_f64(8, 8, 512, 2047, 2047, 1e-10, 8, 8, None) == 1
    assert L.pocean_ppm_transport_f64(8, 8, 8, 8, 8, 8, 8, 8, 512, 2047, 2047, 1.0, 20, 8, 256, 1 << 20, None) == 1
    nl, wn = ctypes.c_int(0), ctypes.c_int(0)
    assert L.pocean_limit_outflow_f64(8, 8, 8, 8, 8, 2, 3, 4, 1.0, 1e-10, 50, 0x1, ctypes.byref(nl), ctypes.byref(wn),
                                      256, 1 << 20, None) == 1                     # open flag
    assert L.pocean_lagrangian_thickness_f64(8, 8, 8, 2, 3, 4, 1.0, 1e-9, 8, None, None) == 1


@fake_pointers
def test_noalloc_refuses_shapes_beyond_its_scratch():
    # the allocation-free FCT entry point refuses a shape whose scratch need exceeds its fixed array, before any
    # device call
    L = _lib.lib()
    nt, n, ny, nx = 2, 50, 512, 512
    assert L.pocean_advect_fct_workspace_bytes(nt, n, ny, nx) > (64 << 20)
    p = ctypes.c_void_p(256)
    rc = L.pocean_advect_fct_f64_noalloc(p, p, p, p, p, p, None, nt, n, ny, nx, 0, 1.0, p, 0, None, None, None)
    assert rc == 1
    assert b"scratch" in L.pocean_last_error()
    assert L.pocean_advect_fct_f64_noalloc(p, p, p, p, p, p, None, 0, n, ny, nx, 0, 1.0, p, 0, None, None, None) == 1
