"""Pinned host tensors take the overlapped-copy paths (row blocks for the remap; layer blocks for the FCT step, or
one tracer at a time when side outputs are asked for); their results equal the device-tensor and NumPy paths bit
for bit, side outputs included."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import pyocean_b200 as P
from pyocean_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _pin(a) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


def _dev(a) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def test_remap_of_pinned_host_tensors_equals_device_path():
    w = W.basin(seed=3, nx=256, ny=200, n=40)
    ref = P.remap_columns(_dev(w.h_src), _dev(w.C), _dev(w.h_tgt), 2, _dev(w.wet)).cpu()
    out = P.remap_columns(_pin(w.h_src), _pin(w.C), _pin(w.h_tgt), 2, _pin(w.wet))
    assert out.is_pinned() and torch.equal(out, ref)
    one = P.remap_columns(_pin(w.h_src), _pin(w.C[0]), _pin(w.h_tgt), 2, _pin(w.wet))   # a single field
    assert torch.equal(one, ref[0])
    np.testing.assert_array_equal(P.remap_columns(w.h_src, w.C, w.h_tgt, 2, w.wet), ref.numpy())


@pytest.mark.parametrize("mixed", [False, True])
def test_fct_step_of_pinned_host_tensors_equals_device_path(mixed):
    w = W.zstar_box(seed=5, nx=256, ny=192, n=30, nt=3)
    w.periodic, w.open = (), ("west", "east")
    kw = dict(scheme="weno5", time="ssprk3", dt=w.dt, ob=P.OpenEdges(w.open))

    def run(conv, ok):
        adv = P.TracerAdvection(**kw, precision="mixed" if mixed else "f64")
        adv.record_open_flux = True
        out, fx = adv.advect_fct(conv(w.C), conv(w.V0), conv(w.V1), conv(w.Qx), conv(w.Qy), ok, flux_face_i=-1)
        return out, fx, adv.last_open_flux

    ref = run(_dev, _dev(w.ok))
    got = run(_pin, _pin(w.ok))
    assert got[0].is_pinned()
    assert torch.equal(got[0], ref[0].cpu()) and torch.equal(got[1], ref[1].cpu())
    np.testing.assert_array_equal(got[2], ref[2])
    got2 = run(_pin, _pin(w.ok[0]))                      # ok given per column (ny, nx), broadcast over the layers
    assert torch.equal(got2[0], run(_dev, _dev(w.ok[0]))[0].cpu())
    adv = P.TracerAdvection(**kw)
    un = adv.advect_fct(_pin(w.C), _pin(w.V0), _pin(w.V1), _pin(w.Qx), _pin(w.Qy), _pin(w.ok), unlimited=True)
    assert torch.equal(un, adv.advect_fct(_dev(w.C), _dev(w.V0), _dev(w.V1), _dev(w.Qx), _dev(w.Qy), _dev(w.ok),
                                          unlimited=True).cpu())


@pytest.mark.parametrize("mixed,js", [(False, False), (True, False), (False, True)])
def test_fct_step_in_layer_blocks_equals_device_path(mixed, js):
    w = W.basin(seed=9, nx=256, ny=160, n=40, nt=2)
    kw = dict(scheme="weno5js" if js else "weno5", time="ssprk3", dt=w.dt, ob=P.OpenEdges(w.open),
              precision="mixed" if mixed else "f64")
    adv = P.TracerAdvection(**kw)
    adv.per = P.Periodic(w.periodic)
    ref = adv.advect_fct(_dev(w.C), _dev(w.V0), _dev(w.V1), _dev(w.Qx), _dev(w.Qy), _dev(w.ok)).cpu()
    for ok in (w.ok, w.ok[0]):                            # per cell-layer, and per column broadcast over the layers
        got = adv.advect_fct(_pin(w.C), _pin(w.V0), _pin(w.V1), _pin(w.Qx), _pin(w.Qy), _pin(ok))
        want = ref if ok is w.ok else adv.advect_fct(_dev(w.C), _dev(w.V0), _dev(w.V1), _dev(w.Qx), _dev(w.Qy),
                                                     _dev(ok)).cpu()
        assert got.is_pinned() and torch.equal(got, want)


def test_remap_of_pinned_host_tensors_onto_a_different_layer_count():
    w = W.basin(seed=4, nx=192, ny=256, n=30)
    rng = np.random.default_rng(2)
    h1 = rng.uniform(0.5, 2.0, (45,) + w.h_src.shape[1:])
    h1 *= w.h_src.sum(0) / h1.sum(0)
    ref = P.remap_columns(_dev(w.h_src), _dev(w.C), _dev(h1), 1, _dev(w.wet)).cpu()
    got = P.remap_columns(_pin(w.h_src), _pin(w.C), _pin(h1), 1, _pin(w.wet))
    assert got.shape == (2, 45) + w.h_src.shape[1:]
    np.testing.assert_array_equal(got.numpy(), ref.numpy())            # dry columns are NaN when N1 != N0


def test_fct_step_in_layer_blocks_on_a_periodic_box():
    w = W.zstar_box(seed=6, nx=256, ny=256, n=24, nt=3)                  # periodic x, walls in y (36 MB stack)
    from pyocean_b200 import _pipeline
    assert w.C.nbytes >= _pipeline.MIN_BYTES                           # large enough for the overlapped path
    adv = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=w.dt)
    adv.per = P.Periodic(w.periodic)
    ref = adv.advect_fct(_dev(w.C), _dev(w.V0), _dev(w.V1), _dev(w.Qx), _dev(w.Qy), _dev(w.ok)).cpu()
    got = adv.advect_fct(_pin(w.C), _pin(w.V0), _pin(w.V1), _pin(w.Qx), _pin(w.Qy), _pin(w.ok))
    assert torch.equal(got, ref)


@pytest.mark.parametrize("mixed", [False, True])
def test_fused_ale_step_equals_advect_then_remap(mixed):
    # ale_tracer_step: advect_fct then remap_columns in one call; pinned host tensors take the overlapped path
    # whose advected stack never leaves the device, NumPy and device tensors the one-shot paths
    w = W.basin(seed=8, nx=256, ny=200, n=40, nt=3)
    adv = P.TracerAdvection(scheme="weno5", time="ssprk3", dt=w.dt, precision="mixed" if mixed else "f64")
    args = (w.C, w.V0, w.V1, w.Qx, w.Qy, w.ok)
    ref = P.remap_columns(_dev(w.h_src), adv.advect_fct(*(_dev(a) for a in args)), _dev(w.h_tgt), 2,
                          _dev(w.wet)).cpu()
    got = P.ale_tracer_step(adv, *(_pin(a) for a in args), _pin(w.h_src), _pin(w.h_tgt), 2, _pin(w.wet))
    assert got.is_pinned() and torch.equal(got, ref)
    dev = P.ale_tracer_step(adv, *(_dev(a) for a in args), _dev(w.h_src), _dev(w.h_tgt), 2, _dev(w.wet))
    assert dev.is_cuda and torch.equal(dev.cpu(), ref)
    np.testing.assert_array_equal(P.ale_tracer_step(adv, *args, w.h_src, w.h_tgt, 2, w.wet), ref.numpy())
