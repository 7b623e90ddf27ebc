"""Batched steps of uneven domains: every domain's result equals the single-domain entry points, bit for bit, for
every tile shape, through a CUDA graph, in FP64 and mixed precision."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from pyocean_b200 import _lib
from pyocean_b200 import workloads as W
from pyocean_b200.batch import Domain, DomainBatch
from pyocean_b200.step import ALETracerStep

pytestmark = pytest.mark.gpu

STEPS = 3


def _workloads():
    a = W.zstar_box(seed=11, nx=40, ny=24, n=8, nt=2)
    b = W.zstar_box(seed=12, nx=70, ny=33, n=5)
    c = W.basin(seed=5, nx=48, ny=40, n=6, nt=3)                      # land, walls, dry columns
    d = W.zstar_box(seed=13, nx=33, ny=65, n=3)
    d.periodic, d.open = (), ("west", "east")                        # open edges, inflow from a given stack
    e = W.zstar_box(seed=14, nx=17, ny=9, n=2, nt=4)                 # smaller than one tile
    return [a, b, c, d, e]


def _domains(dev):
    ds = []
    for i, w in enumerate(_workloads()):
        dom = Domain.from_workload(w, dev)
        if w.open:
            rng = np.random.default_rng(40 + i)
            dom.inflow = torch.from_numpy(10.0 + 10.0 * rng.uniform(size=w.C.shape)).to(dev)
        ds.append(dom)
    return ds


def _alone(dom: Domain, steps: int, mixed: bool = False) -> torch.Tensor:
    """The same steps through pocean_advect_fct_f64 / _mixed and pocean_remap_columns_f64 on this domain alone."""
    nt, n, ny, nx = dom.shape
    st = ALETracerStep(nt, n, ny, nx, dom.dt, dom.flags, dom.remap_scheme, device=dom.C.device, mixed=mixed)
    c, nxt = dom.C.clone(), torch.empty_like(dom.C)
    for _ in range(steps):
        a = st.advect(c, dom.V0, dom.V1, dom.Qx, dom.Qy, dom.ok, inflow=dom.inflow)
        st.remap(dom.h_src, a, dom.h_tgt, dom.wet, nxt)
        c, nxt = nxt, c
    return c


@pytest.fixture(scope="module")
def dev():
    return torch.device("cuda", 0)


@pytest.fixture(scope="module")
def expected(dev):
    return [_alone(d, STEPS) for d in _domains(dev)]


@pytest.mark.parametrize("tile_rows,nf", [(4, 1), (8, 2), (16, 2), (16, 1)])
def test_batched_equals_each_domain_alone(dev, expected, tile_rows, nf):
    b = DomainBatch(_domains(dev), tile_rows=tile_rows, remap_nf=nf)
    b.step(STEPS)
    torch.cuda.synchronize()
    for i, ref in enumerate(expected):
        assert torch.equal(b.state(i), ref), f"domain {i} {b.domains[i].shape}"


def test_graph_replay_equals_eager_steps(dev):
    eager = DomainBatch(_domains(dev))
    eager.step(4)
    graphed = DomainBatch(_domains(dev))
    g = graphed.capture(2)
    g.replay()
    g.replay()
    graphed.parity = 0          # two replays of two steps: back at parity 0
    torch.cuda.synchronize()
    for i in range(len(eager.domains)):
        assert torch.equal(graphed.state(i), eager.state(i)), i
    del g


def test_mixed_batch_equals_mixed_alone(dev):
    b = DomainBatch(_domains(dev), mixed=True)
    b.step(2)
    torch.cuda.synchronize()
    for i, d in enumerate(_domains(dev)):
        assert torch.equal(b.state(i), _alone(d, 2, mixed=True)), i


def test_autotune_keeps_state_and_results(dev, expected):
    b = DomainBatch(_domains(dev))
    before = [b.state(i).clone() for i in range(len(b.domains))]
    cfg = b.autotune(steps=1, tile_rows=(4, 16), nfs=(1, 2))
    assert cfg["tile_rows"] in (4, 16) and cfg["remap_nf"] in (1, 2) and len(cfg["ms_per_step"]) == 4
    for i, s in enumerate(before):
        assert torch.equal(b.state(i), s)
    b.step(STEPS)
    torch.cuda.synchronize()
    for i, ref in enumerate(expected):
        assert torch.equal(b.state(i), ref), i


def test_weno_variants_cannot_mix(dev):
    ds = _domains(dev)[:2]
    ds[1].flags |= _lib.WENO_JS
    with pytest.raises(ValueError, match="same WENO variant"):
        DomainBatch(ds)


def test_js_batch_equals_js_alone(dev):
    ds = _domains(dev)
    for d in ds:
        d.flags |= _lib.WENO_JS
    b = DomainBatch(ds, tile_rows=4)
    b.step(2)
    torch.cuda.synchronize()
    for i, d in enumerate(_domains(dev)):
        d.flags |= _lib.WENO_JS
        assert torch.equal(b.state(i), _alone(d, 2)), i
