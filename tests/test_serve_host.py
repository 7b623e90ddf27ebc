"""Host side of the job server: the job stream, the HBM estimate and the on-device z* generator (run on the CPU)."""
from __future__ import annotations

import numpy as np
import torch

from pyocean_b200 import _lib
from pyocean_b200 import workloads as W
from pyocean_b200.serve import job_bytes, job_stream


def test_job_stream_is_seeded_and_within_bounds():
    a, b = job_stream(2000, seed=3, rate=50.0), job_stream(2000, seed=3, rate=50.0)
    assert [(j.arrival, j.nx, j.ny, j.nz, j.nt, j.steps) for j in a] == \
        [(j.arrival, j.nx, j.ny, j.nz, j.nt, j.steps) for j in b]
    arr = np.array([j.arrival for j in a])
    assert np.all(np.diff(arr) > 0)
    assert abs(len(a) / arr[-1] - 50.0) < 5.0                      # Poisson rate
    nx = np.array([j.nx for j in a])
    nz = np.array([j.nz for j in a])
    assert nx.min() >= 32 and nx.max() <= 512 and nz.min() >= 10 and nz.max() <= 75
    assert abs(np.median(nx) - np.sqrt(32 * 512)) < 15                # lognormal, median at the geometric mean
    st = np.array([j.steps for j in a])
    assert st.min() >= 10 and st.max() <= 200
    assert {j.nt for j in a} == {1, 2, 3, 4}
    assert len({j.seed for j in a}) == len(a)


def test_job_bytes_cover_state_and_workspace():
    nx, ny, nz, nt = 100, 80, 20, 3
    ws = _lib.lib().pocean_advect_fct_workspace_bytes(nt, nz, ny, nx)
    assert job_bytes(nx, ny, nz, nt) > ws + 3 * 8 * nt * nz * ny * nx


def test_device_generator_builds_a_consistent_zstar_box():
    f = W.zstar_box_device(7, 48, 40, 6, 2, "cpu")
    n, ny, nx = 6, 40, 48
    assert f["C"].shape == (2, n, ny, nx) and f["Qx"].shape == (n, ny, nx + 1) and f["Qy"].shape == (n, ny + 1, nx)
    assert torch.equal(f["Qx"][:, :, 0], f["Qx"][:, :, -1])                    # periodic in x
    assert float(f["Qy"][:, 0].abs().max()) == 0.0 and float(f["Qy"][:, -1].abs().max()) == 0.0  # walls
    umax = max(float(f["Qx"].abs().max()), float(f["Qy"].abs().max())) / (1000.0 * 5.0)
    assert abs(umax - 0.5) < 1e-12
    div = f["Qx"][..., 1:] - f["Qx"][..., :-1] + f["Qy"][:, 1:] - f["Qy"][:, :-1]
    assert float(div.abs().max()) < 1e-9 * float(f["Qx"].abs().max())      # non-divergent
    assert bool(f["ok"].all())
    assert torch.allclose(f["h_src"].sum(0), f["h_tgt"].sum(0), rtol=1e-14, atol=0)
    lo, hi = float(f["C"][..., : nx // 2].mean()), float(f["C"][..., nx // 2:].mean())
    assert abs(lo - 10.0) < 0.01 and abs(hi - 20.0) < 0.01
    g = W.zstar_box_device(7, 48, 40, 6, 2, "cpu")
    assert all(torch.equal(f[k], g[k]) for k in ("C", "Qx", "Qy", "h_src"))   # seeded


def test_oldest_first_policy_keeps_the_oldest_job_and_fills_beside_it():
    from pyocean_b200.serve import Job, Server
    srv = Server(device="cpu", hbm_budget=1 << 30, fill_cells=1_000_000, share=0.25, policy="oldest_first")
    big = Job(0, 0.0, 512, 512, 50, 2, 100, 1)                       # 26 M cells a step, arrived first
    mid = Job(1, 0.1, 256, 256, 50, 2, 50, 2)                        # 6.6 M cells: does not fit beside it
    small = [Job(2 + i, 0.2 + i, 64, 64, 20, 1, 20 + i, 3 + i) for i in range(4)]   # 82 k cells each
    chosen = srv._select([mid, big] + small)
    assert chosen[0] is big and mid not in chosen and all(s in chosen for s in small)
    # the combined step stays within (1 + share) of the oldest job's own step
    cells = lambda j: j.nt * j.nz * j.ny * j.nx                                            # noqa: E731
    assert sum(cells(j) for j in chosen) <= 1.25 * cells(big)
    # a small oldest job: the others fill up to fill_cells, smallest remaining work first
    late = Job(9, 5.0, 256, 256, 50, 2, 50, 9)
    chosen = srv._select(small + [late])
    assert chosen[0] is small[0] and late not in chosen and len(chosen) == 4
    assert Server(device="cpu", hbm_budget=1 << 30, policy="all")._select([big, mid] + small) == [big, mid] + small
    assert Server(device="cpu", hbm_budget=1 << 30, batched=False)._select([mid, big]) == [big]


def test_adaptive_policy_batches_everything_only_behind_a_long_backlog():
    from pyocean_b200.serve import Job, Server
    big = Job(0, 0.0, 512, 512, 50, 2, 100, 1)                       # 26 M cells x 100 steps = 2.6e9 cell-steps
    mid = Job(1, 0.1, 256, 256, 50, 2, 50, 2)
    small = [Job(2 + i, 0.2 + i, 64, 64, 20, 1, 20 + i, 3 + i) for i in range(4)]
    srv = Server(device="cpu", hbm_budget=1 << 30, fill_cells=1_000_000, backlog_cells=2e9)
    assert srv.policy == "adaptive"
    assert srv._select([mid, big] + small) == [mid, big] + small     # backlog 2.9e9 > 2e9: every job
    big.done_steps = 95                                              # backlog now ~0.5e9: oldest first again
    chosen = srv._select([mid, big] + small)
    assert chosen[0] is big and mid not in chosen and all(s in chosen for s in small)
