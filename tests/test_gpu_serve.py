"""The job server: every job's result is the same served in the mix as run alone, admission respects the HBM
budget, and jobs that arrive while others run join them (continuous batching)."""
from __future__ import annotations

import pytest
import torch

from pyocean_b200.batch import sequential_step
from pyocean_b200.serve import Job, Server, job_bytes, make_domain

pytestmark = pytest.mark.gpu


class TickClock:
    """A clock that advances one unit per reading: arrivals then depend on server iterations only."""

    def __init__(self) -> None:
        self.t = -1.0

    def __call__(self) -> float:
        self.t += 1.0
        return self.t


def _jobs():
    shapes = [(40, 24, 8, 2, 9), (70, 33, 5, 1, 6), (17, 9, 3, 4, 11), (64, 64, 12, 3, 5), (33, 65, 7, 1, 8),
              (96, 40, 10, 2, 7), (25, 31, 4, 3, 12), (50, 50, 6, 1, 4)]
    arrivals = [0, 0, 1, 2, 4, 4, 7, 9]
    return [Job(i, float(a), nx, ny, nz, nt, st, 500 + i) for i, (a, (nx, ny, nz, nt, st)) in
            enumerate(zip(arrivals, shapes))]


def _alone(job: Job, mixed: bool) -> torch.Tensor:
    d = make_domain(job, torch.device("cuda", 0))
    for s in range(job.steps):
        sequential_step([d], s & 1, mixed=mixed)
    return d.C_next if job.steps % 2 else d.C


@pytest.mark.parametrize("mixed", [True, False])
def test_each_result_same_alone_and_in_the_mix(mixed):
    jobs = _jobs()
    srv = Server(device="cuda:0", mixed=mixed, max_steps_per_iter=2, keep_results=True)
    rep = srv.run(jobs, clock=TickClock())
    assert rep["served"] == len(jobs) and rep["rejected"] == 0
    assert rep["peak_active"] >= 4 and rep["mean_active"] > 1.5          # jobs overlapped on the device
    for j in jobs:
        assert j.admitted >= j.arrival
        assert torch.equal(j.result, _alone(j, mixed)), f"job {j.id}"
        assert j.latency_s == j.latency_s                                # measured


def test_admission_respects_the_hbm_budget():
    jobs = _jobs()
    budget = 2 * max(job_bytes(j.nx, j.ny, j.nz, j.nt) for j in jobs)
    srv = Server(device="cuda:0", mixed=True, hbm_budget=budget, keep_results=True)
    rep = srv.run(jobs, clock=TickClock())
    assert rep["served"] == len(jobs) and rep["peak_hbm_bytes"] <= budget
    for j in jobs:
        assert torch.equal(j.result, _alone(j, True)), f"job {j.id}"


def test_oversized_job_is_refused_and_the_rest_served():
    jobs = _jobs()
    budget = sorted(job_bytes(j.nx, j.ny, j.nz, j.nt) for j in jobs)[-2]   # the largest job can never fit
    rep = Server(device="cuda:0", hbm_budget=budget).run(jobs, clock=TickClock())
    assert rep["rejected"] == 1 and rep["served"] == len(jobs) - 1


def test_one_at_a_time_server_matches():
    jobs = _jobs()[:4]
    rep = Server(device="cuda:0", mixed=False, batched=False, keep_results=True).run(jobs, clock=TickClock())
    assert rep["served"] == 4 and rep["peak_active"] == 1
    for j in jobs:
        assert torch.equal(j.result, _alone(j, False)), f"job {j.id}"
