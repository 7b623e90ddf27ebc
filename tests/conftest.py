"""Shared test setup: the repository root on sys.path, the ``gpu`` marker, golden-vector loading."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libpocean_b200.so")


def load_golden(name: str) -> dict[str, dict[str, np.ndarray]]:
    """Cases of tests/golden/<name>.npz as {case: {key: array}} (scalars as 0-d arrays)."""
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        out: dict[str, dict[str, np.ndarray]] = {}
        for key in z.files:
            case, field = key.split("/", 1)
            out.setdefault(case, {})[field] = z[key]
    return out


@pytest.fixture(scope="session")
def golden():
    return load_golden


def case_open(rec) -> tuple:
    return tuple(str(s) for s in rec["open"]) if "open" in rec else ()


def case_periodic(rec) -> tuple:
    return tuple(str(s) for s in rec["periodic"]) if "periodic" in rec else ()


def regrid_columns_args(rec) -> tuple:
    """The arguments of ``regrid_columns(rule, H, eta, h, rho, params, wet, n_out)`` of a golden case."""
    rule = str(rec["rule"])
    if rule == "hybrid":
        params = dict(dz_top=rec["dz_top"], rho_target=rec["rho_target"], max_h_top=rec["max_h_top"],
                      h_min=float(rec["h_min"]), keep_isopycnal=bool(rec["keep"]))
        if float(rec["d_hybrid"]) > 0:
            params.update(dsigma=rec["dsigma"], d_sigma=float(rec["d_sigma"]), d_hybrid=float(rec["d_hybrid"]))
        return rule, rec["H"], rec["eta"], rec["h"], rec["rho"], params, rec["wet"], int(rec["n_out"])
    params = {k: rec[k] for k in ("dz_top", "dsigma") if k in rec}
    return rule, rec["H"], rec["eta"], rec["h"], None, params, rec["wet"], None
