"""
Device arithmetic checked on the CPU: tests/hostcore/hostcore.cpp compiles the library's header-only pieces for
the host (g++ -ffp-contract=off, the IEEE-754 operations the GPU executes) —

* the correctly rounded constant divisions (div3_exact / div6_exact) against IEEE division, on random bit
  patterns of every exponent, on ordinary magnitudes, and on the edge values of their guard;
* the plane-index division by the tracer count (plane_div) against integer division, for every plane index;
* the one-pass column remap (remap_column_stream) against the oracle's restatement of remap_column, bit for bit,
  on thousands of seeded columns with vanished source and target layers, both schemes' order reductions, totals
  that differ by round-off, n0 != n1, one or two fields per sweep, and thick source cells spanning many targets
  (the thickest piece after shorter ones, ties for it); the array formulation on the same columns.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as O

SRC = os.path.join(ROOT, "tests", "hostcore", "hostcore.cpp")


@pytest.fixture(scope="module")
def hostcore(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("hostcore") / "hostcore.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                    "-Wno-unknown-pragmas", "-o", so, SRC], check=True)
    L = ctypes.CDLL(so)
    D = ctypes.POINTER(ctypes.c_double)
    L.check_exactdiv.restype = ctypes.c_longlong
    L.check_exactdiv.argtypes = [ctypes.c_longlong, ctypes.c_ulonglong, D]
    L.check_exactdiv_list.restype = ctypes.c_longlong
    L.check_exactdiv_list.argtypes = [D, ctypes.c_longlong]
    L.check_plane_div.restype = ctypes.c_longlong
    L.check_plane_div.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_longlong]
    L.remap_stream_column.restype = ctypes.c_int
    L.remap_stream_column.argtypes = [D, D, ctypes.c_int, D, ctypes.c_int, ctypes.c_int, ctypes.c_int, D]
    L.remap_general_column.restype = ctypes.c_int
    L.remap_general_column.argtypes = [D, D, ctypes.c_int, D, ctypes.c_int, ctypes.c_int, D]
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def test_plane_division_equals_integer_division(hostcore):
    # every divisor up to 2048, then a spread up to the largest tracer count the entry points accept (65535)
    nts = list(range(1, 2049)) + list(range(2049, 65536, 97)) + [2 ** e + d for e in range(11, 16) for d in (-1, 0, 1)]
    nts = np.array(sorted(set(n for n in nts if 1 <= n <= 65535)), dtype=np.int32)
    assert hostcore.check_plane_div(nts.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), nts.size) == 0


def test_exact_constant_division_equals_ieee_division(hostcore):
    bad = np.zeros(2)
    assert hostcore.check_exactdiv(2_000_000, 12345, _p(bad)) == 0, bad
    edges = []
    for e in list(range(-1074, 1024, 7)) + [-1022, -1021, -900, -899, -898, -897, 897, 898, 899, 900, 1023]:
        for m in (1.0, 1.5, 1.0 + 2.0 ** -52, 2.0 - 2.0 ** -52, 1.3333333333333333, 1.6666666666666667):
            v = m * 2.0 ** e if -1074 <= e <= 1023 else 0.0
            if np.isfinite(v):
                edges += [v, -v, v * 3.0 if np.isfinite(v * 3.0) else v]
    edges += [0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, np.finfo(float).tiny, np.finfo(float).max, 3.0, 6.0,
              1.0, 9007199254740993.0, 1e-300, 1e300]
    xs = np.array(edges, dtype=np.float64)
    assert hostcore.check_exactdiv_list(_p(xs), xs.size) == 0


def _columns(seed, count):
    rng = np.random.default_rng(seed)
    for c in range(count):
        n0 = int(rng.integers(1, 61))
        n1 = int(rng.integers(1, 61)) if c % 3 else n0
        kind = c % 6
        h0 = rng.uniform(0.2, 20.0, n0)
        if kind in (1, 2, 5):
            h0 = np.where(rng.random(n0) < 0.5, rng.choice([0.0, 1e-10, 1e-3], n0), h0)
        if kind == 3:
            h0[: max(0, n0 - 4)] = 0.0                        # z*-like: vanished bottom layers
        u0 = rng.normal(15, 3, n0)
        if kind == 4:
            u0 = np.where(np.arange(n0) < n0 // 2, 10.0, 20.0) + rng.normal(0, 0.3, n0)
        h1 = rng.uniform(0.1, 2.0, n1)
        if kind in (2, 5):
            h1 = np.where(rng.random(n1) < 0.3, 0.0, h1)      # vanished targets
        tot0 = h0.sum()
        if h1.sum() > 0:
            h1 *= tot0 / h1.sum()
        if c % 7 == 0:
            h1[-1] += rng.choice([1e-9, -1e-9 * min(1.0, h1[-1]), 1e-13, 0.0])
        if c % 11 == 0 and n0 == n1:
            h1 = h0.copy()                                     # identity
        yield n0, n1, h0, u0, np.maximum(h1, 0.0)


@pytest.mark.parametrize("scheme", [O.PCM, O.PLM, O.PPM_H4])
def test_one_pass_remap_equals_reference_column_remap(hostcore, scheme):
    checked = 0
    for n0, n1, h0, u0, h1 in _columns(100 + scheme, 1500):
        u2 = np.stack([u0, u0 * 0.37 - 4.0])
        for nf in (1, 2):
            out = np.full((nf, n1), np.nan)
            rc = hostcore.remap_stream_column(_p(h0), _p(np.ascontiguousarray(u2[:nf])), n0, _p(h1), n1, nf,
                                              scheme, _p(out))
            if rc:
                assert h0.max() <= 0.0                         # only dry columns are outside the sweep here
                continue
            for m in range(nf):
                ref = O.remap_column(h0, u2[m], h1, scheme)
                np.testing.assert_array_equal(out[m], ref, err_msg=f"n0={n0} n1={n1} scheme={scheme} field={m}")
            checked += 1
    assert checked > 2500


def _wide_cells(seed, count):
    # few thick source cells over many targets of mixed thickness (vanished ones included): each cell spans many
    # pieces, its longest piece often follows shorter ones, and rounded thicknesses make ties for the longest
    rng = np.random.default_rng(seed)
    for c in range(count):
        n0 = int(rng.integers(1, 8))
        n1 = int(rng.integers(2, 61))
        h0 = rng.uniform(0.5, 20.0, n0)
        if c % 3 == 1:
            h0 = np.where(rng.random(n0) < 0.3, 0.0, h0)
        h1 = rng.choice([0.0, 0.05, 0.1, 0.3, 1.0, 2.5], n1) * rng.uniform(0.5, 1.5, n1)
        if c % 4 == 0:
            h1 = np.round(h1, 1)
        if h1.sum() > 0:
            h1 *= h0.sum() / h1.sum()
        yield n0, n1, h0, rng.normal(15, 3, n0), h1


@pytest.mark.parametrize("scheme", [O.PCM, O.PLM, O.PPM_H4])
def test_one_pass_remap_on_cells_spanning_many_targets(hostcore, scheme):
    checked = 0
    for n0, n1, h0, u0, h1 in _wide_cells(900 + scheme, 1500):
        u2 = np.stack([u0, u0 * 0.37 - 4.0])
        for nf in (1, 2):
            out = np.full((nf, n1), np.nan)
            rc = hostcore.remap_stream_column(_p(h0), _p(np.ascontiguousarray(u2[:nf])), n0, _p(h1), n1, nf,
                                              scheme, _p(out))
            if rc:
                assert h0.max() <= 0.0
                continue
            for m in range(nf):
                ref = O.remap_column(h0, u2[m], h1, scheme)
                np.testing.assert_array_equal(out[m], ref, err_msg=f"n0={n0} n1={n1} scheme={scheme} field={m}")
            out1 = np.full(n1, np.nan)
            assert hostcore.remap_general_column(_p(h0), _p(u0), n0, _p(h1), n1, scheme, _p(out1)) == 0
            np.testing.assert_array_equal(out1, O.remap_column(h0, u0, h1, scheme))
            checked += 1
    assert checked > 2000


@pytest.mark.parametrize("scheme", [O.PCM, O.PLM, O.PPM_H4])
def test_array_formulation_equals_reference_including_negative_targets(hostcore, scheme):
    # the device's path for columns outside the sweep: any target thicknesses, negative and NaN included
    rng = np.random.default_rng(7 + scheme)
    for n0, n1, h0, u0, h1 in _columns(300 + scheme, 600):
        h1 = h1.copy()
        if n1 > 2:
            h1[rng.integers(0, n1)] = -abs(rng.normal(0, 0.5))
        out = np.full(n1, np.nan)
        assert hostcore.remap_general_column(_p(h0), _p(u0), n0, _p(h1), n1, scheme, _p(out)) == 0
        np.testing.assert_array_equal(out, O.remap_column(h0, u0, h1, scheme))
