"""Helpers shared by the parity tests (golden fixtures and bit comparisons)."""
import numpy as np


def bits(a):
    a = np.ascontiguousarray(np.asarray(a, np.float32))
    return a.view(np.uint32)


def assert_bits_equal(got, want, what=""):
    g, w = bits(got), bits(want)
    bad = np.flatnonzero(g.reshape(-1) != w.reshape(-1))
    assert bad.size == 0, f"{what}: {bad.size} of {g.size} values differ in bits (first at flat index {bad[:5]})"


def max_abs(got, want):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    both_nan = np.isnan(got) & np.isnan(want)
    assert np.array_equal(np.isnan(got), np.isnan(want)), "NaN placement differs"
    diff = np.abs(got - want)
    diff[both_nan] = 0
    return float(diff.max()) if diff.size else 0.0
