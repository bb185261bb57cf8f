"""Known answers that need no reference run (numeric.cpp, header.h)."""
import ctypes
import math

import numpy as np

from tests.oracle_lib import lib


def p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_equilateral_unit_metric_quality_is_one():
    # numeric.cpp:303-305: q = 1 for an equilateral triangle whose edges have unit metric length
    L = lib()
    h = 0.1
    pa, pb, pc = np.array([0.0, 0.0]), np.array([h, 0.0]), np.array([h / 2, h * math.sqrt(3) / 2])
    t = np.array([1 / h ** 2, 0.0, 1 / h ** 2])
    q = L.orc_quality(p(pa), p(pb), p(pc), p(t), p(t), p(t))
    assert abs(q - 1.0) < 1e-12


def test_eigen_diagonal_shortcut():
    # numeric.cpp:30-38: |m12|^2 < 1e-9 returns the diagonal with swapped order
    L = lib()
    mat = np.array([4.0, 1e-6, 1e-6, 9.0])
    val, v1, v2 = np.zeros(2), np.zeros(2), np.zeros(2)
    L.orc_eigen(p(mat), p(val), p(v1), p(v2))
    assert list(val) == [9.0, 4.0] and list(v1) == [0.0, 1.0] and list(v2) == [1.0, 0.0]


def test_interpolating_identical_tensors_returns_the_tensor():
    L = lib()
    t = np.array([120.0, 35.0, 60.0])
    out = np.zeros(3)
    L.orc_interpolate(p(np.tile(t, 5)), p(out), 5)
    assert np.allclose(out, t, rtol=1e-13)


def test_metric_length_limits_are_the_reference_constants():
    # header.h:66-69
    assert abs(0.707106781186547 - 1 / math.sqrt(2)) < 1e-14
    assert abs(1.414213562373095 - math.sqrt(2)) < 1e-14
