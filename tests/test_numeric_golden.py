"""The oracle's numerics reproduce trinity's numeric.cpp bit for bit on 64
seeded cases (eigendecomposition, log-Euclidean mean, quality, metric edge
length, Steiner point); vectors from oracle/ref_numeric.cpp."""
import ctypes
import json
import os

import numpy as np
import pytest

from tests.oracle_lib import lib

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [json.loads(l) for l in open(os.path.join(HERE, "golden", "numeric_vectors.jsonl"))]


def arr(v):
    return np.array([float.fromhex(x) for x in v], dtype=np.float64)


def p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


@pytest.mark.parametrize("k", range(len(CASES)))
def test_numeric_case(k):
    L = lib()
    c = CASES[k]
    ta, tb, tc = arr(c["ta"]), arr(c["tb"]), arr(c["tc"])
    pa, pb, pc = arr(c["pa"]), arr(c["pb"]), arr(c["pc"])
    mat = np.array([ta[0], ta[1], ta[1], ta[2]])
    val, v1, v2 = np.zeros(2), np.zeros(2), np.zeros(2)
    L.orc_eigen(p(mat), p(val), p(v1), p(v2))
    assert same(val, arr(c["eig_val"])) and same(v1, arr(c["eig_v1"])) and same(v2, arr(c["eig_v2"]))
    three = np.concatenate([ta, tb, tc])
    mean = np.zeros(3)
    L.orc_interpolate(p(three), p(mean), 3)
    assert same(mean, arr(c["mean"]))
    q = L.orc_quality(p(pa), p(pb), p(pc), p(ta), p(tb), p(tc))
    assert same([q], arr(c["quality"]))
    ln = L.orc_length(p(pa), p(pb), p(ta), p(tb))
    assert same([ln], arr(c["length"]))
    sp, st = np.zeros(2), np.zeros(3)
    L.orc_steiner(p(pa), p(pb), p(ta), p(tb), p(sp), p(st))
    assert same(sp, arr(c["steiner_p"])) and same(st, arr(c["steiner_t"]))


def test_cases_cover_the_diagonal_shortcut():
    assert any(arr(c["ta"])[1] == 0.0 for c in CASES)
