"""The polynomial coefficients of the engine's float32 atan2, sine and cosine
(common.cuh) re-derived on the CPU by the committed Lawson fit
(map_b200/csrc/skeleton/fit_poly.py): the fit lands within a few float32 ulps
of every shipped coefficient, and the shipped polynomials reach the same
minimax relative error as the fresh fit (within the perturbation that
rounding the coefficients to float32 causes)."""
import math
import os
import re
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "map_b200", "csrc", "skeleton"))
import fit_poly  # noqa: E402

HDR = os.path.join(ROOT, "map_b200", "csrc", "skeleton", "common.cuh")


def shipped():
    src = open(HDR).read()
    return {n: np.float32(float.fromhex(v))
            for n, v in re.findall(r"#define (MAP_(?:ATAN_Q|SIN_|COS_)\d) (-?0x[0-9a-fp.+-]+)f\b", src)}


@pytest.fixture(scope="module")
def fits():
    return fit_poly.defines()


def ulps(a, b):
    a, b = np.float32(a), np.float32(b)
    return abs(int(a.view(np.int32)) - int(b.view(np.int32)))


def test_every_coefficient_is_re_derived(fits):
    S = shipped()
    assert set(S) == set(fits) and len(S) == 16
    # the low-degree terms fix the accuracy and come out identical or nearly;
    # the highest-degree atan terms are flat directions of the fit (a few ulps
    # there move the error by far less than an ulp of the result)
    tol = {"MAP_ATAN_Q0": 16, "MAP_ATAN_Q1": 8, "MAP_ATAN_Q2": 8, "MAP_ATAN_Q3": 4, "MAP_ATAN_Q4": 2,
           "MAP_COS_4": 4}
    for k in S:
        assert ulps(S[k], fits[k]) <= tol.get(k, 0), (k, S[k], fits[k])


def rel_err_atan(Q):
    t = np.linspace(1e-4, 1.0, 200001)
    s = t * t
    q = np.zeros_like(t)
    for c in Q:
        q = q * s + float(c)
    return np.max(np.abs((t + t * s * q) / np.arctan(t) - 1.0))


def rel_err_sincos(Sc, Cc):
    r = np.linspace(1e-4, math.pi / 4, 200001)
    s = r * r
    p = sum(float(c) * s ** i for i, c in enumerate(Sc))
    c = sum(float(v) * s ** i for i, v in enumerate(Cc))
    return (np.max(np.abs((r + r * s * p) / np.sin(r) - 1.0)),
            np.max(np.abs((1.0 + s * c) / np.cos(r) - 1.0)))


def test_shipped_polynomials_reach_the_minimax_error(fits):
    S = shipped()
    qa = [S["MAP_ATAN_Q%d" % i] for i in range(9)]
    qf = [fits["MAP_ATAN_Q%d" % i] for i in range(9)]
    ea, ef = rel_err_atan(qa), rel_err_atan(qf)
    # float32 rounding of the coefficients moves the error by up to a fifth of it;
    # both stay below a quarter of a float32 ulp (2^-26 relative)
    assert ea < 1.25 * ef and ea < 2 ** -26
    s_ship, c_ship = rel_err_sincos([S["MAP_SIN_%d" % i] for i in (1, 2, 3)],
                                    [S["MAP_COS_%d" % i] for i in (1, 2, 3, 4)])
    s_fit, c_fit = rel_err_sincos([fits["MAP_SIN_%d" % i] for i in (1, 2, 3)],
                                  [fits["MAP_COS_%d" % i] for i in (1, 2, 3, 4)])
    assert s_ship < 1.1 * s_fit and c_ship < 1.1 * c_fit
    assert s_ship < 2 ** -26 and c_ship < 2 ** -26
