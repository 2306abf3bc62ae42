"""Derivation of the polynomial coefficients of the engine's float32 atan2,
sine and cosine (MAP_ATAN_Q*, MAP_SIN_*, MAP_COS_* in common.cuh).

Each polynomial is fitted for minimum maximum RELATIVE error of the function it
serves by Lawson's algorithm (C. L. Lawson, "Contributions to the theory of
linear least maximum approximation", PhD thesis, UCLA 1961): a weighted least
squares fit repeated with each sample's weight multiplied by its current
absolute error, which converges to the minimax (Chebyshev) fit on the sample
set. The work is float64 on a dense Chebyshev-spaced grid; the coefficients are
then rounded to float32.

    atan(t) = t + t s Q(s),   s = t^2, t in [0, 1],   Q of degree 8
    sin(r)  = r + r s S(s),   s = r^2, r in [0, pi/4], S of degree 2
    cos(r)  = 1 + s C(s),     s = r^2, r in [0, pi/4], C of degree 3

Usage: python fit_poly.py   (prints the #define lines)
"""
import math

import numpy as np


def lawson(basis, target, weight, iters=400):
    """Coefficients c minimising max_i |weight_i (basis_i . c - target_i)| by
    Lawson's iteratively reweighted least squares."""
    lam = np.full(len(target), 1.0 / len(target))
    A = basis * weight[:, None]
    b = target * weight
    c = None
    for _ in range(iters):
        sw = np.sqrt(lam)
        c = np.linalg.lstsq(A * sw[:, None], b * sw, rcond=None)[0]
        e = np.abs(A @ c - b)
        lam = lam * e
        tot = lam.sum()
        if not tot > 0:
            break
        lam /= tot
    return c


def cheb_grid(a, b, n):
    k = np.arange(n)
    return (a + b) / 2 + (b - a) / 2 * np.cos(np.pi * (k + 0.5) / n)


def fit_atan(n=6000):
    t = cheb_grid(0.0, 1.0, n)
    t = t[t > 1e-3]
    s = t * t
    at = np.arctan(t)
    g = (at / t - 1.0) / s                  # the Q(s) that would make the identity exact
    basis = np.stack([s ** k for k in range(9)], axis=1)
    # relative error of atan: t s (Q(s) - g(s)) / atan(t)
    c = lawson(basis, g, t * s / at)
    return c[::-1]                          # Q0 (highest degree) ... Q8 (constant)


def fit_sin(n=4000):
    r = cheb_grid(0.0, math.pi / 4, n)
    r = r[r > 1e-3]
    s = r * r
    g = (np.sin(r) / r - 1.0) / s
    basis = np.stack([s ** k for k in range(3)], axis=1)
    c = lawson(basis, g, r * s / np.sin(r))
    return c                                # S_1 (constant) ... S_3


def fit_cos(n=4000):
    r = cheb_grid(0.0, math.pi / 4, n)
    r = r[r > 1e-3]
    s = r * r
    g = (np.cos(r) - 1.0) / s
    basis = np.stack([s ** k for k in range(4)], axis=1)
    c = lawson(basis, g, s / np.cos(r))
    return c                                # C_1 (constant) ... C_4


def f32_hex(v):
    """float32 value as a C hexadecimal float literal's digits, e.g. -0x1.d62fecp-10."""
    m, e = float(np.float32(v)).hex().split("p")
    m = m.rstrip("0")
    return (m + "0" if m.endswith(".") else m) + "p" + e


def defines():
    out = {}
    for i, v in enumerate(fit_atan()):
        out["MAP_ATAN_Q%d" % i] = np.float32(v)
    for i, v in enumerate(fit_sin()):
        out["MAP_SIN_%d" % (i + 1)] = np.float32(v)
    for i, v in enumerate(fit_cos()):
        out["MAP_COS_%d" % (i + 1)] = np.float32(v)
    return out


if __name__ == "__main__":
    for k, v in defines().items():
        print("#define %s %sf" % (k, f32_hex(v)))
