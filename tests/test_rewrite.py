"""The hillshade rewrite on CPU: which compositions the code generator
recognises, what it emits, and a float32 replay of the rewritten formula
against the oracle under the hillshade tolerance (the error table of the
rewrite, stated without a GPU)."""
import math

import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W
from oracle import oracle as O

f32 = np.float32


@pytest.fixture()
def R(M):
    yield M
    M.set_algebraic_rewrite(True)


def dem(M, h=64, w=96):
    return M.from_numpy(np.zeros((h, w), np.float32), bs=[32, 32])


def test_hill_script_is_rewritten(R):
    M = R
    hs = W.hillshade(dem(M))
    src = M.generated_source(hs)
    # hill.py's derivatives (Sobel / 8) take the fast form
    assert "map_shade_fast(" in src and "shade_slow0" in src
    # the group body computes no transcendental function outside the fallback
    body = src[src.index("focal_cell("):]
    assert "map_atan2f" not in body and "atanf" not in body and "map_sincosf" not in body
    assert M.compile_only(hs) == 1
    M.set_algebraic_rewrite(2)
    src = M.generated_source(W.hillshade(dem(M)))
    assert "map_shade<true>" in src and "map_shade_fast" not in src
    M.set_algebraic_rewrite(False)
    hs = W.hillshade(dem(M))
    src = M.generated_source(hs)
    assert "map_shade" not in src and "map_atan2f" in src


def test_operand_orders_and_zfactor(R):
    M = R
    d = dem(M)
    x, y = W.hori(d), W.vert(d)
    s = M.atan(2.5 * M.sqrt(y * y + x * x))
    z1 = M.atan2(y, -x) * (x != 0)
    z1 = (PI2 * (z1 < 0)) + z1
    z0 = ((PIH * (y > 0)) + (y < 0) * PI32) * (x == 0)
    asp = z0 + z1
    hs = M.sin(s) * (M.cos(asp - 2.1) * 0.6) + M.cos(s) * 0.8
    src = M.generated_source(hs)
    assert "map_shade_fast(" in src
    assert M.compile_only(hs) == 1
    M.set_algebraic_rewrite(2)
    assert "map_shade<false>" in M.generated_source(hs)


PI2, PIH, PI32 = 3.141593 * 2, 3.141593 / 2, 3.141593 * 2 - 3.141593 / 2


def test_not_rewritten_when_the_composition_differs(R):
    M = R
    d = dem(M)
    x, y = W.hori(d), W.vert(d)
    s = M.atan(M.sqrt(x * x + y * y))
    # wrap by 6.0 instead of about 2 pi: not the aspect of the identity
    z1 = (x != 0) * M.atan2(y, -x)
    z1 = z1 + (z1 < 0) * 6.0
    z0 = (x == 0) * ((y > 0) * PIH + (y < 0) * PI32)
    hs = 0.7 * M.cos(s) + 0.7 * M.sin(s) * M.cos(2.3 - (z1 + z0))
    assert "map_shade" not in M.generated_source(hs)
    # atan2(y, x) instead of atan2(y, -x)
    z1 = (x != 0) * M.atan2(y, x)
    z1 = z1 + (z1 < 0) * PI2
    hs = 0.7 * M.cos(s) + 0.7 * M.sin(s) * M.cos(2.3 - (z1 + z0))
    assert "map_shade" not in M.generated_source(hs)


def test_shared_slope_stays_computed(R):
    """A pattern node needed by another output (the slope) is still emitted."""
    M = R
    d = dem(M)
    hs = W.hillshade(d)
    sl = W.slope(d)
    src = M.generated_source(hs, sl)
    assert "map_shade" in src
    body = src[src.index("focal_cell("):]
    assert "atanf" in body           # the slope output itself
    assert M.compile_only(hs, sl) >= 1


def test_two_azimuths_share_one_group(R):
    M = R
    d = dem(M)
    a, b = W.hillshade(d, 45, 315), W.hillshade(d, 30, 200)
    src = M.generated_source(a, b)
    assert src.count("= map_shade_fast(") >= 2 and "shade_slow1" in src
    body = src[src.index("focal_cell("):]
    assert "map_sincosf" not in body
    assert M.compile_only(a, b) >= 1


# ---- float32 replay of map_shade (skeleton/common.cuh) against the oracle

def shade_constants(zenith=45.0, azimuth=315.0):
    PI = 3.141593
    zr = (90 - zenith) / 180 * PI
    ar = 360 - azimuth + 90
    ar = ar - 360 if ar > 360 else ar
    ar = float(f32(ar / 180 * PI))
    pi2, pih, pi32 = float(f32(PI * 2)), float(f32(PI / 2)), float(f32(PI * 2 - PI / 2))
    d = pi2 - 2 * math.pi
    return dict(cz=f32(math.cos(zr)), sz=f32(math.sin(zr)), S0=f32(math.sin(ar)), C0=f32(math.cos(ar)),
                S1=f32(math.sin(ar - d)), C1=f32(math.cos(ar - d)), SH=f32(math.cos(ar - pih)),
                S3=f32(-math.cos(ar - pi32)))


def fma32(a, b, c):
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(f32)


def replay_shade(x, y, k):
    """map_shade with K1 = true, each operation rounded once to float32 (the
    products of two floats are exact in float64, so fma is exact there before
    its one rounding); the reciprocal square root correctly rounded, which the
    Newton-refined estimate reaches within about one ulp."""
    q = fma32(x, x, (y * y).astype(f32))
    nz = x != 0
    neg = (y < 0) | (np.signbit(y) & (x > 0))
    S = np.where(nz, np.where(neg, k["S1"], k["S0"]), np.where(y > 0, k["SH"], k["S3"])).astype(f32)
    C = np.where(nz, np.where(neg, k["C1"], k["C0"]), f32(0)).astype(f32)
    num = fma32(y, S, (x * -C).astype(f32))
    v = (f32(1) + q).astype(f32)
    r = (1.0 / np.sqrt(v.astype(np.float64))).astype(f32)
    return (fma32(k["sz"], num, k["cz"]) * r).astype(f32)


@pytest.mark.parametrize("n,seed,scale,border", [(512, 7, 1.0, 0), (512, 3, 10.0, 1), (384, 9, 0.01, 2),
                                                   (640, 5, 1.0, 0)])
def test_rewrite_replay_within_tolerance(n, seed, scale, border):
    d = (synth.fbm_dem(n, n + 64, seed=seed) * f32(scale)).astype(f32)
    bs = (128, 128)
    H = np.array([[-1, 0, 1], [-2, 0, 2], [-1, 0, 1]], f32)
    V = np.array([[-1, -2, -1], [0, 0, 0], [1, 2, 1]], f32)
    x = (O.conv_f32(d, H, bs, border) * f32(0.125)).astype(f32)
    y = (O.conv_f32(d, V, bs, border) * f32(0.125)).astype(f32)
    hs = replay_shade(x, y, shade_constants())
    ref32 = O.hillshade_f32(d, bs, border)
    ref64 = O.hillshade_f64(d, bs, border)
    bound = O.hillshade_bound(d, bs, border)
    ok, diff, only = O.hill_tolerance(hs, ref32, bound)
    assert ok.all()
    # margin: at most half of the cancellation bound is used
    assert np.max(diff / (4 * bound)) < 0.5
    assert only.mean() < 0.01
    # no further from FP64 than the FP32 chain (both carry the same float Sobel sums)
    assert np.abs(hs - ref64).max() <= np.abs(ref32 - ref64).max() + 4 * float(np.spacing(f32(1)))


def test_fast_form_equals_general_form_replay():
    """map_shade_fast on the unscaled Sobel sums (zero weights dropped, products
    by +-1 / +-2 as fused multiply-adds, 1/8 and the light direction folded into
    the constants) replayed in float32 equals map_shade on the derivatives /8,
    bit for bit, on every cell."""
    k = shade_constants()
    d = synth.fbm_dem(300, 400, seed=12)
    d[::37, ::41] = 0.0                     # flat spots: x == 0 / y == 0 cells
    H = np.array([[-1, 0, 1], [-2, 0, 2], [-1, 0, 1]], f32)
    V = np.array([[-1, -2, -1], [0, 0, 0], [1, 2, 1]], f32)
    xl = O.conv_f32(d, H, (128, 128), 0)
    yl = O.conv_f32(d, V, (128, 128), 0)
    # the fast sums as emitted: fma(tap, w, acc) over the non-zero weights, the
    # first (weight -1, exact) the addend of the fma before it (the centre tap
    # times 0, x sum) or after it (y sum)
    p = np.pad(d, 1, mode="symmetric")      # interior cells only are compared below
    def tap(i1, i0):
        return p[i1:i1 + d.shape[0], i0:i0 + d.shape[1]]
    def fast_sum(m, lead_with_centre):
        nz = [(i1, i0) for i1 in range(3) for i0 in range(3) if m[i1, i0] != 0]
        assert m[nz[0]] == -1
        if lead_with_centre:
            acc, rest = fma32(tap(1, 1), f32(0), -tap(*nz[0])), nz[1:]
        else:
            acc, rest = fma32(tap(*nz[1]), m[nz[1]], -tap(*nz[0])), nz[2:]
        for i1, i0 in rest:
            acc = fma32(tap(i1, i0), m[i1, i0], acc)
        return acc
    xc, yc = fast_sum(H, True), fast_sum(V, False)
    inner = (slice(1, -1), slice(1, -1))
    # equal values (a zero sum may carry the other sign)
    assert np.array_equal(xc[inner], xl[inner]) and np.array_equal(yc[inner], yl[inner])
    general = replay_shade((xl * f32(0.125)).astype(f32), (yl * f32(0.125)).astype(f32), k)
    # fast: q = fma(xc, xc, yc*yc) + 0; choice by arithmetic; constants scaled
    q = fma32(xc, xc, (yc * yc).astype(f32))
    negf = (yc < 0).astype(f32)
    dS, dnC, dSx = f32(k["S1"] - k["S0"]), f32(-k["C1"] + k["C0"]), f32(k["S3"] - k["SH"])
    Sn = fma32(negf, dS, k["S0"])
    nC = fma32(negf, dnC, -k["C0"])
    Sx = fma32(negf, dSx, k["SH"])
    S = np.where(xc != 0, Sn, Sx).astype(f32)
    num = fma32(yc, S, (xc * nC).astype(f32))
    v = fma32(f32(2.0 ** -6), q, f32(1))
    r = (1.0 / np.sqrt(v.astype(np.float64))).astype(f32)
    fast = (fma32(f32(k["sz"] / 8), num, k["cz"]) * r).astype(f32)
    assert np.array_equal(fast[inner].view(np.uint32), general[inner].view(np.uint32))


def test_fast_form_kernel_shape(R):
    """The fast hillshade kernel: 64 x 64 tiles of 256 threads with registers
    capped for 6 CTAs per SM, interior tiles stored by one TMA tile store
    (whole-raster outputs; the per-cell stores stay for the other paths). Other
    focal kernels keep their per-cell stores and launch bounds."""
    import re
    M = R
    d = M.from_numpy(np.zeros((512, 512), np.float32), bs=[256, 256])
    src = M.generated_source(W.hillshade(d))
    assert re.search(r"__launch_bounds__\(256, 6\) map_focal_", src)
    assert "tma_store_2d(&a.tm[1], os, t.x0, t.y0 - a.g.oy);" in src
    assert "a.aux[2] != 0 && t.xe == t.x0 + 64 && t.ye == t.y0 + 64" in src
    assert "str_out_row<float>(ob0, op0, k, r0[k]);" in src        # the fallback path
    other = M.generated_source(M.convolve(d, [[1, 2, 1], [2, 4, 2], [1, 2, 1]]) * 0.0625)
    assert "tma_store_2d" not in other and "__launch_bounds__(128) map_focal_" in other
    life = M.generated_source(W.life_step(M.from_numpy(np.zeros((256, 256), np.uint8), bs=[128, 128])))
    assert "tma_store_2d" not in life
