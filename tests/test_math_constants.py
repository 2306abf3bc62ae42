"""The engine's own float32 sine, cosine and atan2 (map_common.cuh) on the CPU:
the constants are read from the shipped header and the device operation
sequence is replayed in float32 (fused multiply-adds emulated in float64, whose
48-bit products are exact), so the fitted polynomials and the Cody-Waite split
of pi/2 are checked without a GPU: within 2 ulp of the correctly rounded value
on samples of every range the device code takes, including the floats nearest
to multiples of pi/2. The GPU tests check the compiled code itself."""
import os
import re

import numpy as np

HDR = os.path.join(os.path.dirname(__file__), "..", "map_b200", "csrc", "skeleton", "common.cuh")
f32 = np.float32


def consts():
    src = open(HDR).read()
    out = {}
    for name, val in re.findall(r"#define (MAP_[A-Z0-9_]+) (-?0x[0-9a-fp.+-]+)f\b", src):
        out[name] = f32(float.fromhex(val))
    return out


C = consts()


def fma(a, b, c):
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(f32)


def mul(a, b):
    return (np.asarray(a, f32) * np.asarray(b, f32)).astype(f32)


def sincos(x):
    x = np.asarray(x, f32)
    t = fma(x, C["MAP_2OPI"], C["MAP_RINT"])
    j = (t - C["MAP_RINT"]).astype(f32)
    q = t.view(np.uint32)
    r = fma(j, -C["MAP_PIO2_1"], x)
    r = fma(j, -C["MAP_PIO2_2"], r)
    r = fma(j, -C["MAP_PIO2_3"], r)
    s = mul(r, r)
    p = fma(s, C["MAP_SIN_3"], C["MAP_SIN_2"])
    p = fma(s, p, C["MAP_SIN_1"])
    sr = fma(mul(r, s), p, r)
    sr = (sr.view(np.uint32) | (r.view(np.uint32) & np.uint32(0x80000000))).view(f32)
    c = fma(s, C["MAP_COS_4"], C["MAP_COS_3"])
    c = fma(s, c, C["MAP_COS_2"])
    c = fma(s, c, C["MAP_COS_1"])
    cr = fma(s, c, f32(1))
    odd = (q & 1) == 1
    so = np.where(odd, cr, sr).view(np.uint32) ^ ((q << np.uint32(30)) & np.uint32(0x80000000))
    co = np.where(odd, sr, cr).view(np.uint32) ^ (((q + np.uint32(1)) << np.uint32(30)) & np.uint32(0x80000000))
    return so.view(f32), co.view(f32)


def atan2(y, x):
    y, x = np.asarray(y, f32), np.asarray(x, f32)
    ax, ay = np.abs(x), np.abs(y)
    mx, mn = np.maximum(ax, ay), np.minimum(ax, ay)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = (mn / mx).astype(f32)
    t = np.where((ax == 0) & (ay == 0), f32(0), t)
    s = mul(t, t)
    q = np.full_like(t, C["MAP_ATAN_Q0"])
    for k in range(1, 9):
        q = fma(q, s, C["MAP_ATAN_Q%d" % k])
    r = fma(mul(t, s), q, t)
    neg = np.signbit(x)
    pio2_lo, pio2_hi = f32(-float.fromhex("0x1.777a5cp-25")), f32(float.fromhex("0x1.921fb6p+0"))
    pi_lo, pi_hi = f32(-float.fromhex("0x1.777a5cp-24")), f32(float.fromhex("0x1.921fb6p+1"))
    up = np.where(neg, ((pio2_lo + r).astype(f32) + pio2_hi).astype(f32), ((pio2_lo - r).astype(f32) + pio2_hi).astype(f32))
    back = ((pi_lo - r).astype(f32) + pi_hi).astype(f32)
    r = np.where(ay > ax, up, np.where(neg, back, r))
    return np.copysign(r, y).astype(f32)


def ulp_err(got, ref):
    ulp = np.spacing(np.abs(ref).astype(f32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - ref) / ulp


def test_constants_parsed():
    for k in ("MAP_2OPI", "MAP_PIO2_1", "MAP_PIO2_2", "MAP_PIO2_3", "MAP_SIN_1", "MAP_COS_4", "MAP_ATAN_Q0", "MAP_ATAN_Q8"):
        assert k in C, k
    # pi/2 = P1 + P2 + P3 to float64 precision, each part positive
    total = float(C["MAP_PIO2_1"]) + float(C["MAP_PIO2_2"]) + float(C["MAP_PIO2_3"])
    assert abs(total - np.pi / 2) < 1e-16
    assert C["MAP_PIO2_1"] > 0 and C["MAP_PIO2_2"] > 0 and C["MAP_PIO2_3"] > 0


def test_sin_cos_within_2_ulp():
    rng = np.random.default_rng(1)
    parts = [rng.uniform(-b, b, 200000) for b in (0.8, 4.0, 1024.0, 65536.0)]
    k = np.arange(1, 40000)
    near = (k * (np.pi / 2)).astype(f32)
    parts += [near, np.nextafter(near, f32(np.inf)), np.nextafter(near, f32(-np.inf)), -near]
    x = np.concatenate(parts).astype(f32)
    s, c = sincos(x)
    assert ulp_err(s, np.sin(x.astype(np.float64))).max() <= 2.0
    assert ulp_err(c, np.cos(x.astype(np.float64))).max() <= 2.0


def test_sin_cos_signed_zero_and_tiny():
    x = np.array([0.0, -0.0, 1e-30, -1e-30, 1e-45], f32)
    s, c = sincos(x)
    assert np.array_equal(s, x) and np.array_equal(np.signbit(s), np.signbit(x))
    assert (c == 1).all()


def test_atan2_within_2_ulp():
    rng = np.random.default_rng(2)
    n = 400000
    y = (rng.uniform(-1, 1, n) * np.exp2(rng.uniform(-40, 40, n))).astype(f32)
    x = (rng.uniform(-1, 1, n) * np.exp2(rng.uniform(-40, 40, n))).astype(f32)
    got = atan2(y, x)
    assert ulp_err(got, np.arctan2(y.astype(np.float64), x.astype(np.float64))).max() <= 2.0


def test_packed_flow_word_arithmetic():
    """The flow sweep's 64-bit cell word: sum in the high half, pending pushes in
    the low half; a push adds (value << 32) - 1. Whatever the order of the
    pushes, the count never borrows, the push that sees the count at 1 is the
    last, and old sum + its value is the 32-bit wrap-around sum of all pushes."""
    rng = np.random.default_rng(3)
    M64 = (1 << 64) - 1
    for trial in range(2000):
        k = int(rng.integers(1, 9))
        vals = [int(v) for v in rng.integers(-2 ** 31, 2 ** 31, k)]
        word = k                                  # the in-degree count, sum 0
        last = None
        for i in rng.permutation(k):
            v = vals[i] & 0xFFFFFFFF
            old = word
            word = (word + ((v << 32) - 1)) & M64
            assert (old & 0xFFFFFFFF) >= 1        # no borrow out of the count
            if (old & 0xFFFFFFFF) == 1:
                assert last is None
                last = (((old >> 32) + v) & 0xFFFFFFFF)
        want = sum(vals) & 0xFFFFFFFF
        assert last == want and (word & 0xFFFFFFFF) == 0 and (word >> 32) == want
