"""The packed byte-cell form (Q4 in skeleton/common.cuh: four cells of a row as
16-bit lanes of two 32-bit words) on the CPU.

The lane identities the device helpers rely on are replayed with 32-bit
unsigned NumPy arithmetic over every boundary value of a lane and random
samples (no carry or borrow crosses a lane for operands in [0, 0x7FFF]), and
the code generator's choice of the form is checked: integer bodies on byte
rasters take it, bodies whose values could leave the lanes' range do not."""
import numpy as np
import pytest

from map_b200 import workloads as W

u32 = np.uint32
LANE = np.array(sorted({0, 1, 2, 3, 127, 128, 254, 255, 256, 257, 0x3FFF, 0x4000, 0x7FFE, 0x7FFF} |
                       set(np.random.default_rng(5).integers(0, 0x8000, 200).tolist())), np.uint64)


def pairs():
    a, b = np.meshgrid(LANE, LANE, indexing="ij")
    return a.ravel(), b.ravel()


def word(lo, hi):
    return ((hi << 16) | lo).astype(u32)


def lanes(w):
    w = w.astype(np.uint64)
    return w & 0xFFFF, w >> 16


# the device helpers, restated in 32-bit unsigned arithmetic
def ne0_w(a):
    return ((a + u32(0x7FFF7FFF)) & u32(0x80008000)) >> u32(15)


def ge_w(a, b):
    return (((a | u32(0x80008000)) - b) & u32(0x80008000)) >> u32(15)


def mul01_w(m, b):
    return (m * u32(0xFFFF)) & b


def mul_w(a, b):
    return ((a & u32(0xFFFF)) * (b & u32(0xFFFF))) | (((a >> u32(16)) * (b >> u32(16))) << u32(16))


def test_relations_never_cross_lanes():
    a, b = pairs()
    rng = np.random.default_rng(1)
    # each lane of a word paired with an independent partner lane
    c, d = rng.permutation(a), rng.permutation(b)
    A, B = word(a, c), word(b, d)
    with np.errstate(over="ignore"):
        for got, want in ((ne0_w(A ^ B), (a != b, c != d)), (ge_w(A, B), (a >= b, c >= d)),
                          (ge_w(B, A), (b >= a, d >= c)), (ne0_w(A), (a != 0, c != 0))):
            lo, hi = lanes(got)
            assert np.array_equal(lo, want[0].astype(np.uint64)) and np.array_equal(hi, want[1].astype(np.uint64))


def test_sums_products_and_masks_stay_in_their_lanes():
    a, b = pairs()
    rng = np.random.default_rng(2)
    c, d = rng.permutation(a), rng.permutation(b)
    A, B = word(a, c), word(b, d)
    with np.errstate(over="ignore"):
        lo, hi = lanes((A + B).astype(u32))          # sums below 0x10000
        assert np.array_equal(lo, a + b) and np.array_equal(hi, c + d)
        keep = (a >= b) & (c >= d)                    # differences that stay non-negative
        lo, hi = lanes((A - B).astype(u32)[keep])
        assert np.array_equal(lo, (a - b)[keep]) and np.array_equal(hi, (c - d)[keep])
        m = word(a & 1, c & 1)
        lo, hi = lanes(mul01_w(m, B))
        assert np.array_equal(lo, (a & 1) * b) and np.array_equal(hi, (c & 1) * d)
        small = (a * b < 0x10000) & (c * d < 0x10000)
        lo, hi = lanes(mul_w(A, B)[small])
        assert np.array_equal(lo, (a * b)[small]) and np.array_equal(hi, (c * d)[small])
        lo, hi = lanes((A + B).astype(u32) & u32(0x00FF00FF))   # mod-256 reduction lane by lane
        assert np.array_equal(lo, (a + b) & 255) and np.array_equal(hi, (c + d) & 255)


def byte_perm(x, y, s):
    """__byte_perm(x, y, s) for selectors whose nibbles are 0-7 (CUDA's
    documented byte selection from the 8 bytes of y:x)."""
    src = (np.asarray(y, np.uint64) << 32) | np.asarray(x, np.uint64)
    out = np.zeros_like(src)
    for i in range(4):
        sel = (s >> (4 * i)) & 7
        out |= ((src >> (8 * sel)) & 0xFF) << (8 * i)
    return out.astype(u32)


def q4_even(w):
    return byte_perm(w, 0, 0x4240)


def q4_odd(w):
    return byte_perm(w, 0, 0x4341)


def tap4(words, lx, dx):
    """SmemTap::tap4 restated: the interleaved lanes (lo: cells 0 and 2, hi:
    cells 1 and 3 of lx + dx .. lx + dx + 3) from the aligned words."""
    o, m = dx & 3, (dx - (dx & 3)) // 4
    W = lambda k: u32(words[lx // 4 + k])
    e = lambda k: byte_perm(q4_even(W(k)), W(k + 1), 0x1412)
    od = lambda k: byte_perm(W(k), q4_odd(W(k + 1)), 0x5453)
    if o == 0:
        return q4_even(W(m)), q4_odd(W(m))
    if o == 1:
        return q4_odd(W(m)), e(m)
    if o == 2:
        return e(m), od(m)
    return od(m), q4_even(W(m + 1))


def test_byte_lanes_round_trip_and_taps():
    rng = np.random.default_rng(3)
    row = rng.integers(0, 256, 96, dtype=np.uint8)
    words = row.view("<u4")
    for lx in range(16, 64, 4):
        for dx in range(-16, 17):
            lo, hi = tap4(words, lx, dx)
            cells = [int(lo) & 0xFFFF, int(hi) & 0xFFFF, int(lo) >> 16, int(hi) >> 16]
            assert cells == row[lx + dx:lx + dx + 4].tolist(), (lx, dx)
            v = words[(lx + dx) // 4] if dx % 4 == 0 else None
            if v is not None:                                     # q4_pack_u8 undoes q4_bytes
                assert int(byte_perm(lo, hi, 0x6240)) == int(v)


def test_life_takes_the_packed_form(M):
    s = M.from_numpy(np.zeros((256, 512), np.uint8), bs=[256, 256])
    src = M.generated_source(W.life_step(s))
    assert "focal_cell4(" in src and "q4_eq(" in src and "str_out_row<u32>" in src
    assert M.compile_only(W.life_step(s)) == 1


def test_packed_form_only_where_lanes_provably_hold(fresh):
    M = fresh
    s = M.from_numpy(np.zeros((256, 512), np.uint8), bs=[256, 256])
    big = [[300, 300, 300], [300, 300, 300], [300, 300, 300]]     # 9 x 300 x 255 > 0xFFFF
    cases = {
        "weights": M.convolve(s, big) > 5,
        "float": (M.convolve(s, [[1, 1, 1], [1, 0, 1], [1, 1, 1]]) * 0.5) > 1.0,
        "negative": M.convolve(s, [[1, 1, 1], [1, 0, 1], [1, 1, 1]]) - 9 > 0,
        "s32 out": M.convolve(s, [[1, 1, 1], [1, 0, 1], [1, 1, 1]]),
    }
    for name, r in cases.items():
        assert "focal_cell4(" not in M.generated_source(r), name
    # a difference the intervals show non-negative: [300, 4380] - [0, 255]
    ok = (M.convolve(s, [[1, 2, 1], [2, 4, 2], [1, 2, 1]]) + 300) - M.convolve(s, [[0, 0, 0], [0, 1, 0], [0, 0, 0]]) > 700
    assert "focal_cell4(" in M.generated_source(ok)
    M.set_paired_cells(False)
    assert "focal_cell4(" not in M.generated_source(W.life_step(s))
