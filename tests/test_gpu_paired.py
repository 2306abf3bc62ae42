"""Paired cells: float focal groups compute the cells of rows y and y + 1 in one
thread step on packed f32x2 instructions. Every result must be bit-identical to
computing one cell at a time, for every operation the pair form covers, with
special values (NaN, infinities, signed zeros, subnormals, huge and
near-multiple-of-pi/2 arguments) in the input, on ragged rasters (odd row
counts leave a last single row), under every border rule."""
import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture()
def P(fresh):
    yield fresh
    fresh.set_paired_cells(True)


def specials(h, w, seed):
    """A float raster of mixed magnitudes with special values scattered in."""
    rng = np.random.default_rng(seed)
    x = (rng.uniform(-1, 1, (h, w)) * np.exp2(rng.integers(-6, 12, (h, w)))).astype(np.float32)
    sp = np.array([np.nan, np.inf, -np.inf, 0.0, -0.0, 1e-40, -1e-40, 3e38, -3e38, 1e30, 65537.0,
                   np.float32(np.pi / 2), np.float32(-np.pi), np.float32(100 * np.pi)], np.float32)
    idx = rng.choice(h * w, size=(h * w) // 50, replace=False)
    x.ravel()[idx] = sp[rng.integers(0, len(sp), idx.size)]
    return x


def both(M, build):
    """(paired result, one-cell result) of the program build(); checks that the
    paired form was generated when on and not when off."""
    M.set_paired_cells(True)
    r = build()
    assert "focal_cell2" in M.generated_source(r)
    a = M.to_numpy(r)
    M.set_paired_cells(False)
    r = build()
    assert "focal_cell2" not in M.generated_source(r)
    b = M.to_numpy(r)
    M.set_paired_cells(True)
    return a, b


def same(a, b):
    assert a.dtype == b.dtype and a.shape == b.shape
    diff = a.view(np.uint8) != b.view(np.uint8)
    assert not diff.any(), int(diff.sum())


# the fast rewritten form (mode 1, the default) runs one cell at a time; the
# general rewritten form (2) and the literal chain (0) have pair forms
@pytest.mark.parametrize("rewrite", [2, 0])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_hillshade_paired_bit_identical(P, border, rewrite):
    M = P
    M.set_border(border)
    M.set_algebraic_rewrite(rewrite)
    dem = synth.fbm_dem(777, 1000, seed=4)
    dem.ravel()[::997] = np.nan
    dem.ravel()[5::1999] = -0.0
    a, b = both(M, lambda: W.hillshade(M.from_numpy(dem, bs=[256, 256])))
    same(a, b)


def test_every_pair_form_operation(P):
    M = P
    h, w = 515, 389
    x = specials(h, w, 1)
    z = np.random.default_rng(2).integers(-50, 50, (h, w)).astype(np.int32)
    k3 = [[1, 2, 1], [2, 4, 2], [1, 2, 1]]
    lap = [[0, -1, 0], [-1, 5, -1], [0, -1, 0]]
    box = [[1, 1, 1], [1, 1, 1], [1, 1, 1]]

    def prog():
        r = M.from_numpy(x, bs=[128, 128])
        zi = M.from_numpy(z, bs=[128, 128])
        c = M.convolve(r, k3) / 16                   # division by a power of two
        d = M.convolve(r, lap) / 3                   # and by another literal
        n = r([1, -1])                               # neighbour access
        fm, fn, fs = M.fmax(r, box), M.fmin(r, box), M.fsum(r)
        s = M.sin(c) * M.cos(c) + M.sin(d) * 1 + 1 * M.cos(n)
        t = M.atan2(n, d) + M.sqrt(M.abs(c)) + M.atan(fm) + M.exp(M.fmin(r, box) * 1e-3)
        u = M.con(c > d, M.pow(M.abs(n), 0.5), M.hypot(fm, fn)) + M.fmod(c, 3.0) + c * c + d * n
        ix = M.index(r, M.D1).astype(M.F32) * 0.5 - M.index(r, M.D2).astype(M.F32)
        zu = M.abs(zi).astype(M.U32)
        u2, u12 = M.full_like(2, zu, M.U32), M.full_like(12, zu, M.U32)
        zz = (zu * 3 + 7) % 5 + (zu >> u2) + (zu & u12) + (zu ^ u2) + (~zu | u2)
        b = ((c > 0) & (d < 1)) | (zi > 2)
        return (s + t + u + ix + zz.astype(M.F32) + b * 2.0 + M.max(c, d) - M.min(n, fs) + (-c)
                + (zi == 0) * fn)
    a, b = both(M, prog)
    same(a, b)


def test_integer_and_boolean_outputs(P):
    M = P
    h, w = 301, 257
    x = specials(h, w, 3)

    def prog():
        r = M.from_numpy(x, bs=[128, 128])
        c = M.convolve(r, [[1, 0, -1], [2, 0, -2], [1, 0, -1]])
        return (M.atan2(c, r) > 0.5) + (M.sqrt(M.abs(c)) < 3)      # U8 output
    a, b = both(M, prog)
    same(a, b)

    def prog_s32():
        r = M.from_numpy(x, bs=[128, 128])
        c = M.convolve(r, [[1, 1, 1], [1, 1, 1], [1, 1, 1]])
        return M.floor(M.sin(c) * 1000).astype(M.S32) + M.index(r, M.D2).astype(M.S32)
    a, b = both(M, prog_s32)
    same(a, b)


@pytest.mark.parametrize("bs", [[64, 64], [100, 60], [256, 256]])
def test_plain_mode_blocks(P, bs):
    M = P
    M.set_exec_mode(M.EXEC_PLAIN)
    M.set_algebraic_rewrite(2)
    dem = synth.fbm_dem(333, 517, seed=8)
    a, b = both(M, lambda: W.hillshade(M.from_numpy(dem, bs=bs)))
    same(a, b)


@pytest.mark.parametrize("rewrite", [True, False])
def test_paired_hillshade_matches_oracle(P, rewrite):
    from oracle import oracle as O
    M = P
    M.set_algebraic_rewrite(rewrite)
    dem = synth.fbm_dem(300, 500, seed=6)
    got = M.to_numpy(W.hillshade(M.from_numpy(dem, bs=[128, 128])))
    ref = O.hillshade_f32(dem, (128, 128), 0)
    ok, d, only = O.hill_tolerance(got, ref, O.hillshade_bound(dem, (128, 128), 0))
    assert ok.all()
