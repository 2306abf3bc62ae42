"""GPU parity of the focal skeleton (TMA-staged tiles + border gather path)
against the CPU oracle: hillshade (float, within tolerance) and Game of Life,
generic correlations, neighbour reads, focal min/max and D8 flow directions
(bit-exact)."""
import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def hill_check(gpu, dem_np, bs, border):
    """Hillshade against the oracle: within 4 ulp or 1e-5 relative of the FP32
    oracle, or, where the formula's two terms cancel, within 4 times the FP32
    chain's own first-order rounding-error scale at the cell (O.hill_tolerance);
    and no further from the FP64 value than the FP32 restatement, up to 4 ulp of 1.
    Returns the share of cells that pass only through the cancellation clause."""
    ref32 = O.hillshade_f32(dem_np, bs, border)
    ref64 = O.hillshade_f64(dem_np, bs, border)
    ok, d, only = O.hill_tolerance(gpu, ref32, O.hillshade_bound(dem_np, bs, border))
    bad = np.argwhere(~ok)
    assert ok.all(), "%d cells out of tolerance, first %s: gpu %r ref %r" % (
        len(bad), bad[:3].tolist(), gpu[tuple(bad[0])], ref32[tuple(bad[0])])
    err_gpu = np.nanmax(np.abs(gpu - ref64))
    err_ref = np.nanmax(np.abs(ref32 - ref64))
    assert err_gpu <= err_ref + 4 * float(np.spacing(np.float32(1.0)))
    return ref32, only.mean()


@pytest.mark.parametrize("rewrite", [True, False])
@pytest.mark.parametrize("shape,bs,border,mode", [
    ((1024, 1024), (256, 256), 0, 0),
    ((1024, 1024), (256, 256), 0, 1),
    ((300, 500), (128, 128), 0, 0),
    ((257, 129), (64, 64), 0, 1),
    ((300, 500), (128, 128), 1, 0),
    ((190, 333), (64, 64), 2, 0),
    ((64, 64), (64, 64), 0, 0),
    ((1, 40), (16, 16), 1, 0),
    ((300, 500), (500, 300), 0, 0),   # one block: edge tiles staged like interior ones
    ((200, 270), (90, 70), 0, 1),     # plain launches from block origins not on a 16-byte boundary
    ((190, 333), (100, 60), 1, 1),
])
def test_hillshade_matches_oracle(fresh, shape, bs, border, mode, rewrite):
    M = fresh
    M.set_border(border)
    M.set_exec_mode(mode)
    M.set_algebraic_rewrite(rewrite)
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=7)
    dem = M.from_numpy(dem_np, bs=list(bs))
    hs = W.hillshade(dem)
    assert ("map_shade" in M.generated_source(hs)) == rewrite
    gpu = M.to_numpy(hs)
    assert M.last_launch_count() >= 1
    ref32, only = hill_check(gpu, dem_np, bs, border)
    # the literal chain is bit-identical to the FP32 restatement on the large
    # majority of cells (differences come only from transcendental-function
    # implementations); the rewrite evaluates none of them
    if gpu.size >= 4096 and not rewrite:
        assert (gpu == ref32).mean() > 0.5
    assert only < 0.02


def test_hillshade_rewrite_literal_chain_where_not_finite(fresh):
    """Cells whose x^2 + y^2 is not finite (NaN or infinite DEM cells, gradients
    above 1.8e19) take the literal chain: identical to the switch turned off."""
    M = fresh
    dem_np = synth.fbm_dem(200, 300, seed=11)
    dem_np.ravel()[::503] = np.nan
    dem_np.ravel()[7::701] = np.inf
    dem_np.ravel()[11::907] = -np.inf
    dem_np.ravel()[13::1009] = 3e25
    dem_np.ravel()[17::1103] = -1e30
    out = {}
    for rw in (True, False):
        M.set_algebraic_rewrite(rw)
        out[rw] = M.to_numpy(W.hillshade(M.from_numpy(dem_np, bs=[64, 64])))
    x = O.conv_f32(dem_np, np.array([[-1, 0, 1], [-2, 0, 2], [-1, 0, 1]], np.float32), (64, 64)) * np.float32(0.125)
    y = O.conv_f32(dem_np, np.array([[-1, -2, -1], [0, 0, 0], [1, 2, 1]], np.float32), (64, 64)) * np.float32(0.125)
    with np.errstate(over="ignore", invalid="ignore"):
        q = np.float32(x) * x + np.float32(y) * y
    lit = ~(q < np.inf)
    assert lit.sum() > 100
    a, b = out[True][lit], out[False][lit]
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    fin = ~lit
    ref32 = O.hillshade_f32(dem_np, (64, 64), 0)
    bound = O.hillshade_bound(dem_np, (64, 64), 0)
    ok, d, only = O.hill_tolerance(out[True][fin], ref32[fin], bound[fin])
    assert ok.all()


def test_hillshade_fused_and_plain_are_identical(fresh):
    M = fresh
    dem_np = synth.fbm_dem(512, 768, seed=3)
    dem = M.from_numpy(dem_np, bs=[128, 256])
    hs = W.hillshade(dem)
    M.set_exec_mode(M.EXEC_FUSED)
    a = M.to_numpy(hs)
    M.set_exec_mode(M.EXEC_PLAIN)
    b = M.to_numpy(hs)
    assert M.last_launch_count() == 6 * 2      # one launch per block (6 x 2 blocks)
    assert np.array_equal(a, b)


def test_hillshade_constant_dem_known_answer(M):
    dem = M.from_numpy(np.full((96, 160), 1234.5, np.float32), bs=[32, 32])
    hs = M.to_numpy(W.hillshade(dem))
    # flat terrain: slope 0, hillshade = cos(zenith angle) in F32
    assert np.all(hs == np.float32(np.cos((90 - 45.0) / 180 * 3.141593)))


@pytest.mark.parametrize("border", [0, 2])
def test_life_bit_exact(fresh, border):
    M = fresh
    M.set_border(border)
    st_np = synth.bernoulli_u8(256, 384, 0.3, seed=11)
    st = M.from_numpy(st_np, bs=[64, 64])
    out = M.to_numpy(W.life(st, 12))
    ref = O.life(st_np, (64, 64), 12, border)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("border,bs,mode", [(0, (100, 60), 1), (2, (100, 60), 1), (1, (384, 256), 0)])
def test_life_odd_blocks_and_staged_edges_bit_exact(fresh, border, bs, mode):
    # U8 rasters stage in 16-byte units: plain launches from block origins at x = 100,
    # 200, ... take the gather path; one-block rasters stage their edge tiles too
    M = fresh
    M.set_border(border)
    M.set_exec_mode(mode)
    st_np = synth.bernoulli_u8(256, 384, 0.3, seed=12)
    out = M.to_numpy(W.life(M.from_numpy(st_np, bs=list(bs)), 6))
    ref = O.life(st_np, bs, 6, border)
    assert np.array_equal(out, ref)


def test_life_known_patterns(fresh):
    M = fresh
    M.set_border(M.BORDER_DEAD)
    g = np.zeros((32, 32), np.uint8)
    g[10, 9:12] = 1                      # blinker
    g[20:22, 20:22] = 1                  # block (still life)
    glider = np.zeros((32, 32), np.uint8)
    glider[1, 2] = glider[2, 3] = glider[3, 1] = glider[3, 2] = glider[3, 3] = 1
    r1 = M.to_numpy(W.life(M.from_numpy(g, bs=[16, 16]), 1))
    assert r1[9:12, 10].tolist() == [1, 1, 1] and r1[10, 9] == 0
    assert np.array_equal(r1[20:22, 20:22], np.ones((2, 2), np.uint8))
    r2 = M.to_numpy(W.life(M.from_numpy(g, bs=[16, 16]), 2))
    assert np.array_equal(r2, g)
    r4 = M.to_numpy(W.life(M.from_numpy(glider, bs=[16, 16]), 4))
    assert np.array_equal(r4, np.roll(np.roll(glider, 1, 0), 1, 1))   # glider moves (1,1) every 4 generations


def test_life_initial_state_from_rand(M):
    ds, bs = [200, 120], [64, 64]
    st = W.life_initial(ds, bs, seed=16)
    got = M.to_numpy(st)
    ref = (O.rand_u8(16, (ds[1], ds[0]), bs) > 128).astype(np.uint8)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("border", [0, 1, 2])
def test_generic_correlation_bit_exact(fresh, border):
    M = fresh
    M.set_border(border)
    a = synth.uniform_f32(200, 300, seed=5)
    masks = [np.array([[1.0 / 16, 1.0 / 8, 1.0 / 16], [1.0 / 8, 1.0 / 4, 1.0 / 8], [1.0 / 16, 1.0 / 8, 1.0 / 16]], np.float32),
             np.arange(25, dtype=np.float32).reshape(5, 5) / 7.0,
             np.array([[0.5, -1.25, 3.0]], np.float32)]
    r = M.from_numpy(a, bs=[64, 64])
    for m in masks:
        # the reference writes float masks into kernel text with six decimals
        mr = np.array([[float("%f" % v) for v in row] for row in m], np.float32)
        got = M.to_numpy(M.convolve(r, m.tolist()))
        ref = O.conv_f32(a, mr, (64, 64), border)
        assert np.array_equal(got, ref)


def test_neighbor_and_focal_minmax(fresh):
    M = fresh
    a = synth.uniform_f32(130, 70, seed=9)
    r = M.from_numpy(a, bs=[32, 32])
    for border in (0, 1, 2):
        M.set_border(border)
        got = M.to_numpy(r([1, -2]) - r([0, 1]))
        H, Wd = a.shape

        def at(x, y, dx, dy):
            s = O.focal_src(Wd, H, (32, 32), border, x, y, dx, dy)
            return np.float32(0) if s is None else a[s[1], s[0]]
        ref = np.array([[np.float32(at(x, y, 1, -2) - at(x, y, 0, 1)) for x in range(Wd)] for y in range(H)], np.float32)
        assert np.array_equal(got, ref)
        mn = M.to_numpy(M.fmin(r, [[1, 1, 1]] * 3))
        refmn = np.array([[min(at(x, y, dx, dy) for dy in (-1, 0, 1) for dx in (-1, 0, 1)) for x in range(Wd)]
                          for y in range(H)], np.float32)
        assert np.array_equal(mn, refmn)


def test_d8_flow_direction_bit_exact(fresh):
    M = fresh
    dem_np = synth.fbm_dem(300, 200, seed=21)
    for border in (0, 2):
        M.set_border(border)
        got = M.to_numpy(M.flow_direction(M.from_numpy(dem_np, bs=[64, 64])))
        assert np.array_equal(got, O.d8(dem_np, (64, 64), border))


def test_block_mirror_corner_rule(fresh):
    """At the raster edge a read that also crosses a block boundary is served
    from the centre cell's own block (runtime/skeleton/util.cpp:498-506)."""
    M = fresh
    M.set_border(M.BORDER_BLOCK_MIRROR)
    a = np.arange(64 * 64, dtype=np.float32).reshape(64, 64)
    r = M.from_numpy(a, bs=[32, 32])
    got = M.to_numpy(r([-1, -1]))
    # cell (32, 0) is the first column of block (1,0): its up-left read mirrors
    # inside block (1,0) to (32, 0), not to (31, 0) of the neighbouring block
    assert got[0, 32] == a[0, 32]
    assert got[0, 31] == a[0, 30]
    M.set_border(M.BORDER_RASTER_MIRROR)
    got = M.to_numpy(r([-1, -1]))
    assert got[0, 32] == a[0, 31]


@pytest.mark.parametrize("typ", [1, 2])
@pytest.mark.parametrize("dtype,border", [(np.float32, 0), (np.float32, 1), (np.uint8, 2), (np.uint8, 0)])
def test_focal_percent_matches_oracle(fresh, typ, dtype, border):
    """FocalPercent (percentage: share of the window equal to the centre;
    percentile: share below it), 3x3 and 5x3 windows, bit-exact."""
    M = fresh
    M.set_border(border)
    rng = np.random.default_rng(31 + typ)
    a_np = (rng.integers(0, 6, size=(150, 211))).astype(dtype)     # few values: many ties
    a = M.from_numpy(a_np, bs=[64, 64])
    fn = M.percentage if typ == 1 else M.percentile
    for mask, (hx, hy) in (([[1, 1, 1]] * 3, (1, 1)), ([[1, 2, 3, 4, 5]] * 3, (2, 1))):
        got = M.to_numpy(fn(a, mask))
        ref = O.focal_percent(a_np, hx, hy, typ, (64, 64), border)
        assert got.dtype == ref.dtype
        assert np.array_equal(got, ref), (mask, int((got != ref).sum()))


@pytest.mark.parametrize("shape,bs,border", [((1024, 1024), (256, 256), 0), ((300, 500), (128, 128), 1),
                                              ((190, 333), (64, 64), 2), ((257, 129), (64, 64), 0)])
def test_hillshade_fast_form_equals_general_form(fresh, shape, bs, border):
    """The fast form of the rewrite (Sobel sums without zero weights, 1/8 and the
    light direction folded into constants) is bit-identical to the general
    rewritten form, including flat cells, NaN and infinite DEM cells."""
    M = fresh
    M.set_border(border)
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=17)
    dem_np[::29, ::31] = 100.0
    dem_np[5::97, 3::89] = np.nan
    dem_np[7::113, 11::101] = np.inf
    out = {}
    for mode in (1, 2):
        M.set_algebraic_rewrite(mode)
        r = W.hillshade(M.from_numpy(dem_np, bs=list(bs)))
        assert ("map_shade_fast" in M.generated_source(r)) == (mode == 1)
        out[mode] = M.to_numpy(r)
    assert np.array_equal(out[1].view(np.uint32), out[2].view(np.uint32))


@pytest.mark.parametrize("shape,bs", [((47, 65), (16, 16)), ((50, 49), (8, 16)), ((34, 97), (32, 8)),
                                      ((300, 257), (128, 128))])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_wide_halo_edges_bit_exact(fresh, shape, bs, border):
    """A 5 x 5 correlation on rasters whose last block is narrower than the halo
    (the reference's in-block reflection clamps there): staged edge tiles plus
    the recomputed block-mirror cells equal the oracle cell for cell."""
    M = fresh
    M.set_border(border)
    rng = np.random.default_rng(44)
    a = rng.integers(-50, 50, shape).astype(np.float32)
    mask = rng.integers(-3, 4, (5, 5)).astype(np.float32)
    got = M.to_numpy(M.convolve(M.from_numpy(a, bs=list(bs)), mask.tolist()))
    ref = O.conv_f32(a, mask, bs, border)
    assert np.array_equal(got, ref)
