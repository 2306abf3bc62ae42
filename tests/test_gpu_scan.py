"""GPU parity of the Radiating (viewshed radial max) and Spreading (D8 flow
accumulation) skeletons against the CPU oracle (bit-exact)."""
import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def slope_from_observer(dem, obs, h):
    """view.py's slope raster in F32 with the same operator sequence."""
    H, Wd = dem.shape
    xs = obs[0] - np.arange(Wd, dtype=np.int64)[None, :]
    ys = obs[1] - np.arange(H, dtype=np.int64)[:, None]
    d2 = xs * xs + ys * ys                                   # S64
    dist = np.sqrt(d2.astype(np.float32) + np.float32(0.0))   # S64 + F32 -> F32
    shift = dem - np.float32(h)
    with np.errstate(divide="ignore", invalid="ignore"):
        slope = shift / dist
    return slope.astype(np.float32), dist.astype(np.float32)


@pytest.mark.parametrize("shape,obs", [((96, 128), (40, 50)), ((200, 150), (0, 0)), ((129, 257), (256, 64)),
                                        ((64, 64), (31, 63))])
def test_radial_max_bit_exact(M, shape, obs):
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=31, hi=100.0)
    dem = M.from_numpy(dem_np, bs=[64, 64])
    slope_np, dist_np = slope_from_observer(dem_np, obs, 10.0)
    maxr = M.rmax(W.distance(dem, obs) * 0 + (dem - 10.0) / W.distance(dem, obs), obs)
    got = M.to_numpy(maxr)
    ref = O.radial_f32(slope_np, obs, 6)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    m = ~np.isnan(ref)
    assert np.array_equal(got[m], ref[m])


@pytest.mark.parametrize("shape,obs", [((2100, 2300), (700, 1050)), ((2048, 2049), (2048, 2047)), ((3000, 2100), (2099, 13))])
def test_radial_max_cluster_bit_exact(M, shape, obs):
    # rasters of 2048 cells or more across: a cluster of CTAs per octant, each
    # holding a segment of the fronts, the segment edges read from the
    # neighbour's shared memory
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=33, hi=100.0)
    dem = M.from_numpy(dem_np, bs=[512, 512])
    slope_np, dist_np = slope_from_observer(dem_np, obs, 10.0)
    got = M.to_numpy(M.rmax((dem - 10.0) / W.distance(dem, obs), obs))
    ref = O.radial_f32(slope_np, obs, 6)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    m = ~np.isnan(ref)
    assert np.array_equal(got[m], ref[m])


def test_viewshed_program(M):
    dem_np = synth.fbm_dem(160, 200, seed=5, hi=50.0)
    obs = [77, 91]
    dem = M.from_numpy(dem_np, bs=[64, 64])
    view = W.viewshed(dem, obs, 10.0)
    got = M.to_numpy(view)
    slope_np, dist_np = slope_from_observer(dem_np, obs, 10.0)
    maxr = O.radial_f32(slope_np, obs, 6)
    ref = (maxr * dist_np + np.float32(10.0)) - dem_np
    both_nan = np.isnan(got) & np.isnan(ref)
    assert np.array_equal(got[~both_nan], ref[~both_nan])
    # every visible cell has view == 0 and nothing is below the sight line
    assert (got[~both_nan] >= 0).all()


def test_radial_radius_limit(M):
    dem_np = synth.fbm_dem(120, 120, seed=6, hi=20.0)
    obs = [60, 60]
    dem = M.from_numpy(dem_np)
    slope = (dem - 10.0) / W.distance(dem, obs)
    full = M.to_numpy(M.rmax(slope, obs))
    lim = M.to_numpy(M.rmax(slope, obs, radius=20))
    ys, xs = np.mgrid[0:120, 0:120]
    near = np.maximum(np.abs(xs - 60), np.abs(ys - 60)) <= 20
    assert np.array_equal(lim[near], full[near])
    assert np.isnan(lim[~near]).all()


@pytest.mark.parametrize("shape", [(64, 64), (300, 200), (517, 333)])
def test_flow_accumulation_bit_exact(M, shape):
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=13)
    dem = M.from_numpy(dem_np, bs=[128, 128])
    dirs = M.flow_direction(dem)
    acc = M.flow_accumulation(M.ones_like(dem, M.S32), dirs)
    got_dirs = M.to_numpy(dirs)
    got = M.to_numpy(acc)
    ref, cyclic = O.flowacc_s32(np.ones(shape, np.int32), got_dirs)
    assert not cyclic
    assert np.array_equal(got, ref)
    # every cell's upstream count is consistent with its upstream neighbours
    assert got.sum() > 0


@pytest.mark.parametrize("dtype", [np.int32, np.uint32])
def test_flow_accumulation_integer_water_one_cta_sweep(M, dtype):
    # rasters up to 64 K cells take the one-CTA frontier sweep, whose 32-bit
    # integer form carries the sum and the pending count in one 64-bit word
    rng = np.random.default_rng(17)
    shape = (250, 255)
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=23)
    dem = M.from_numpy(dem_np, bs=[128, 128])
    dirs = M.flow_direction(dem)
    lo = -1000 if dtype == np.int32 else 0
    water = rng.integers(lo, 1000, shape).astype(dtype)
    got = M.to_numpy(M.flow_accumulation(M.from_numpy(water, bs=[128, 128]), dirs))
    ref, cyclic = O.flowacc_s32(water.astype(np.int32), M.to_numpy(dirs))
    assert not cyclic
    assert got.dtype == dtype
    assert np.array_equal(got.astype(np.int32), ref)


def test_flow_accumulation_known_answer(M):
    # a ramp falling to the east: every cell drains east (mirrored border reads
    # give no drop), the last column holds pits, and a cell's upstream count is
    # its column index
    dem_np = np.tile(np.arange(40, 0, -1, dtype=np.float32), (10, 1))
    dem = M.from_numpy(dem_np)
    dirs = M.to_numpy(M.flow_direction(dem))
    assert (dirs[:, :-1] == 1).all() and (dirs[:, -1] == 0).all()
    acc = M.to_numpy(M.flow_accumulation(M.ones_like(dem, M.S32), M.from_numpy(dirs)))
    assert np.array_equal(acc, np.tile(np.arange(40, dtype=np.int32), (10, 1)))


def test_flow_accumulation_large_raster_walks_bit_exact(M):
    # a large raster: the grid-wide in-degree pass and downstream walks
    shape = (2100, 2100)
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=21)
    dem = M.from_numpy(dem_np, bs=[512, 512])
    dirs = M.flow_direction(dem)
    got = M.to_numpy(M.flow_accumulation(M.ones_like(dem, M.S32), dirs))
    ref, cyclic = O.flowacc_s32(np.ones(shape, np.int32), M.to_numpy(dirs))
    assert not cyclic
    assert np.array_equal(got, ref)


def test_flow_accumulation_large_raster_integer_water(M):
    # the walk path with the packed (sum, pending) word: signed water with
    # negative values, compared with the oracle
    rng = np.random.default_rng(29)
    shape = (600, 640)
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=24)
    dem = M.from_numpy(dem_np, bs=[256, 256])
    dirs = M.flow_direction(dem)
    water = rng.integers(-500, 500, shape).astype(np.int32)
    got = M.to_numpy(M.flow_accumulation(M.from_numpy(water, bs=[256, 256]), dirs))
    ref, cyclic = O.flowacc_s32(water, M.to_numpy(dirs))
    assert not cyclic
    assert np.array_equal(got, ref)


def test_flow_accumulation_large_raster_float_water(M):
    # float water on the walk path: sums of exactly representable values stay exact
    shape = (2100, 2050)
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=22)
    dem = M.from_numpy(dem_np, bs=[512, 512])
    dirs = M.flow_direction(dem)
    water = np.full(shape, 0.5, np.float32)
    got = M.to_numpy(M.flow_accumulation(M.from_numpy(water, bs=[512, 512]), dirs))
    ref, _ = O.flowacc_s32(np.ones(shape, np.int32), M.to_numpy(dirs))
    assert np.array_equal(got, ref.astype(np.float32) * np.float32(0.5))


@pytest.mark.parametrize("shape,dtype", [((300, 260), np.int32), ((517, 333), np.uint32), ((1024, 1024), np.int32),
                                         ((700, 650), np.int64)])
def test_flow_accumulation_pointer_jumping_equals_walk_and_oracle(fresh, shape, dtype):
    # rasters above 64 K cells: the Euler-tour pointer jumping (fixed rounds) and
    # the downstream walks give the same integer sums, equal to the oracle's
    M = fresh
    rng = np.random.default_rng(41)
    dem_np = synth.fbm_dem(shape[0], shape[1], seed=42)
    dem = M.from_numpy(dem_np, bs=[256, 256])
    dirs = M.flow_direction(dem)
    lo = -700 if np.issubdtype(dtype, np.signedinteger) else 0
    water_np = rng.integers(lo, 700, shape).astype(dtype)
    out = {}
    for cells in (1 << 30, 0):
        M.set_flow_jump_cells(cells)
        out[cells] = M.to_numpy(M.flow_accumulation(M.from_numpy(water_np, bs=[256, 256]), dirs))
    M.set_flow_jump_cells(-1)
    assert np.array_equal(out[1 << 30], out[0])
    d = M.to_numpy(dirs)
    if dtype != np.int64:
        ref, cyclic = O.flowacc_s32(water_np.astype(np.int32), d)
        assert not cyclic
        assert np.array_equal(out[0].astype(np.int32), ref)


def test_flow_accumulation_pointer_jumping_roots_and_edges(fresh):
    # zero codes (pits), invalid codes (several bits) and codes leading out of
    # the raster are roots. Codes E, SE, S, SW never decrease y and E alone
    # keeps it, so the random direction raster is acyclic.
    M = fresh
    rng = np.random.default_rng(43)
    shape = (400, 300)
    codes = np.array([0, 1, 2, 4, 8, 1, 2, 4, 8, 3, 6], np.uint8)
    d = codes[rng.integers(0, len(codes), shape)]
    ref, cyclic = O.flowacc_s32(np.ones(shape, np.int32), d)
    assert not cyclic
    M.set_flow_jump_cells(1 << 30)
    got = M.to_numpy(M.flow_accumulation(M.ones_like(M.from_numpy(d), M.S32), M.from_numpy(d)))
    assert np.array_equal(got, ref)


def test_flow_accumulation_pointer_jumping_reports_a_cycle(fresh):
    # two cells draining into each other: the tour never ends, the kernel sets
    # the error flag after its fixed rounds and the call fails
    M = fresh
    shape = (300, 300)
    d = np.full(shape, 1, np.uint8)         # everything drains east
    d[100, 100], d[100, 101] = 1, 16        # (100,100) -> E, (100,101) -> W: a 2-cycle
    M.set_flow_jump_cells(1 << 30)
    with pytest.raises(M.MapError):
        M.to_numpy(M.flow_accumulation(M.ones_like(M.from_numpy(d), M.S32), M.from_numpy(d)))
    # the engine stays usable
    d[100, 101] = 1
    got = M.to_numpy(M.flow_accumulation(M.ones_like(M.from_numpy(d), M.S32), M.from_numpy(d)))
    assert got[0, 299] == 299
