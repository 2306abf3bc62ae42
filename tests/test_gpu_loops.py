"""While-loops over 2-D rasters on the GPU (the reference's symbolic loops,
python/map.py:234-330, which its runtime cannot execute): one evaluation per
iteration with the loop-carried rasters resident in device memory, results
bit-identical to the same loop over NumPy arrays or to the oracle."""
import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

K3 = [[1, 1, 1], [1, 1, 1], [1, 1, 1]]


def dilate_np(x, mask):
    p = np.pad(x, 1)
    h, w = x.shape
    m = np.max(np.stack([p[i:i + h, j:j + w] for i in range(3) for j in range(3)]), axis=0)
    return (m * mask).astype(np.int32)


@pytest.mark.parametrize("shape,bs", [((300, 500), (128, 128)), ((257, 129), (64, 64))])
def test_dilation_until_it_stops_growing(fresh, shape, bs):
    """Grow a seed inside a mask until no cell is added: a raster carried
    across iterations, a scalar test from a zonal sum over the body's result."""
    M = fresh
    M.set_border(2)                                  # dead border: reads outside are 0
    rng = np.random.default_rng(5)
    h, w = shape
    mask = (rng.random((h, w)) < 0.65).astype(np.int32)
    seed = np.zeros((h, w), np.int32)
    seed[h // 2, w // 3] = 1
    mask[h // 2, w // 3] = 1
    x = M.from_numpy(seed, bs=list(bs))
    m = M.from_numpy(mask, bs=list(bs))
    d = M.ones(dt=M.S32)
    n = 0
    per_iteration = []
    while d > 0:
        per_iteration.append(M.last_launch_count())  # the evaluation that ran the previous test
        y = M.fmax(x, K3) * m
        d = M.zsum(y - x)
        x = y
        n += 1
    xs, cnt, dd = seed, 0, 1
    while dd > 0:
        ys = dilate_np(xs, mask)
        dd = int((ys - xs).sum())
        xs, cnt = ys, cnt + 1
    assert n == cnt and n > 10
    got = M.to_numpy(x)
    assert M.last_launch_count() == 0                # x is resident: nothing recomputed
    assert np.array_equal(got, xs)
    # each iteration evaluates its own groups only, not the loop's history
    assert max(per_iteration[2:]) <= 4 and max(per_iteration[2:]) == min(per_iteration[2:])
    M.collect_garbage()
    assert M.node_count() < 64


@pytest.mark.parametrize("border", [0, 2])
def test_life_generations_counted_by_a_scalar_raster(fresh, border):
    """life.py's generations under a raster counter: `while g < 20`."""
    M = fresh
    M.set_border(border)
    init = synth.bernoulli_u8(200, 300, 0.3, seed=9)
    s = M.from_numpy(init, bs=[64, 64])
    g = M.zeros(dt=M.S32)
    while g < 20:
        s = W.life_step(s)
        g = g + 1
    assert M.value(g) == 20
    want = O.life(init, (64, 64), 20, border)
    assert np.array_equal(M.to_numpy(s), want)


def test_materialize_keeps_a_raster_resident(fresh):
    M = fresh
    a = synth.fbm_dem(256, 384, seed=3)
    r = M.from_numpy(a, bs=[128, 128])
    hs = W.hillshade(r)
    (kept,) = M.materialize(hs)
    first = M.to_numpy(kept)
    assert M.last_launch_count() == 0
    assert np.array_equal(first, M.to_numpy(hs))
    again = M.to_numpy(kept * 2.0)
    assert np.array_equal(again, first * np.float32(2.0))
