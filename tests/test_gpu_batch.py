"""Batched persistent execution: many rasters of uneven size, each running the
fused hillshade group and a weighted overlay, in one persistent launch; results
are bit-identical to evaluating every raster on its own."""
import ctypes as ct

import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W

pytestmark = pytest.mark.gpu


class DevBuf:
    def __init__(self, M, shape, dtype=np.float32):
        self.M = M
        self.shape = shape
        self.dtype = np.dtype(dtype)
        self.pitch = ((shape[1] * self.dtype.itemsize + 127) // 128) * 128
        self.nbytes = self.pitch * shape[0]
        self.ptr = M._lib.ma_devAlloc(self.nbytes)

    def numpy(self):
        raw = np.empty(self.nbytes, np.uint8)
        self.M._lib.ma_memcpy(raw.ctypes.data_as(ct.c_void_p), ct.c_void_p(self.ptr), self.nbytes, 2)
        return raw.view(self.dtype).reshape(self.shape[0], self.pitch // self.dtype.itemsize)[:, :self.shape[1]]

    def free(self):
        self.M._lib.ma_devFree(ct.c_void_p(self.ptr))


@pytest.mark.parametrize("autotune", [False, True])
def test_batch_matches_individual_evaluation(M, autotune):
    rng = np.random.default_rng(0)
    weights = [0.1, 0.2, 0.3, 0.15, 0.15, 0.1]
    b = M.Batch()
    cases = []
    for i in range(9):
        h, w = int(rng.integers(40, 400)), int(rng.integers(40, 400))
        dem_np = synth.fbm_dem(h, w, seed=100 + i)
        layers_np = [synth.uniform_f32(h, w, seed=200 + 10 * i + j) for j in range(6)]
        dem = M.from_numpy(dem_np, bs=[w, h])
        layers = [M.from_numpy(l, bs=[w, h]) for l in layers_np]
        hs, ov = W.hillshade(dem), W.wsum(layers, weights)
        o1, o2 = DevBuf(M, (h, w)), DevBuf(M, (h, w))
        b.add([hs, ov], [(o1.ptr, o1.pitch), (o2.ptr, o2.pitch)])
        cases.append((hs, ov, o1, o2))
    b.prepare(autotune=autotune)
    b.run()
    info = b.info()
    assert info["instances"] == 9 and len(info["kinds"]) == 2 and info["phases"] == 1
    for hs, ov, o1, o2 in cases:
        assert np.array_equal(o1.numpy(), M.to_numpy(hs))
        assert np.array_equal(o2.numpy(), M.to_numpy(ov))
    # replaying the captured graph gives the same results
    b.run()
    for hs, ov, o1, o2 in cases:
        assert np.array_equal(o1.numpy(), M.to_numpy(hs))
        o1.free()
        o2.free()


def test_batch_with_dependent_groups(M):
    """A program whose second focal group reads the first one's output runs as
    two dependency levels (two persistent launches in one graph)."""
    b = M.Batch()
    outs = []
    for i in range(4):
        a_np = synth.uniform_f32(100 + 30 * i, 90 + 20 * i, seed=i)
        a = M.from_numpy(a_np, bs=[64, 64])
        blur = M.convolve(M.convolve(a, [[1, 2, 1]] * 3) * 0.5, [[1, 1, 1]] * 3)
        o = DevBuf(M, a_np.shape)
        b.add([blur], [(o.ptr, o.pitch)])
        outs.append((blur, o))
    b.run()
    assert b.info()["phases"] == 2
    for r, o in outs:
        assert np.array_equal(o.numpy(), M.to_numpy(r))
        o.free()


def test_mix_rasters_against_oracle(fresh):
    """Rasters of the 512-raster mix's kind at its large end, checked against the
    oracle (not only against the engine itself): raster-edge mirror border,
    sides of 1500 and more, sizes that are multiples of neither 256 nor 64,
    aspect ratios near 0.5 and near 2, 256 x 256 blocks; hillshade within the
    hillshade tolerance, the 6-layer overlay bit-exact."""
    from oracle import oracle as O
    M = fresh
    M.set_border(M.BORDER_RASTER_MIRROR)
    weights = [0.1, 0.2, 0.3, 0.15, 0.15, 0.1]
    shapes = [(1537, 3070), (3001, 1501), (1999, 1999), (1500, 1700), (2047, 1503), (1601, 2900),
              (1777, 1555), (2900, 1450)]   # (width, height)
    b = M.Batch()
    cases = []
    for i, (w, h) in enumerate(shapes):
        dem_np = synth.fbm_dem(h, w, seed=300 + i)
        layers_np = [synth.uniform_f32(h, w, seed=400 + 10 * i + j) for j in range(6)]
        dem = M.from_numpy(dem_np, bs=[256, 256])
        layers = [M.from_numpy(l, bs=[256, 256]) for l in layers_np]
        hs, ov = W.hillshade(dem), W.wsum(layers, weights)
        o1, o2 = DevBuf(M, (h, w)), DevBuf(M, (h, w))
        b.add([hs, ov], [(o1.ptr, o1.pitch), (o2.ptr, o2.pitch)])
        cases.append((dem_np, layers_np, o1, o2))
    b.prepare(autotune=True)
    b.run()
    only_total = 0
    for dem_np, layers_np, o1, o2 in cases:
        got = o1.numpy()
        ref32 = O.hillshade_f32(dem_np, (256, 256), 1)
        ok, d, only = O.hill_tolerance(got, ref32, O.hillshade_bound(dem_np, (256, 256), 1))
        assert ok.all(), (dem_np.shape, int((~ok).sum()), float(d.max()))
        only_total += int(only.sum())
        ref_ov = O.wsum_f32(layers_np, np.array(weights, np.float32))
        assert np.array_equal(o2.numpy().view(np.uint32), ref_ov.view(np.uint32))
        o1.free()
        o2.free()
    assert only_total < 0.02 * sum(w * h for w, h in shapes)
