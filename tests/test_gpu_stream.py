"""Streamed (row-band) evaluation of host-to-host programs: every result must be
bit-identical to whole-raster evaluation of the same program, whatever the band
height, border rule, halo depth, data type or mix of host and device inputs."""
import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture()
def S(fresh):
    yield fresh
    fresh.set_stream_rows(0)


def both(M, build, rows):
    """(streamed result, band count, whole-raster result) of the program `build()`."""
    M.set_stream_rows(rows)
    a = M.to_numpy(build())
    bands = M.last_band_count()
    M.set_stream_rows(-1)
    b = M.to_numpy(build())
    assert M.last_band_count() == 0
    return a, bands, b


def same(a, b):
    assert a.dtype == b.dtype and a.shape == b.shape
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("rows", [32, 64, 100, 257])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_hillshade_bands_match_whole_raster(S, rows, border):
    M = S
    M.set_border(border)
    dem = synth.fbm_dem(1300, 1000, seed=12)
    a, bands, b = both(M, lambda: W.hillshade(M.from_numpy(dem, bs=[256, 256])), rows)
    assert bands == -(-1300 // rows)
    same(a, b)


def test_chained_focal_groups_and_wide_halo(S):
    M = S
    x = synth.uniform_f32(777, 523, seed=3)
    k3 = [[1, 2, 1], [2, 4, 2], [1, 2, 1]]
    k5 = [[1] * 5 for _ in range(5)]

    def prog():
        r = M.from_numpy(x, bs=[128, 128])
        c = M.convolve(M.convolve(r, k3), k3)            # two focal groups: margin 2
        return M.fmax(c, k5) - M.fmin(r, k5) * 0.5       # halo 2 on top
    a, bands, b = both(M, prog, 40)
    assert bands == -(-777 // 40)
    same(a, b)


def test_life_generations_bit_exact(S):
    M = S
    M.set_border(2)
    grid = synth.bernoulli_u8(600, 700, 0.3, seed=9)
    a, bands, b = both(M, lambda: W.life(M.from_numpy(grid, bs=[128, 128]), 5), 64)
    assert bands > 1
    same(a, b)


def test_local_overlay_with_index_nodes(S):
    M = S
    layers = [synth.uniform_f32(1000, 300, seed=20 + i) for i in range(3)]

    def prog():
        r = [M.from_numpy(l, bs=[256, 256]) for l in layers]
        return r[0] * 0.2 + r[1] * 0.3 + r[2] * 0.5 + M.index(r[0], M.D1) * 0.001 - M.index(r[0], M.D2) * 0.002
    a, bands, b = both(M, prog, 96)
    assert bands == -(-1000 // 96)
    same(a, b)


def test_device_and_host_inputs_mixed(S):
    import torch
    M = S
    h, w = 900, 640
    dem = synth.fbm_dem(h, w, seed=31)
    lay = synth.uniform_f32(h, w, seed=32)
    dt = torch.from_numpy(dem).cuda()
    torch.cuda.synchronize()

    def prog():
        d = M.from_device(dt.data_ptr(), w * 4, [w, h], M.F32, [256, 256])
        return W.hillshade(d) * M.from_numpy(lay, bs=[256, 256])
    a, bands, b = both(M, prog, 128)
    assert bands == -(-h // 128)
    same(a, b)


def test_automatic_bands_on_a_large_raster(S):
    M = S
    dem = synth.fbm_dem(4096, 4096, seed=5)
    M.set_stream_rows(0)
    a = M.to_numpy(W.hillshade(M.from_numpy(dem, bs=[256, 256])))
    assert M.last_band_count() >= 4
    M.set_stream_rows(-1)
    b = M.to_numpy(W.hillshade(M.from_numpy(dem, bs=[256, 256])))
    same(a, b)


def test_programs_that_do_not_stream(S):
    M = S
    x = synth.uniform_f32(300, 200, seed=1)
    M.set_stream_rows(16)
    r = M.from_numpy(x, bs=[64, 64])
    z = M.zsum(r)
    M.eval(z)
    assert np.isclose(M.value(z), np.float64(x.astype(np.float64).sum()), rtol=1e-5)
    assert M.last_band_count() == 0          # zonal groups are not streamed
    M.set_stream_rows(400)                   # band taller than the raster
    M.to_numpy(r * 2)
    assert M.last_band_count() == 0
