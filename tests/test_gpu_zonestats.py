"""Per-zone statistics (count / min / max / sum / mean of a float32 raster over
an int32 zone raster) against the oracle.

count, min and max must be bit-exact. The float32 sum is accumulated in a
different order than the oracle's row-major float32 loop (lane, warp, CTA and
grid levels with atomics), so it is compared with the float64 sum: the bound
used is |gpu - sum64| <= SUM_RTOL * sum(|x|) per zone, SUM_RTOL = 1e-4 (a
float32 sum of n terms in any order is within (n-1) * 2^-24 * sum|x| of the
exact sum; the longest sequential chain here is a few thousand additions, and
in practice the error is ~1e-6 relative). mean = sum / count in float32 gets
the same bound plus one rounding.
"""
import numpy as np
import pytest

from map_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-4


def _check(res, value, zone, nzones):
    ref = O.zone_stats(value, zone, nzones)
    np.testing.assert_array_equal(res["count"], ref["count"])
    np.testing.assert_array_equal(res["min"].view(np.uint32), ref["min"].view(np.uint32))
    np.testing.assert_array_equal(res["max"].view(np.uint32), ref["max"].view(np.uint32))
    absum = O.zone_stats(np.abs(value), zone, nzones)["sum64"]
    err = np.abs(res["sum"].astype(np.float64) - ref["sum64"])
    assert np.all(err <= SUM_RTOL * absum + 1e-30), float(np.max(err / np.maximum(absum, 1e-30)))
    cnt = ref["count"].astype(np.float64)
    full = cnt > 0
    mean64 = np.where(full, ref["sum64"] / np.maximum(cnt, 1), np.nan)
    merr = np.abs(res["mean"][full].astype(np.float64) - mean64[full])
    assert np.all(merr <= SUM_RTOL * absum[full] / cnt[full] + 1e-30)
    assert np.all(np.isnan(res["mean"][~full]))
    assert np.all(res["sum"][~full] == 0)
    return float(np.max(err / np.maximum(absum, 1e-30)))


def test_voronoi_lognormal(M):
    h, w = 1536, 2048
    value = synth.lognormal_f32(h, w, seed=3)
    zone = synth.voronoi_s32(h, w, 1024, seed=4)
    res = M.zonal_stats(value, zone, 1024)
    rel = _check(res, value, zone, 1024)
    assert int(res["count"].sum()) == h * w
    print("max relative sum error %.3g" % rel)


@pytest.mark.parametrize("w,h", [(1, 1), (3, 5), (1001, 37), (130, 129), (4096, 3)])
def test_ragged_sizes(M, w, h):
    rng = np.random.default_rng(w * 7 + h)
    value = rng.standard_normal((h, w)).astype(np.float32)
    zone = rng.integers(0, 17, size=(h, w)).astype(np.int32)
    _check(M.zonal_stats(value, zone, 17), value, zone, 17)


def test_skipped_cells_and_signed_zeros(M):
    rng = np.random.default_rng(11)
    h, w = 257, 515
    value = rng.standard_normal((h, w)).astype(np.float32)
    value[rng.random((h, w)) < 0.05] = np.nan
    value[rng.random((h, w)) < 0.05] = -0.0
    value[rng.random((h, w)) < 0.05] = 0.0
    value[rng.random((h, w)) < 0.01] = np.inf
    value[rng.random((h, w)) < 0.01] = -np.inf
    zone = rng.integers(-3, 40, size=(h, w)).astype(np.int32)
    zone[0, :50] = 2 ** 31 - 1
    zone[1, :50] = -2 ** 31
    value[2, :] = np.nan   # a row of skipped cells
    res = M.zonal_stats(value, zone, 37)
    ref = O.zone_stats(value, zone, 37)
    np.testing.assert_array_equal(res["count"], ref["count"])
    np.testing.assert_array_equal(res["min"].view(np.uint32), ref["min"].view(np.uint32))
    np.testing.assert_array_equal(res["max"].view(np.uint32), ref["max"].view(np.uint32))
    # infinities make the sums infinite or NaN; those must agree in kind
    fin = np.isfinite(ref["sum64"])
    np.testing.assert_array_equal(np.isfinite(res["sum"]), fin)


def test_only_signed_zeros(M):
    value = np.array([[0.0, -0.0, 0.0, -0.0], [0.0, 0.0, -0.0, -0.0]], np.float32)
    zone = np.array([[0, 0, 1, 1], [2, 2, 3, 3]], np.int32)
    res = M.zonal_stats(value, zone, 4)
    assert list(np.signbit(res["min"])) == [True, True, False, True]
    assert list(np.signbit(res["max"])) == [False, False, False, True]


def test_empty_zones_and_empty_raster(M):
    value = np.ones((4, 8), np.float32)
    zone = np.zeros((4, 8), np.int32)
    res = M.zonal_stats(value, zone, 5)
    assert list(res["count"]) == [32, 0, 0, 0, 0]
    assert res["sum"][0] == 32.0 and res["mean"][0] == 1.0
    assert np.all(np.isposinf(res["min"][1:])) and np.all(np.isneginf(res["max"][1:]))
    assert np.all(np.isnan(res["mean"][1:])) and np.all(res["sum"][1:] == 0)
    res = M.zonal_stats(np.zeros((0, 8), np.float32), np.zeros((0, 8), np.int32), 3)
    assert list(res["count"]) == [0, 0, 0] and np.all(np.isposinf(res["min"]))


def test_many_zones_use_global_bins(M):
    # more zones than fit in shared memory: the kernel accumulates straight into global bins
    h, w = 700, 900
    value = synth.lognormal_f32(h, w, seed=5)
    zone = synth.voronoi_s32(h, w, 20000, seed=6)
    _check(M.zonal_stats(value, zone, 20000), value, zone, 20000)


def test_single_zone_whole_raster(M):
    value = synth.lognormal_f32(1024, 1024, seed=8)
    zone = np.zeros((1024, 1024), np.int32)
    res = M.zonal_stats(value, zone, 1)
    _check(res, value, zone, 1)


def test_pitched_device_buffers(M):
    import torch
    h, w = 333, 1022            # rows of 4088 bytes: padded to a 16-byte pitch below
    rng = np.random.default_rng(21)
    value = rng.random((h, w), dtype=np.float32)
    zone = rng.integers(0, 9, size=(h, w)).astype(np.int32)
    pw = 1024
    dv = torch.zeros((h, pw), dtype=torch.float32, device="cuda")
    dz = torch.full((h, pw), 7, dtype=torch.int32, device="cuda")   # padding holds a valid zone id
    dv[:, :w] = torch.from_numpy(value).cuda()
    dz[:, :w] = torch.from_numpy(zone).cuda()
    out = torch.zeros(9 * 6, dtype=torch.float32, device="cuda")
    cnt = torch.zeros(9, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    M.zonal_stats_device(dv.data_ptr(), pw * 4, dz.data_ptr(), pw * 4, w, h, 9, cnt.data_ptr(), out.data_ptr(),
                         out.data_ptr() + 36, out.data_ptr() + 72, out.data_ptr() + 108,
                         stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    res = {"count": cnt.cpu().numpy().astype(np.uint64), "min": o[0:9], "max": o[9:18], "sum": o[18:27],
           "mean": o[27:36]}
    _check(res, value, zone, 9)


def test_raster_inputs(M):
    h, w = 300, 400
    value = synth.lognormal_f32(h, w, seed=9)
    zone = synth.voronoi_s32(h, w, 50, seed=10)
    v = M.from_numpy(value, bs=[128, 128]) * 2
    z = M.from_numpy(zone, bs=[128, 128])
    res = M.zonal_stats(v, z, 50)
    _check(res, value * np.float32(2), zone, 50)


def test_argument_errors(M):
    v = np.zeros((4, 4), np.float32)
    z = np.zeros((4, 4), np.int32)
    with pytest.raises(M.MapError, match="nzones"):
        M.zonal_stats(v, z, 0)
    with pytest.raises(M.MapError, match="pitch"):
        M.zonal_stats_device(16, 8, 16, 16, 4, 4, 1, 0, 0, 0, 0, 0)
    with pytest.raises(M.MapError, match="differ"):
        M.zonal_stats(v, np.zeros((4, 5), np.int32), 1)
