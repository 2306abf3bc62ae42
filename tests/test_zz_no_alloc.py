"""ma_zoneStatsNoAlloc (per-zone statistics whose working bins are a fixed
device array instead of a pool allocation) against ma_zoneStats, both called
through the C ABI on the same device buffers.

count, min and max must be identical; sum and mean are float32 sums whose
rounding depends on the order of the device's atomic additions, so they must
agree within |a - b| <= SUM_RTOL * sum(|x|) per zone, the bound the zone
statistics tests hold each entry point to against the float64 oracle.

This file is collected last and makes no assumption about what ran before it,
so it passes alone in a fresh process as well as after the other tests.
"""
import ctypes as ct
import os

import numpy as np
import pytest

from map_b200 import synth

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-4
STATIC_ZONES = 16384
LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "map_b200", "libmap_b200.so")


@pytest.fixture(scope="module")
def lib(_built):
    L = ct.CDLL(LIB)
    args = [ct.c_void_p, ct.c_longlong, ct.c_void_p, ct.c_longlong, ct.c_int, ct.c_int, ct.c_int,
            ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    for name in ("ma_zoneStats", "ma_zoneStatsNoAlloc"):
        getattr(L, name).argtypes = args
        getattr(L, name).restype = ct.c_int
    L.ma_lastError.restype = ct.c_char_p
    return L


def _call(torch, L, name, val, zone, nzones):
    h, w = val.shape
    out = torch.full((4 * nzones,), 7.0, dtype=torch.float32, device="cuda")      # non-zero: all must be written
    cnt = torch.full((nzones,), 12345, dtype=torch.int64, device="cuda")
    o = out.data_ptr()
    st = torch.cuda.current_stream().cuda_stream
    rc = getattr(L, name)(val.data_ptr(), w * 4, zone.data_ptr(), w * 4, w, h, nzones, cnt.data_ptr(), o,
                          o + 4 * nzones, o + 8 * nzones, o + 12 * nzones, st)
    assert rc == 0, L.ma_lastError()
    torch.cuda.synchronize()
    a = out.cpu().numpy()
    return {"count": cnt.cpu().numpy(), "min": a[:nzones], "max": a[nzones:2 * nzones],
            "sum": a[2 * nzones:3 * nzones], "mean": a[3 * nzones:]}


def _same(a, b, absum):
    np.testing.assert_array_equal(a["count"], b["count"])
    np.testing.assert_array_equal(a["min"].view(np.uint32), b["min"].view(np.uint32))
    np.testing.assert_array_equal(a["max"].view(np.uint32), b["max"].view(np.uint32))
    for k in ("sum", "mean"):
        x, y = a[k].astype(np.float64), b[k].astype(np.float64)
        nan = np.isnan(x)
        np.testing.assert_array_equal(nan, np.isnan(y))
        bound = SUM_RTOL * absum if k == "sum" else SUM_RTOL * absum / np.maximum(a["count"], 1)
        assert np.all(np.abs(x[~nan] - y[~nan]) <= bound[~nan] + 1e-30), k


def test_no_alloc_matches_allocating_entry_on_two_calls_in_a_row(lib):
    import torch
    cases = [(1024, 1536, 1024, 41), (700, 900, 300, 42)]   # the second call uses fewer zones than the first
    for h, w, nz, seed in cases:
        v_np = synth.lognormal_f32(h, w, seed=seed)
        z_np = synth.voronoi_s32(h, w, nz, seed=seed + 100)
        z_np[::7, ::5] = -1                                  # skipped cells
        val = torch.from_numpy(v_np).cuda()
        zone = torch.from_numpy(z_np).cuda()
        absum = np.bincount(z_np[z_np >= 0].ravel(), weights=np.abs(v_np[z_np >= 0]).ravel(), minlength=nz)
        ref = _call(torch, lib, "ma_zoneStats", val, zone, nz)
        got = _call(torch, lib, "ma_zoneStatsNoAlloc", val, zone, nz)
        _same(got, ref, absum)
        assert int(got["count"].sum()) == int((z_np >= 0).sum())


def test_no_alloc_allocates_no_device_memory_after_setup(lib):
    import torch
    h, w, nz = 512, 640, 200
    val = torch.from_numpy(synth.lognormal_f32(h, w, seed=5)).cuda()
    zone = torch.from_numpy(synth.voronoi_s32(h, w, nz, seed=6)).cuda()
    _call(torch, lib, "ma_zoneStatsNoAlloc", val, zone, nz)          # set-up (if not done already)
    out = torch.zeros(4 * nz, dtype=torch.float32, device="cuda")
    cnt = torch.zeros(nz, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    o = out.data_ptr()
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        rc = lib.ma_zoneStatsNoAlloc(val.data_ptr(), w * 4, zone.data_ptr(), w * 4, w, h, nz, cnt.data_ptr(), o,
                                     o + 4 * nz, o + 8 * nz, o + 12 * nz, st)
        assert rc == 0, lib.ma_lastError()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert int(cnt.sum().item()) == h * w


def test_no_alloc_rejects_more_zones_than_its_scratch(lib):
    import torch
    val = torch.ones((4, 4), dtype=torch.float32, device="cuda")
    zone = torch.zeros((4, 4), dtype=torch.int32, device="cuda")
    nz = STATIC_ZONES + 1
    out = torch.zeros(nz, dtype=torch.float32, device="cuda")
    rc = lib.ma_zoneStatsNoAlloc(val.data_ptr(), 16, zone.data_ptr(), 16, 4, 4, nz, None, out.data_ptr(), None,
                                 None, None, torch.cuda.current_stream().cuda_stream)
    assert rc != 0
    assert b"16384" in lib.ma_lastError()
    # the largest accepted count works
    res = _call(torch, lib, "ma_zoneStatsNoAlloc", val, zone, STATIC_ZONES)
    assert res["count"][0] == 16 and res["count"][1:].sum() == 0 and res["sum"][0] == 16.0
