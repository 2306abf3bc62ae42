"""Serving with continuous batching: every program's result over a window equals
the same program evaluated alone on the cropped window, a request's result is
identical alone and inside a mixed batch, the HBM budget bounds the memory in
use, and an open-loop Poisson load reports latency percentiles."""
import ctypes as ct

import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W

pytestmark = pytest.mark.gpu

WD, HD = 1500, 1300


@pytest.fixture(scope="module")
def served(M):
    dem_np = synth.fbm_dem(HD, WD, seed=77)
    pitch = WD * 4
    d = M._lib.ma_devAlloc(pitch * HD)
    M._lib.ma_memcpy(ct.c_void_p(d), dem_np.ctypes.data_as(ct.c_void_p), pitch * HD, 1)
    srv = M.Server(d, pitch, WD, HD, budget_bytes=256 << 20, max_batch=64)
    yield M, srv, dem_np
    srv.close()
    M._lib.ma_devFree(ct.c_void_p(d))


def window_expected(M, dem_np, kind, x0, y0, w, h, obs=(0, 0), obs_h=10.0, radius=0):
    win = M.from_numpy(np.ascontiguousarray(dem_np[y0:y0 + h, x0:x0 + w]), bs=[w, h])
    if kind == M.Server.HILLSHADE:
        return M.to_numpy(W.hillshade(win))
    if kind == M.Server.SLOPE:
        return M.to_numpy(W.slope(win))
    if kind == M.Server.VIEWSHED:
        shift = win - obs_h
        dist = W.distance(win, obs)
        maxr = M.rmax(shift / dist, list(obs), radius=radius)
        return M.to_numpy((maxr * dist + obs_h) - win)
    dirs = M.flow_direction(win)
    return M.to_numpy(M.flow_accumulation(M.ones_like(win, M.S32), dirs))


def same(a, b):
    return np.array_equal(np.isnan(a), np.isnan(b)) if a.dtype.kind == "f" and np.isnan(a).any() else True


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_each_program_matches_windowed_evaluation(served, kind):
    M, srv, dem_np = served
    x0, y0, w, h, obs = 123, 77, 300, 260, (131, 97)
    rid = srv.submit(kind, x0, y0, w, h, obs=obs, obs_h=10.0, radius=80 if kind == 2 else 0)
    got = srv.result(rid, (h, w), np.int32 if kind == 3 else np.float32)
    want = window_expected(M, dem_np, kind, x0, y0, w, h, obs, 10.0, 80 if kind == 2 else 0)
    nan = np.isnan(want) if want.dtype.kind == "f" else np.zeros(want.shape, bool)
    assert np.array_equal(np.isnan(got) if got.dtype.kind == "f" else nan, nan)
    assert np.array_equal(got[~nan], want[~nan])


def test_result_identical_alone_and_in_a_mix(served):
    M, srv, dem_np = served
    target = (M.Server.HILLSHADE, 500, 400, 512, 512)
    rid = srv.submit(*target)
    alone = srv.result(rid, (512, 512), np.float32)
    rng = np.random.default_rng(3)
    ids = []
    for i in range(40):
        kind = int(rng.integers(0, 4))
        w = int(rng.choice([64, 128, 256]))
        x0, y0 = int(rng.integers(0, WD - w)), int(rng.integers(0, HD - w))
        ids.append(srv.submit(kind, x0, y0, w, w, obs=(w // 2, w // 3), radius=50))
        if i == 20:
            mixed_id = srv.submit(*target)
    mixed = srv.result(mixed_id, (512, 512), np.float32)
    for i in ids:
        srv.wait(i)
        srv.release(i)
    assert np.array_equal(alone, mixed)
    assert srv.stats()["max_batch"] > 1


def test_budget_admission_bounds_memory(M):
    dem_np = synth.fbm_dem(600, 600, seed=5)
    d = M._lib.ma_devAlloc(600 * 600 * 4)
    M._lib.ma_memcpy(ct.c_void_p(d), dem_np.ctypes.data_as(ct.c_void_p), 600 * 600 * 4, 1)
    budget = 3 * 2 * 256 * 256 * 4
    srv = M.Server(d, 600 * 4, 600, 600, budget_bytes=budget, max_batch=64)
    ids = [srv.submit(M.Server.HILLSHADE, 10 * i, 5 * i, 256, 256) for i in range(12)]
    outs = [srv.result(i, (256, 256), np.float32) for i in ids]
    st = srv.stats()
    assert st["completed"] == 12 and st["peak_bytes"] <= budget
    assert np.array_equal(outs[3], window_expected(M, dem_np, 0, 30, 15, 256, 256))
    srv.close()
    M._lib.ma_devFree(ct.c_void_p(d))


def test_open_loop_load_reports_percentiles(served):
    M, srv, dem_np = served
    r = srv.load(rate=300, seconds=1.0, seed=1, radius=167)
    assert r["completed"] == r["requests"] > 100
    assert 0 < r["p50_ms"] <= r["p99_ms"]


def test_observer_height_is_an_argument(served):
    # any observer height reuses the compiled viewshed kernel and matches the engine
    M, srv, dem_np = served
    kinds0 = srv.stats()["kinds"]
    x0, y0, w, h, obs = 40, 60, 200, 180, (70, 90)
    for oh in (25.0, 3.5):
        rid = srv.submit(M.Server.VIEWSHED, x0, y0, w, h, obs=obs, obs_h=oh, radius=60)
        got = srv.result(rid, (h, w), np.float32)
        want = window_expected(M, dem_np, M.Server.VIEWSHED, x0, y0, w, h, obs, oh, 60)
        nan = np.isnan(want)
        assert np.array_equal(np.isnan(got), nan)
        assert np.array_equal(got[~nan], want[~nan])
    assert srv.stats()["kinds"] == kinds0


def test_window_sizes_beyond_the_template_cache_still_work(served):
    # odd window sizes each build a template; results stay exact whether cached or not
    M, srv, dem_np = served
    for k in range(5):
        w, h = 97 + 13 * k, 61 + 7 * k
        rid = srv.submit(M.Server.SLOPE, 11 * k, 5 * k, w, h)
        got = srv.result(rid, (h, w), np.float32)
        want = window_expected(M, dem_np, M.Server.SLOPE, 11 * k, 5 * k, w, h)
        assert np.array_equal(got, want)


def test_closed_loop_load_batches_requests(served):
    """With many requests kept in flight the dispatcher admits several per batch
    (continuous batching), every request completes, and the report counts the
    batches of this run only."""
    M, srv, _ = served
    res = srv.load_closed(32, 1.0, seed=5)
    assert res["mode"] == "closed" and res["requests"] >= 32
    assert res["completed"] == res["requests"]
    assert res["batches"] >= 1 and res["mean_batch"] > 1.0
    assert res["p99_ms"] >= res["p50_ms"] > 0
