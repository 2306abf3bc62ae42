"""Float32 atan2 of the engine (map_common.cuh map_atan2f) against float64
atan2: at most 2 ulp from the correctly rounded value on random operands of
every magnitude (the bound the hillshade parity tolerance assumes for one
library function), and the IEEE 754 special cases exactly (signed zeros,
infinities, NaN)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _atan2(M, y, x):
    h, w = y.shape
    ry = M.from_numpy(y, bs=[w, h])
    rx = M.from_numpy(x, bs=[w, h])
    return M.to_numpy(M.atan2(ry, rx))


def _ulp_err(got, y, x):
    ref = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - ref) / ulp


def test_atan2_random_operands_within_2_ulp(M):
    rng = np.random.default_rng(5)
    n = 1024
    for trial in range(4):
        y = (rng.uniform(-1, 1, (n, n)) * np.exp2(rng.uniform(-60, 60, (n, n)))).astype(np.float32)
        if trial % 2:
            x = (y * rng.uniform(0.5, 2, (n, n)) * np.where(rng.random((n, n)) < 0.5, -1, 1)).astype(np.float32)
        else:
            x = (rng.uniform(-1, 1, (n, n)) * np.exp2(rng.uniform(-60, 60, (n, n)))).astype(np.float32)
        err = _ulp_err(_atan2(M, y, x), y, x)
        assert err.max() <= 2.0, err.max()


def test_atan2_subnormal_and_unit_operands(M):
    rng = np.random.default_rng(6)
    y = np.concatenate([rng.uniform(-1e-38, 1e-38, 4096), rng.uniform(-1, 1, 4096)]).astype(np.float32).reshape(64, 128)
    x = np.concatenate([rng.uniform(-1, 1, 4096), rng.uniform(-1e-38, 1e-38, 4096)]).astype(np.float32).reshape(64, 128)
    assert _ulp_err(_atan2(M, y, x), y, x).max() <= 2.0


def test_atan2_special_cases_exact(M):
    sp = np.array([0.0, -0.0, 1.0, -1.0, 2.5, -2.5, np.inf, -np.inf, np.nan, 1e-40, -1e-40, 3e38], np.float32)
    Y, X = np.meshgrid(sp, sp)
    got = _atan2(M, Y.astype(np.float32), X.astype(np.float32))
    ref = np.arctan2(Y, X).astype(np.float32)
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(got), nan)
    exact = np.isin(Y, [0.0, np.inf, -np.inf]) | np.isin(X, [0.0, np.inf, -np.inf])
    sel = exact & ~nan
    assert np.array_equal(got[sel], ref[sel])
    assert np.array_equal(np.signbit(got[sel]), np.signbit(ref[sel]))
    assert _ulp_err(got[~nan], Y[~nan], X[~nan]).max() <= 2.0
