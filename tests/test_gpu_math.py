"""Float32 atan2, sin and cos of the engine (map_common.cuh map_atan2f,
map_sinf, map_cosf, map_sincosf) against float64: at most 2 ulp from the
correctly rounded value on random operands of every magnitude (the bound the
hillshade parity tolerance assumes for one library function), in the scalar and
the packed-pair forms, and the IEEE 754 special cases exactly (signed zeros,
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


# ---- sine and cosine (map_common.cuh map_sinf / map_cosf / map_sincosf)

def _trig_inputs(seed):
    rng = np.random.default_rng(seed)
    parts = [rng.uniform(-b, b, 1 << 18) for b in (0.8, 4.0, 1024.0, 65536.0, 1e6, 1e30)]
    k = np.arange(1, 1 << 16)
    near = (k * (np.pi / 2)).astype(np.float32)        # the floats nearest to multiples of pi/2
    parts += [near, np.nextafter(near, np.float32(np.inf)), np.nextafter(near, np.float32(-np.inf)), -near]
    x = np.concatenate(parts).astype(np.float32)
    return x[: (x.size // 1024) * 1024].reshape(-1, 1024)


def _trig_err(got, x, fn):
    ref = fn(x.astype(np.float64))
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - ref) / ulp


def test_sin_cos_within_2_ulp(M):
    x = _trig_inputs(11)
    h, w = x.shape
    r = M.from_numpy(x, bs=[w, 256])
    assert _trig_err(M.to_numpy(M.sin(r)), x, np.sin).max() <= 2.0
    assert _trig_err(M.to_numpy(M.cos(r)), x, np.cos).max() <= 2.0
    # sin and cos of one argument in one group share one reduction (map_sincosf)
    s, c = M.to_numpy(M.sin(r) + M.cos(r) * 0), M.to_numpy(M.cos(r) + M.sin(r) * 0)
    assert _trig_err(s, x, np.sin).max() <= 2.0
    fin = np.isfinite(x)
    assert _trig_err(c[fin], x[fin], np.cos).max() <= 2.0


def test_sin_cos_special_values_exact(M):
    sp = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 1e-40, -3e-39, 1e-30, 3e38, -3e38],
                  np.float32).reshape(1, -1)
    r = M.from_numpy(sp, bs=[sp.shape[1], 1])
    for fn, ref in ((M.sin, np.sin), (M.cos, np.cos)):
        got = M.to_numpy(fn(r))
        want = ref(sp.astype(np.float64)).astype(np.float32)
        nan = np.isnan(want)
        assert np.array_equal(np.isnan(got), nan)
        small = np.abs(sp) < 1e-20                      # sin x = x and cos x = 1 exactly, zeros keep their sign
        assert np.array_equal(got[small], want[small])
        assert np.array_equal(np.signbit(got[small]), np.signbit(want[small]))
        assert _trig_err(got[~nan], sp[~nan], ref).max() <= 2.0


def test_paired_sin_cos_within_2_ulp(M):
    """The packed form inside a focal group (two rows per thread step)."""
    x = _trig_inputs(12)[:512]
    h, w = x.shape
    r = M.from_numpy(x, bs=[w, 256])
    centre = M.convolve(r, [[0, 0, 0], [0, 1, 0], [0, 0, 0]])     # equals x except that -0 becomes +0
    s, c = M.sin(centre), M.cos(centre)
    assert "focal_cell2" in M.generated_source(s) and "focal_cell2" in M.generated_source(c)
    assert _trig_err(M.to_numpy(s), x, np.sin).max() <= 2.0
    assert _trig_err(M.to_numpy(c), x, np.cos).max() <= 2.0
