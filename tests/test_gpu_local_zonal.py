"""GPU parity of the local and zonal skeletons: element-wise operators
(bit-exact against NumPy restatements of the C semantics), the weighted
overlay, global zonal reductions (min/max exact, sums against FP64), the
stats.py program, .bin file I/O and device-resident inputs/outputs."""
import os

import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_elementwise_integer_ops_bit_exact(M):
    rng = np.random.default_rng(1)
    a_np = rng.integers(-1000, 1000, size=(70, 90)).astype(np.int32)
    b_np = rng.integers(1, 50, size=(70, 90)).astype(np.int32)
    a, b = M.from_numpy(a_np), M.from_numpy(b_np)
    cases = {
        "add": (a + b, a_np + b_np), "sub": (a - b, a_np - b_np), "mul": (a * b, a_np * b_np),
        "div": (a / b, (np.trunc(a_np / b_np)).astype(np.int32)), "mod": (a % b, np.fmod(a_np, b_np)),
        "lt": (a < b, (a_np < b_np).astype(np.uint8)), "max": (M.max(a, b), np.maximum(a_np, b_np)),
        "con": (M.con(a > 0, a, b), np.where(a_np > 0, a_np, b_np)), "neg": (-a, -a_np),
        "abs": (M.abs(a), np.abs(a_np)),
    }
    for name, (r, ref) in cases.items():
        got = M.to_numpy(r)
        assert got.dtype == ref.dtype, name
        assert np.array_equal(got, ref), name


def test_elementwise_float_ops_bit_exact(M):
    rng = np.random.default_rng(2)
    a_np = rng.standard_normal((65, 129)).astype(np.float32)
    b_np = (rng.random((65, 129)) + 0.5).astype(np.float32)
    a, b = M.from_numpy(a_np), M.from_numpy(b_np)
    f32 = np.float32
    cases = {
        "expr": ((a * 2.5 + b) / (b - 0.25), ((a_np * f32(2.5) + b_np) / (b_np - f32(0.25)))),
        "sqrt": (M.sqrt(b), np.sqrt(b_np)),
        "cast": (M.astype(a * 100.0, M.S32), (a_np * f32(100.0)).astype(np.int32)),
        "u8mul": ((a > 0) * b, (a_np > 0).astype(np.uint8) * b_np),
        "floor": (M.floor(a), np.floor(a_np)),
        "minmax": (M.min(M.max(a, -0.5), 0.5), np.minimum(np.maximum(a_np, f32(-0.5)), f32(0.5))),
    }
    for name, (r, ref) in cases.items():
        got = M.to_numpy(r)
        assert np.array_equal(got, ref.astype(got.dtype)), name


def test_transcendentals_within_ulps(M):
    rng = np.random.default_rng(3)
    a_np = (rng.random((50, 60)) * 6 - 3).astype(np.float32)
    a = M.from_numpy(a_np)
    for fn, ref in [(M.sin, np.sin), (M.cos, np.cos), (M.atan, np.arctan), (M.exp, np.exp), (M.tanh, np.tanh)]:
        got = M.to_numpy(fn(a)).astype(np.float64)
        want = ref(a_np.astype(np.float64))
        ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
        assert (np.abs(got - want) <= 4 * ulp + 1e-30).all(), fn


def test_wsum_bit_exact(M):
    layers_np = [synth.uniform_f32(257, 321, seed=40 + i) for i in range(6)]
    w = [0.1, 0.2, 0.3, 0.15, 0.15, 0.1]
    layers = [M.from_numpy(l, bs=[128, 128]) for l in layers_np]
    got = M.to_numpy(W.wsum(layers, w))
    ref = O.wsum_f32(layers_np, np.array(w, np.float32))
    assert np.array_equal(got, ref)
    assert M.last_launch_count() == 1


@pytest.mark.parametrize("mode", [0, 1])
def test_zonal_reductions(fresh, mode):
    M = fresh
    M.set_exec_mode(mode)
    v_np = synth.lognormal_f32(777, 1025, seed=4)
    v = M.from_numpy(v_np, bs=[256, 256])
    zs, zx, zn = M.zsum(v), M.zmax(v), M.zmin(v)
    M.eval(zs, zx, zn)
    assert M.value(zx) == v_np.max()
    assert M.value(zn) == v_np.min()
    exact = v_np.astype(np.float64).sum()
    assert abs(M.value(zs) - exact) <= 2e-6 * exact
    i_np = np.random.default_rng(5).integers(0, 1 << 20, size=(300, 200)).astype(np.int64)
    i = M.from_numpy(i_np)
    s = M.zsum(i)
    M.eval(s)
    assert M.value(s) == int(i_np.sum())


def test_stats_program(M):
    dem_np = synth.fbm_dem(512, 512, seed=8, lo=1.0, hi=3000.0)
    dem = M.from_numpy(dem_np, bs=[256, 256])
    s = W.stats(dem)
    M.eval(*s.values())
    d = dem_np.astype(np.float64)
    N = d.size
    mean = np.float32(np.float32(d.sum()) / np.float32(N))
    exp = dict(maxv=d.max(), minv=d.min(), mean=d.mean(), harm=N / (1.0 / d).sum(), quam=np.sqrt((d ** 2).mean()),
               cubm=np.cbrt((d ** 3).mean()), std=np.sqrt(((d - mean) ** 2).mean()))
    for k, want in exp.items():
        got = M.value(s[k])
        assert abs(got - want) <= 1e-5 * abs(want) + 1e-6, (k, got, want)
    assert M.value(s["geom"]) == float("inf")     # the F32 product of the raster overflows, as in the reference


def test_bin_file_roundtrip(M, tmp_path):
    a_np = synth.fbm_dem(300, 260, seed=2)
    src = M.from_numpy(a_np, bs=[128, 128])
    p1 = str(tmp_path / "a.bin")
    assert M.write(src * 2.0, p1) == 0
    assert os.path.getsize(p1) == 4096 + 3 * 3 * 128 * 128 * 4     # header page + padded blocks
    r = M.read(p1)
    assert r.datasize() == [260, 300] and r.blocksize() == [128, 128] and r.datatype() == M.F32
    back = M.to_numpy(r)
    assert np.array_equal(back, a_np * np.float32(2.0))


def test_device_resident_input_and_output(M):
    import ctypes as ct
    a_np = synth.uniform_f32(128, 192, seed=3)
    nbytes = a_np.nbytes
    d_in = M._lib.ma_devAlloc(nbytes)
    d_out = M._lib.ma_devAlloc(nbytes)
    M._lib.ma_memcpy(ct.c_void_p(d_in), a_np.ctypes.data_as(ct.c_void_p), nbytes, 1)
    r = M.from_device(d_in, 192 * 4, [192, 128], M.F32)
    M.to_device(r * 3.0 + 1.0, d_out, 192 * 4)
    out = np.empty_like(a_np)
    M._lib.ma_memcpy(out.ctypes.data_as(ct.c_void_p), ct.c_void_p(d_out), nbytes, 2)
    assert np.array_equal(out, a_np * np.float32(3.0) + np.float32(1.0))
    M._lib.ma_devFree(ct.c_void_p(d_in))
    M._lib.ma_devFree(ct.c_void_p(d_out))


def test_sincos_pairing_is_bit_identical(M):
    """sin(x) and cos(x) of one argument compile to one sincosf call; its
    results equal separate sinf / cosf calls on every input."""
    rng = np.random.default_rng(7)
    x_np = np.concatenate([rng.uniform(-10, 10, 200000), rng.uniform(-1e4, 1e4, 50000),
                           np.linspace(0, 1.5707964, 50000)]).astype(np.float32).reshape(300, 1000)
    x = M.from_numpy(x_np)
    pair_s = M.to_numpy(M.sin(x) + 0.0 * M.cos(x) + M.cos(x) * 0.0)
    only_s = M.to_numpy(M.sin(x))
    only_c = M.to_numpy(M.cos(x))
    both = M.to_numpy(M.sin(x) * 1.0 + M.cos(x) * 0.0)   # same shape of program, paired
    assert np.array_equal(M.to_numpy(M.sin(x) * 1.0), only_s)
    s_pair = M.from_numpy(x_np)
    a = M.sin(s_pair)
    b = M.cos(s_pair)
    src = M.generated_source(a + b)
    assert "sincosf(" in src
    ab = M.to_numpy(a + b)
    assert np.array_equal(ab, only_s + only_c)


@pytest.mark.parametrize("mode", [0, 1])
def test_prediction_fills_fixed_groups_without_launches(fresh, mode):
    """A program of constants only (element-wise and focal operators of a
    constant raster, block-mirror border) is written by fills, with no kernel
    launch, in fused and plain mode; switching prediction off launches kernels
    and gives the same cells."""
    M = fresh
    M.set_exec_mode(mode)
    c = M.zeros((300, 200), M.F32, M.ROW + M.BLK, [64, 64]) + 2.5
    prog = M.convolve(c * 3.0 - 1.0, [[1, 2, 1], [0, 1, 0], [1, 2, 1]]) + (c > 1.0)
    got = M.to_numpy(prog)
    assert M.last_launch_count() == 0 and M.last_predicted_count() >= 1
    want = np.float32(0)
    for w in (1, 2, 1, 0, 1, 0, 1, 2, 1):
        want = np.float32(want + np.float32(6.5) * np.float32(w))
    assert np.all(got == np.float32(want + np.float32(1)))
    M.set_prediction(False)
    again = M.to_numpy(prog)
    assert M.last_launch_count() >= 1
    assert np.array_equal(got, again)
    # a cell-dependent node keeps the launch
    M.set_prediction(True)
    idx = M.to_numpy(c + M.index(c, M.D1))
    assert M.last_launch_count() >= 1
    assert np.array_equal(idx, np.float32(2.5) + np.arange(300, dtype=np.float32)[None, :] + np.zeros((200, 1), np.float32))
