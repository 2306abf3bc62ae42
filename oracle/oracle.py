"""Python bindings of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Used by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg
as the checker. Never imported by the product (map_b200/).

  liboracle.so    -- oracle/oracle.c, the C restatement of the reference semantics
  libref_util.so  -- the reference's own util/ operator tables (oracle/ref_util)

PARITY UNPINNED: the reference's execution path cannot run here and it ships no
golden vectors; see oracle/oracle.c.
"""
import ctypes as ct
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref = None
_lock = threading.Lock()


def lib():
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = os.path.join(HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle library missing: run `python oracle/build_oracle.py`")
        L = ct.CDLL(path)
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        I = ct.c_int
        L.orc_conv_f32.argtypes = [f32p, I, I, I, I, I, f32p, I, I, f32p]
        L.orc_hillshade_f32.argtypes = [f32p, I, I, I, I, I, ct.c_double, ct.c_double, f32p, ct.c_void_p, ct.c_void_p]
        L.orc_hillshade_f64.argtypes = [f32p, I, I, I, I, I, ct.c_double, ct.c_double, f64p]
        L.orc_hillshade_f32_rows.argtypes = [ct.c_void_p, I, I, I, I, I, ct.c_double, ct.c_double, I, I, ct.c_void_p]
        L.orc_hillshade_bound.argtypes = [f32p, I, I, I, I, I, ct.c_double, ct.c_double, f64p]
        L.orc_life.argtypes = [u8p, I, I, I, I, I, I, u8p]
        L.orc_life_rows.argtypes = [u8p, I, I, I, I, I, I, I, u8p]
        L.orc_rand_u8.argtypes = [ct.c_uint32, I, I, I, I, u8p]
        L.orc_d8.argtypes = [f32p, I, I, I, I, I, u8p]
        L.orc_flowacc_s32.argtypes = [i32p, u8p, I, I, i32p]
        L.orc_flowacc_s32.restype = ct.c_int
        L.orc_radial_f32.argtypes = [f32p, I, I, I, I, I, f32p]
        L.orc_wsum_f32.argtypes = [ct.POINTER(ct.c_void_p), f32p, I, ct.c_size_t, f32p]
        u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
        L.orc_zone_stats.argtypes = [f32p, i32p, ct.c_longlong, I, u64p, f32p, f32p, f32p, f64p]
        L.orc_focal_src.argtypes = [I, I, I, I, I, I, I, I, I, ct.POINTER(I), ct.POINTER(I)]
        L.orc_focal_src.restype = I
        _lib = L
    return _lib


_native = None


def lib_native():
    """The -O3 -march=native build of the same oracle, compiled on this host
    (oracle/build_oracle.py:build_oracle_native), for timing the CPU baseline."""
    global _native
    with _lock:
        if _native is None:
            from oracle import build_oracle
            L = ct.CDLL(build_oracle.build_oracle_native())
            f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
            I = ct.c_int
            L.orc_hillshade_f32_rows.argtypes = [ct.c_void_p, I, I, I, I, I, ct.c_double, ct.c_double, I, I, ct.c_void_p]
            L.orc_wsum_f32.argtypes = [ct.POINTER(ct.c_void_p), f32p, I, ct.c_size_t, ct.c_void_p]
            _native = L
    return _native


def hillshade_rows(L, dem, out, bs, border, y0, y1, zenith=45.0, azimuth=315.0):
    """Rows [y0, y1) of the FP32 hillshade of the whole `dem` into `out` (both
    C-contiguous float32 arrays of the raster's shape), with library L."""
    L.orc_hillshade_f32_rows(dem.ctypes.data, dem.shape[1], dem.shape[0], bs[0], bs[1], border, zenith, azimuth,
                             y0, y1, out.ctypes.data)


def ref_util():
    """The reference's own host operator tables, or None when not built here."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libref_util.so")
        if not os.path.exists(path):
            return None
        _ref = ct.CDLL(path)
        vp, I = ct.c_void_p, ct.c_int
        _ref.ref_promote.argtypes = [I, I]
        _ref.ref_promote.restype = I
        _ref.ref_binary.argtypes = [I, vp, I, vp, I, vp, ct.POINTER(I)]
        _ref.ref_unary.argtypes = [I, vp, I, vp, ct.POINTER(I)]
        _ref.ref_neutral.argtypes = [I, I, vp, ct.POINTER(I)]
        _ref.ref_reduce.argtypes = [I, vp, vp, I, vp, ct.POINTER(I)]
    return _ref


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def conv_f32(a, mask, bs, border=0):
    a = _c(a, np.float32)
    m = _c(mask, np.float32)
    out = np.empty_like(a)
    lib().orc_conv_f32(a, a.shape[1], a.shape[0], bs[0], bs[1], border, m, m.shape[1], m.shape[0], out)
    return out


def hillshade_f32(dem, bs, border=0, zenith=45.0, azimuth=315.0):
    dem = _c(dem, np.float32)
    out = np.empty_like(dem)
    lib().orc_hillshade_f32(dem, dem.shape[1], dem.shape[0], bs[0], bs[1], border, zenith, azimuth, out, None, None)
    return out


def hillshade_f64(dem, bs, border=0, zenith=45.0, azimuth=315.0):
    dem = _c(dem, np.float32)
    out = np.empty(dem.shape, np.float64)
    lib().orc_hillshade_f64(dem, dem.shape[1], dem.shape[0], bs[0], bs[1], border, zenith, azimuth, out)
    return out


def hillshade_bound(dem, bs, border=0, zenith=45.0, azimuth=315.0):
    """Per-cell first-order rounding-error scale of the FP32 hillshade chain
    (angle roundings and the two terms' own roundings; see oracle.c)."""
    dem = _c(dem, np.float32)
    out = np.empty(dem.shape, np.float64)
    lib().orc_hillshade_bound(dem, dem.shape[1], dem.shape[0], bs[0], bs[1], border, zenith, azimuth, out)
    return out


def hill_tolerance(gpu, ref32, bound):
    """The hillshade tolerance against the FP32 oracle: within 4 ulp or 1e-5
    relative of it, or, where its two terms cancel, within 4 times the chain's
    own first-order rounding-error scale at that cell (hillshade_bound).
    Returns (ok mask, |gpu - ref32|, mask of cells that pass only through the
    cancellation clause)."""
    d = np.abs(np.asarray(gpu, np.float64) - np.asarray(ref32, np.float64))
    strict = (d <= 4 * ulp_f32(ref32)) | (d <= 1e-5 * np.abs(np.asarray(ref32, np.float64)))
    cancel = d <= 4 * bound
    nan_same = np.isnan(np.asarray(gpu, np.float64)) & np.isnan(np.asarray(ref32, np.float64))
    ok = strict | cancel | nan_same
    return ok, d, ok & ~strict & ~nan_same


def life(state, bs, gens, border=0):
    s = _c(state, np.uint8)
    out = np.empty_like(s)
    lib().orc_life(s, s.shape[1], s.shape[0], bs[0], bs[1], border, gens, out)
    return out


def life_rows(state, out, bs, border, y0, y1):
    """One life.py generation for rows [y0, y1) of `state` (whole-raster
    array; only rows [y0 - 1, y1 + 1) are read) into the same rows of `out`."""
    lib().orc_life_rows(state, state.shape[1], state.shape[0], bs[0], bs[1], border, y0, y1, out)


def rand_u8(seed, shape, bs):
    out = np.empty(shape, np.uint8)
    lib().orc_rand_u8(seed, shape[1], shape[0], bs[0], bs[1], out)
    return out


def d8(dem, bs, border=0):
    dem = _c(dem, np.float32)
    out = np.empty(dem.shape, np.uint8)
    lib().orc_d8(dem, dem.shape[1], dem.shape[0], bs[0], bs[1], border, out)
    return out


def flowacc_s32(water, dirs):
    w = _c(water, np.int32)
    d = _c(dirs, np.uint8)
    out = np.empty(w.shape, np.int32)
    cyclic = lib().orc_flowacc_s32(w, d, w.shape[1], w.shape[0], out)
    return out, bool(cyclic)


def radial_f32(a, start, op=6):
    a = _c(a, np.float32)
    out = np.empty_like(a)
    lib().orc_radial_f32(a, a.shape[1], a.shape[0], start[0], start[1], op, out)
    return out


def wsum_f32(layers, weights):
    ls = [_c(l, np.float32) for l in layers]
    w = _c(weights, np.float32)
    ptrs = (ct.c_void_p * len(ls))(*[l.ctypes.data for l in ls])
    out = np.empty_like(ls[0])
    lib().orc_wsum_f32(ptrs, w, len(ls), ls[0].size, out)
    return out


def zone_stats(value, zone, nzones):
    """Per-zone count (uint64), min, max, float32 sum (row-major order) and
    float64 sum of `value` (float32) over `zone` (int32); cells with a zone id
    outside [0, nzones) or a NaN value are skipped."""
    v = _c(value, np.float32)
    z = _c(zone, np.int32)
    assert v.shape == z.shape
    cnt = np.zeros(nzones, np.uint64)
    mn = np.zeros(nzones, np.float32)
    mx = np.zeros(nzones, np.float32)
    s32 = np.zeros(nzones, np.float32)
    s64 = np.zeros(nzones, np.float64)
    lib().orc_zone_stats(v, z, v.size, nzones, cnt, mn, mx, s32, s64)
    return {"count": cnt, "min": mn, "max": mx, "sum32": s32, "sum64": s64}


def focal_src(W, H, bs, border, x, y, dx, dy):
    sx, sy = ct.c_int(), ct.c_int()
    ok = lib().orc_focal_src(W, H, bs[0], bs[1], border, x, y, dx, dy, ct.byref(sx), ct.byref(sy))
    return (sx.value, sy.value) if ok else None


def ulp_f32(x):
    """Size of one float32 ulp at |x|."""
    x = np.abs(np.asarray(x, np.float32))
    return np.spacing(x).astype(np.float64)
