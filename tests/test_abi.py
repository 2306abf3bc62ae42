"""C ABI: the library loads, exports every symbol include/map_b200.h declares,
reports errors instead of aborting, and applies the reference's metadata and
type rules when nodes are created (no GPU needed)."""
import ctypes as ct
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "map_b200.h")
LIB = os.path.join(ROOT, "map_b200", "libmap_b200.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ma_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ct.CDLL(LIB)
    names = declared_functions()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_abi_names_present():
    # the 37 entry points of the reference C ABI (front/bindings.hpp:27-92)
    ref = ["ma_setupDevices", "ma_increaseRef", "ma_decreaseRef", "ma_eval", "ma_value", "ma_nodeid", "ma_datatype",
           "ma_numdim", "ma_memorder", "ma_datasize", "ma_blocksize", "ma_read", "ma_write", "ma_constant", "ma_rand",
           "ma_cast", "ma_index", "ma_conditional", "ma_unary", "ma_binary", "ma_diversity", "ma_access",
           "ma_lhsAccess", "ma_neighbor", "ma_boundedNbh", "ma_spreadNeighbor", "ma_convolution", "ma_focalFunc",
           "ma_focalPercent", "ma_zonalReduc", "ma_radialScan", "ma_spreadScan", "ma_stats", "ma_barrier",
           "ma_loopStart", "ma_loopCond", "ma_loopBody", "ma_loopAgain", "ma_loopAssemble", "ma_loopEnd",
           "ma_loopAgainTail"]
    assert set(ref) <= set(declared_functions())


def test_pod_layouts(M):
    assert ct.sizeof(M.Variant) == 16
    assert ct.sizeof(M.Array) == 12


def test_errors_are_reported_not_fatal(M):
    with pytest.raises(M.MapError, match="null node"):
        M._lib.ma_unary(M.Raster(), M.SIN)
    with pytest.raises(M.MapError):
        M.read("/nonexistent/file.bin")
    with pytest.raises(M.MapError, match="symbolic loop capture"):
        M._lib.ma_loopStart()
    # the error state clears on the next successful call
    r = M.zeros([8, 8])
    assert r.datasize() == [8, 8]
    assert M._lib.ma_errorCode() == 0


def test_metadata_rules(M):
    a = M.ones([32, 16], M.U8, bs=[16, 16])
    b = M.ones([32, 16], M.S32, bs=[16, 16])
    f = M.ones([32, 16], M.F32, bs=[16, 16])
    assert (a + b).datatype() == M.S32                 # promote(U8,S32)
    assert (a * f).datatype() == M.F32
    assert (f < 1).datatype() == M.U8                  # relational -> U8 (runtime/dag/Binary.cpp:54)
    assert (~a).datatype() == M.U8
    assert M.convolve(a, [[1, 1, 1], [1, 0, 1], [1, 1, 1]]).datatype() == M.S32   # promote(U8, S32 mask)
    assert M.convolve(f, [[0.5, 1.0, 0.5]] * 3).datatype() == M.F32
    assert M.zsum(f).numdim() == M.D0
    assert M.index(f, M.D1).datatype() == M.S64
    assert M.astype(f, M.U16).datatype() == M.U16
    assert (f + 1).datasize() == [32, 16]
    assert f.blocksize() == [16, 16]
    assert f.numblock() == [2, 1]
    with pytest.raises(M.MapError, match="differ in shape"):
        M.ones([8, 8]) + M.ones([16, 8])
    with pytest.raises(M.MapError, match="unsigned"):
        b & b


def test_hash_consing_returns_existing_node(M):
    d = M.from_numpy(__import__("numpy").zeros((8, 8), "float32"))
    x1 = M.sqrt(d * 2.0)
    x2 = M.sqrt(d * 2.0)
    assert x1.nodeid() == x2.nodeid()
    assert M.convolve(d, [[1, 2, 1]] * 3).nodeid() == M.convolve(d, [[1, 2, 1]] * 3).nodeid()
    assert M.convolve(d, [[1, 2, 1]] * 3).nodeid() != M.convolve(d, [[1, 2, 2]] * 3).nodeid()


def test_scalar_graph_evaluates_on_host(M):
    a = M._const_to_raster(7)
    b = M._const_to_raster(2.5)
    c = M.sqrt(a * b + 1)
    M.eval(c)
    import numpy as np
    assert M.value(c) == np.float32(np.sqrt(np.float32(7 * 2.5 + 1)))


def test_truth_of_a_2d_raster_is_rejected(M):
    r = M.zeros([4, 4])
    with pytest.raises(M.MapError, match="2-D raster"):
        bool(r)
