"""The C++ front end (include/map_b200.hpp): a C++ program written against it
builds the same operator graph as the Python module (identical generated
kernels, checked without a GPU) and computes the same results (GPU)."""
import ctypes as ct
import os
import subprocess

import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "map_b200")


@pytest.fixture(scope="module")
def program(tmp_path_factory, _built):
    exe = str(tmp_path_factory.mktemp("cpp") / "frontend_programs")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "frontend_programs.cpp"), "-o", exe, "-L", LIBDIR,
                    "-lmap_b200", "-Wl,-rpath," + LIBDIR], check=True, capture_output=True, text=True)
    return exe


def _python_source(M, w, h):
    r = M.from_numpy(np.zeros((h, w), np.float32), bs=[w, h])
    arr = M._node_array([W.hillshade(r)])
    n = M._lib.ma_generatedSource(arr, 1, None, 0)
    buf = ct.create_string_buffer(n + 1)
    M._lib.ma_generatedSource(arr, 1, buf, n + 1)
    return buf.value.decode()


def test_cpp_hillshade_builds_the_same_kernels_as_python(M, program):
    got = subprocess.run([program, "source", "300", "200"], check=True, capture_output=True, text=True).stdout
    assert got.strip() == _python_source(M, 300, 200).strip()
    assert "map_focal_" in got


def test_cpp_scalar_loop_with_materialize(program):
    out = subprocess.run([program, "loop"], check=True, capture_output=True, text=True).stdout.split()
    assert out[:2] == ["12", "4"]
    assert int(out[2]) < 16          # the loop's history is dropped as it goes


@pytest.mark.gpu
def test_cpp_programs_match_python_results(M, program, tmp_path):
    h, w = 240, 310
    dem = synth.fbm_dem(h, w, seed=44)
    src, out = tmp_path / "dem.f32", tmp_path / "out.bin"
    dem.tofile(src)
    subprocess.run([program, "eval", str(src), str(w), str(h), str(out)], check=True, capture_output=True, text=True)
    raw = np.fromfile(out, np.uint8)
    n = w * h
    hs = raw[:4 * n].view(np.float32).reshape(h, w)
    vs = raw[4 * n:8 * n].view(np.float32).reshape(h, w)
    acc = raw[8 * n:].view(np.int32).reshape(h, w)
    d = M.from_numpy(dem, bs=[w, h])
    assert np.array_equal(hs, M.to_numpy(W.hillshade(d)))
    ref_vs = M.to_numpy(M.viewshed(d, [w // 3, h // 2], 10.0))
    assert np.array_equal(np.isnan(vs), np.isnan(ref_vs))
    assert np.array_equal(vs[~np.isnan(vs)], ref_vs[~np.isnan(ref_vs)])
    assert np.array_equal(acc, M.to_numpy(M.flow_accumulation(M.ones_like(d, M.S32), M.flow_direction(d))))
