"""The reference's example scripts (python/hill.py, life.py, wsum.py, view.py),
copied byte for byte into a temporary directory and run unchanged with this
package's `map` module on the path (`from map import *`), on `.bin` inputs
written by the engine; their `.bin` outputs are checked against the oracle
(hill, life, wsum) or against the same program built in-process (view).

The scripts are read from MAP_REFERENCE_SCRIPTS (a directory holding them) or
from python/ of the reference checkout beside this repository; the test is
skipped where neither exists."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from map_b200 import synth
from map_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def scripts_dir():
    d = os.environ.get("MAP_REFERENCE_SCRIPTS")
    if d:
        return os.path.abspath(d)
    return os.path.join(os.path.dirname(ROOT), "reference", "python")


def copy_unchanged(name, tmp):
    src = os.path.join(scripts_dir(), name)
    if not os.path.exists(src):
        pytest.skip("reference script %s not available here" % name)
    dst = os.path.join(tmp, name)
    shutil.copyfile(src, dst)
    assert open(src, "rb").read() == open(dst, "rb").read()
    return dst


def run_script(path, *args):
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "map_b200"))
    r = subprocess.run([sys.executable, path] + [str(a) for a in args], cwd=os.path.dirname(path), env=env,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:]


def write_bin(M, arr, path, bs):
    M.write(M.from_numpy(arr, bs=list(bs)), path)


def read_bin(M, path):
    return M.to_numpy(M.read(path))


def test_hill_py_unchanged(M, tmp_path):
    script = copy_unchanged("hill.py", str(tmp_path))
    dem = synth.fbm_dem(1024, 1024, seed=21)
    inp, out = str(tmp_path / "dem.bin"), str(tmp_path / "hs.bin")
    write_bin(M, dem, inp, (256, 256))
    run_script(script, inp, out)
    got = read_bin(M, out)
    ref32 = O.hillshade_f32(dem, (256, 256), 0)
    ok, d, only = O.hill_tolerance(got, ref32, O.hillshade_bound(dem, (256, 256), 0))
    assert ok.all(), float(d.max())


def test_life_py_unchanged(M, tmp_path):
    script = copy_unchanged("life.py", str(tmp_path))
    out = str(tmp_path / "life.bin")
    ds, bs, gens = (600, 520), 128, 16
    run_script(script, out, ds[0], ds[1], bs, gens)
    got = read_bin(M, out)
    # rand(N, ds, U8, ROW+BLK, bs) > 128 with seed N = gens, then N generations
    # under the reference's block-mirror border
    init = (O.rand_u8(gens, (ds[1], ds[0]), (bs, bs)) > 128).astype(np.uint8)
    ref = O.life(init, (bs, bs), gens, border=0)
    assert got.dtype == np.uint8 and got.shape == ref.shape
    assert np.array_equal(got, ref)


def test_wsum_py_unchanged(M, tmp_path):
    script = copy_unchanged("wsum.py", str(tmp_path))
    layers = [synth.uniform_f32(700, 900, seed=60 + i) for i in range(4)]
    paths = []
    for i, l in enumerate(layers):
        p = str(tmp_path / ("r%d.bin" % (i + 1)))
        write_bin(M, l, p, (256, 256))
        paths.append(p)
    out = str(tmp_path / "wsum.bin")
    run_script(script, *paths, out)
    got = read_bin(M, out)
    ref = O.wsum_f32(layers, np.array([0.1, 0.2, 0.3, 0.4], np.float32))
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_view_py_unchanged(M, tmp_path):
    script = copy_unchanged("view.py", str(tmp_path))
    dem = synth.fbm_dem(400, 500, seed=23, hi=300.0)
    inp, out = str(tmp_path / "dem.bin"), str(tmp_path / "view.bin")
    write_bin(M, dem, inp, (128, 128))
    obs, h = (210, 170), 10.0
    run_script(script, inp, out, obs[0], obs[1], h)
    got = read_bin(M, out)
    # the same program built in-process (view.py:18-42)
    d = M.from_numpy(dem, bs=[128, 128])
    norm = (d - M.zmin(d)) / (M.zmax(d) - M.zmin(d))
    view = W.viewshed(norm, list(obs), h)
    f = [[1.0 / 16, 1.0 / 8, 1.0 / 16], [1.0 / 8, 1.0 / 4, 1.0 / 8], [1.0 / 16, 1.0 / 8, 1.0 / 16]]
    soft = M.convolve(view, f)
    want = M.to_numpy(M.con(soft < 0.1, d, M.zeros_like(d)))
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # the output keeps DEM values where the smoothed view is below 0.1, else 0
    assert np.all((got == dem) | (got == 0))
