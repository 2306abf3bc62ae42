"""Row-range evaluation on the GPU (ma_fromDeviceRows / ma_evalRows): rows
[y0, y1) evaluated from inputs that hold only the rows the range reads equal
the same rows of a whole-raster evaluation, bit for bit, under every border
rule; and the row-band split of map_b200/rowsplit.py with two ranks as
processes on a gloo group, each computing its rows with the engine on the one
GPU (independent kernels; halo rows travel through host memory)."""
import os

import numpy as np
import pytest
import torch

from map_b200 import synth
from map_b200 import workloads as W

pytestmark = pytest.mark.gpu


def band_eval(M, arrays, dts, build, y0, y1):
    """Rows [y0, y1) of build(*inputs) from device bands holding rows [ya, yb)."""
    H, Wd = arrays[0].shape
    probe = build(*[M.from_numpy(a) for a in arrays])
    m = M.row_margin(probe)
    ya, yb = max(0, y0 - m), min(H, y1 + m)
    keep, nodes = [], []
    for a, dt in zip(arrays, dts):
        es = a.dtype.itemsize
        wp = (Wd * es + 127) // 128 * 128 // es
        t = torch.zeros((yb - ya, wp), dtype=torch.from_numpy(a[:1, :1]).dtype, device="cuda")
        t[:, :Wd] = torch.from_numpy(a[ya:yb]).cuda()
        keep.append(t)
        nodes.append(M.from_device_rows(t.data_ptr(), t.stride(0) * es, [Wd, H], dt, ya, yb - ya, bs=[128, 128]))
    prog = build(*nodes)
    es_out = np.dtype(M._np_dtype[prog.datatype()]).itemsize
    wpo = (Wd * es_out + 127) // 128 * 128 // es_out
    out = torch.zeros((y1 - y0, wpo), dtype=torch.from_numpy(np.zeros(1, M._np_dtype[prog.datatype()])).dtype,
                      device="cuda")
    torch.cuda.synchronize()   # the engine's stream does not wait for torch's
    M.eval_rows([prog], [(out.data_ptr(), out.stride(0) * es_out)], y0, y1)
    return out[:, :Wd].cpu().numpy()


RANGES = [(0, 37), (37, 300), (130, 131), (450, 517), (0, 517)]


@pytest.mark.parametrize("border", [0, 1, 2])
def test_hillshade_rows_equal_whole(fresh, border):
    M = fresh
    M.set_border(border)
    dem = synth.fbm_dem(517, 389, seed=61)
    whole = M.to_numpy(W.hillshade(M.from_numpy(dem, bs=[128, 128])))
    for y0, y1 in RANGES:
        got = band_eval(M, [dem], [M.F32], W.hillshade, y0, y1)
        assert np.array_equal(got.view(np.uint32), whole[y0:y1].view(np.uint32)), (y0, y1)


@pytest.mark.parametrize("border", [0, 2])
def test_life_generations_rows_equal_whole(fresh, border):
    M = fresh
    M.set_border(border)
    grid = synth.bernoulli_u8(517, 389, 0.3, seed=62)
    whole = M.to_numpy(W.life(M.from_numpy(grid, bs=[128, 128]), 7))
    for y0, y1 in RANGES:
        got = band_eval(M, [grid], [M.U8], lambda s: W.life(s, 7), y0, y1)
        assert np.array_equal(got, whole[y0:y1]), (y0, y1)


def test_overlay_and_chained_focal_rows(fresh):
    M = fresh
    a = synth.uniform_f32(300, 260, seed=63)
    b = synth.uniform_f32(300, 260, seed=64)

    def prog(x, y):
        blur = M.convolve(M.convolve(x, [[1, 2, 1]] * 3) * 0.5, [[1, 1, 1, 1, 1]] * 5)
        return blur * 0.25 + y
    whole = M.to_numpy(prog(M.from_numpy(a, bs=[128, 128]), M.from_numpy(b, bs=[128, 128])))
    for y0, y1 in [(0, 50), (120, 181), (250, 300)]:
        got = band_eval(M, [a, b], [M.F32, M.F32], prog, y0, y1)
        assert np.array_equal(got.view(np.uint32), whole[y0:y1].view(np.uint32)), (y0, y1)


def test_row_band_errors(fresh):
    M = fresh
    dem = synth.fbm_dem(200, 128, seed=65)
    t = torch.from_numpy(dem[40:90]).cuda()
    band = M.from_device_rows(t.data_ptr(), 128 * 4, [128, 200], M.F32, 40, 50)
    hs = W.hillshade(band)
    out = torch.zeros((10, 128), device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(M.MapError):     # rows [59, 71) read, but [40, 90) held: fine; rows [30, 40) are not
        M.eval_rows([hs], [(out.data_ptr(), 512)], 30, 40)
    M.eval_rows([hs], [(out.data_ptr(), 512)], 60, 70)
    whole = M.to_numpy(W.hillshade(M.from_numpy(dem)))
    assert np.array_equal(out.cpu().numpy(), whole[60:70])
    with pytest.raises(M.MapError):     # a band input cannot be evaluated whole
        M.to_numpy(hs)
    with pytest.raises(M.MapError):
        M.from_device_rows(t.data_ptr(), 512, [128, 200], M.F32, 190, 50)


@pytest.mark.parametrize("mode", ["enginehill0", "enginehill2", "enginelife0", "enginelife2"])
def test_two_ranks_on_one_gpu_equal_one(mode):
    outs = _run_gpu(mode)
    assert outs[0]["identical"]


def _run_gpu(mode):
    import json
    import socket
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(here, "_rowsplit_worker.py"), mode], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = {}
    for p in procs:
        try:
            o, e = p.communicate(timeout=600)
        except subprocess.TimeoutExpired:
            p.kill()
            o, e = p.communicate()
        lines = [l for l in o.splitlines() if l.startswith("{")]
        res = json.loads(lines[-1]) if lines else {"error": e[-2000:]}
        assert p.returncode == 0 and "error" not in res, (mode, res, e[-2000:])
        outs[res["rank"]] = res
    return outs
