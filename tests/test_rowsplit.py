"""One raster split over ranks by row bands (map_b200/rowsplit.py), with 2 and
3 ranks as processes on a gloo group over 127.0.0.1: halo rows exchanged by
point-to-point send / recv into each rank's own buffer, rows computed per rank
(here by the CPU oracle), gathered on rank 0 and compared with the one-rank
evaluation. Hillshade under the three border rules and Game of Life over 100
generations (halo of 4 rows exchanged every 4 generations) are bit-identical;
per-zone count / min / max are bit-identical and sums agree to float64
rounding; whole-raster reductions (zsum, zprod, zmax, zmin, rAND, rOR)
combined across ranks are exact for integers and float max / min."""
import json
import os
import socket
import subprocess
import sys

import pytest

from map_b200 import rowsplit as RS

HERE = os.path.dirname(os.path.abspath(__file__))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(mode, world, timeout=180):
    port = _port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "_rowsplit_worker.py"), mode], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = {}
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            o, e = p.communicate()
        lines = [l for l in o.splitlines() if l.startswith("{")]
        res = json.loads(lines[-1]) if lines else {"error": e[-2000:]}
        assert p.returncode == 0 and "error" not in res, (mode, res, e[-2000:])
        outs[res["rank"]] = res
    return outs


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_hillshade_split_is_identical(world, border):
    assert _run("hill%d" % border, world)[0]["identical"]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("border", [0, 2])
def test_life_100_generations_split_is_identical(world, border):
    assert _run("life%d" % border, world)[0]["identical"]


@pytest.mark.parametrize("world", [2, 3])
def test_zone_stats_allreduce(world):
    outs = _run("zones", world)
    for r in range(world):
        assert outs[r]["count"] and outs[r]["min"] and outs[r]["max"], outs[r]
        assert outs[r]["sum_rel"] < 1e-12


@pytest.mark.parametrize("world", [2, 3])
def test_whole_raster_reductions_allreduce(world):
    """zsum / zprod / zmax / zmin / rAND / rOR of a row-split raster: each
    rank's reduction of its own rows combined on every rank. Integer results
    and float max / min are exact, float sums agree to float64 rounding."""
    outs = _run("zonal", world)
    for r in range(world):
        o = outs[r]
        assert all(o[k] for k in ("fmax", "fmin", "isum", "imax", "imin", "iprod_wrapped", "and", "or")), o
        assert o["fsum_rel"] < 1e-12


def test_band_rows_partition():
    for H in (7, 100, 1001):
        for world in (1, 2, 3, 7):
            rows = [RS.band_rows(H, world, r) for r in range(world)]
            assert rows[0][0] == 0 and rows[-1][1] == H
            assert all(rows[i][1] == rows[i + 1][0] for i in range(world - 1))
            assert max(b - a for a, b in rows) - min(b - a for a, b in rows) <= 1
    with pytest.raises(ValueError):
        RS.RowSplit(10, 4, 0, 4, margin=3)    # bands of 2-3 rows cannot carry a 3-row halo
