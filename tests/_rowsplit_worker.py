"""One rank of the row-band split tests (launched by test_rowsplit.py with RANK /
WORLD_SIZE / MASTER_* set, as torchrun would): joins a gloo group, runs the
split's host steps of map_b200/rowsplit.py (band ownership, halo exchange by
point-to-point send / recv, gather, per-zone all-reduce) with the CPU oracle
computing each rank's rows, and on rank 0 compares the result with the
one-rank oracle evaluation of the whole raster. Prints one JSON line."""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from map_b200 import multigpu as MG  # noqa: E402
from map_b200 import rowsplit as RS  # noqa: E402
from map_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402


def full_rows(split, buf, fill):
    """A whole-raster array holding the buffer's rows [ya, yb) in place (other rows `fill`)."""
    a = np.full((split.H, split.W), fill, dtype=buf.numpy().dtype)
    a[split.ya:split.yb] = buf[:, :split.W].numpy()
    return a


def hill(rank, world, dist, border):
    H, W, bs = 301, 253, (64, 64)
    dem = synth.fbm_dem(H, W, seed=41)
    sp = RS.RowSplit(H, W, rank, world, margin=1)
    buf = sp.alloc(torch.float32)
    sp.own(buf)[:, :W] = torch.from_numpy(dem[sp.y0:sp.y1])
    sp.exchange(buf, dist)
    src = full_rows(sp, buf, np.nan)
    out = np.full((H, W), np.nan, np.float32)
    O.hillshade_rows(O.lib(), src, out, bs, border, sp.y0, sp.y1)
    full = sp.gather(torch.from_numpy(np.ascontiguousarray(out[sp.y0:sp.y1])), dist)
    if rank == 0:
        ref = O.hillshade_f32(dem, bs, border)
        return {"identical": bool(np.array_equal(full.numpy().view(np.uint32), ref.view(np.uint32)))}
    return {}


def life(rank, world, dist, border):
    H, W, bs, gens = 203, 150, (64, 64), 100
    grid = synth.bernoulli_u8(H, W, 0.3, seed=42)
    sp = RS.RowSplit(H, W, rank, world, margin=4)
    buf = sp.alloc(torch.uint8)
    sp.own(buf)[:, :W] = torch.from_numpy(grid[sp.y0:sp.y1])

    def run_chunk(src, dst_own, n):
        a = full_rows(sp, src, 0)
        b = np.zeros_like(a)
        for g in range(n):
            lo = max(0, sp.y0 - (n - 1 - g))
            hi = min(H, sp.y1 + (n - 1 - g))
            O.life_rows(a, b, bs, border, lo, hi)
            a, b = b, a
        dst_own[:, :W] = torch.from_numpy(a[sp.y0:sp.y1])

    res = RS.iterate(sp, buf, gens, dist, run_chunk)
    full = sp.gather(sp.own(res)[:, :W].contiguous(), dist)
    if rank == 0:
        ref = O.life(grid, bs, gens, border=border)
        return {"identical": bool(np.array_equal(full.numpy(), ref))}
    return {}


def zones(rank, world, dist):
    H, W, nz = 257, 311, 37
    val = synth.lognormal_f32(H, W, seed=43)
    val[5, 7] = -2.5                              # negative values and signed zeros take part too
    val[100, 200] = -0.0
    zone = synth.voronoi_s32(H, W, nz, seed=44)
    sp = RS.RowSplit(H, W, rank, world, margin=0)
    part = O.zone_stats(val[sp.y0:sp.y1], zone[sp.y0:sp.y1], nz)
    c, mn, mx, s = RS.zone_stats_allreduce(torch.from_numpy(part["count"].astype(np.int64)), torch.from_numpy(part["min"]),
                                           torch.from_numpy(part["max"]), torch.from_numpy(part["sum64"]), dist)
    ref = O.zone_stats(val, zone, nz)
    return {"count": bool(np.array_equal(c.numpy(), ref["count"].astype(np.int64))),
            "min": bool(np.array_equal(mn.numpy().view(np.uint32), ref["min"].view(np.uint32))),
            "max": bool(np.array_equal(mx.numpy().view(np.uint32), ref["max"].view(np.uint32))),
            "sum_rel": float(np.max(np.abs(s.numpy() - ref["sum64"]) / np.abs(ref["sum64"])))}


def zonal(rank, world, dist):
    """Whole-raster reductions of a row-split raster: each rank reduces its own
    rows, zonal_allreduce combines them."""
    H, W = 257, 311
    val = synth.lognormal_f32(H, W, seed=45).astype(np.float64)
    val[3, 4] = -7.25
    ints = (np.arange(H * W, dtype=np.int64).reshape(H, W) * 2654435761) % 1000003 - 500000
    small = (ints % 3 + 1).astype(np.int64)
    sp = RS.RowSplit(H, W, rank, world, margin=0)
    mine = slice(sp.y0, sp.y1)
    res = {}
    s = RS.zonal_allreduce(float(val[mine].sum()), RS.SUM, dist)
    res["fsum_rel"] = abs(s - float(val.sum())) / abs(float(val.sum()))
    res["fmax"] = RS.zonal_allreduce(float(val[mine].max()), RS.MAX, dist) == float(val.max())
    res["fmin"] = RS.zonal_allreduce(float(val[mine].min()), RS.MIN, dist) == float(val.min())
    res["isum"] = RS.zonal_allreduce(int(ints[mine].sum()), RS.SUM, dist) == int(ints.sum())
    res["imax"] = RS.zonal_allreduce(int(ints[mine].max()), RS.MAX, dist) == int(ints.max())
    res["imin"] = RS.zonal_allreduce(int(ints[mine].min()), RS.MIN, dist) == int(ints.min())
    tot = 1
    for v in small[:, :2].ravel():
        tot = (tot * int(v)) & 0xFFFFFFFF
    want = tot - (1 << 32) if tot >= 1 << 31 else tot
    p = 1
    for v in small[mine, :2].ravel():
        p = (p * int(v)) & 0xFFFFFFFF
    res["iprod_wrapped"] = RS.zonal_allreduce(p, RS.PROD, dist, bits=32) == want
    res["and"] = RS.zonal_allreduce(bool((ints[mine] != 0).all()), RS.AND, dist) == bool((ints != 0).all())
    res["or"] = RS.zonal_allreduce(bool((ints[mine] == 7).any()), RS.OR, dist) == bool((ints == 7).any())
    return res


def engine(rank, world, dist, kind, border):
    """The same split with each rank's rows computed by the engine on the GPU
    (ma_fromDeviceRows / ma_evalRows); rank 0 compares with a one-process
    whole-raster engine evaluation."""
    from map_b200 import map as M
    from map_b200 import workloads as W
    M.set_border(border)
    dev = torch.device("cuda", 0)
    H, Wd, bs = 517, 389, [128, 128]
    if kind == "hill":
        dem = synth.fbm_dem(H, Wd, seed=51)
        sp = RS.RowSplit(H, Wd, rank, world, margin=1)
        buf = sp.alloc(torch.float32, dev)
        sp.own(buf)[:, :Wd] = torch.from_numpy(dem[sp.y0:sp.y1]).to(dev)
        sp.exchange(buf, dist)
        out = sp.alloc(torch.float32, dev)
        RS.run_rows(M, sp, lambda d: W.hillshade(d), [(buf, M.F32)], sp.own(out), bs=bs)
        full = sp.gather(sp.own(out)[:, :Wd].contiguous(), dist)
        if rank == 0:
            ref = M.to_numpy(W.hillshade(M.from_numpy(dem, bs=bs)))
            return {"identical": bool(np.array_equal(full.cpu().numpy().view(np.uint32), ref.view(np.uint32)))}
        return {}
    gens = 30
    grid = synth.bernoulli_u8(H, Wd, 0.3, seed=52)
    sp = RS.RowSplit(H, Wd, rank, world, margin=8)
    buf = sp.alloc(torch.uint8, dev)
    sp.own(buf)[:, :Wd] = torch.from_numpy(grid[sp.y0:sp.y1]).to(dev)
    res = RS.iterate(sp, buf, gens, dist, RS.engine_chunk(M, sp, W.life_step, M.U8, bs=bs))
    full = sp.gather(sp.own(res)[:, :Wd].contiguous(), dist)
    if rank == 0:
        ref = M.to_numpy(W.life(M.from_numpy(grid, bs=bs), gens))
        return {"identical": bool(np.array_equal(full.cpu().numpy(), ref))}
    return {}


def main():
    mode = sys.argv[1]
    rank, local, world = MG.rank_info()
    dist = MG.init("gloo", world, timeout_s=60)
    try:
        if mode.startswith("engine"):
            res = engine(rank, world, dist, mode[6:10], int(mode[10:]))
        elif mode.startswith("hill"):
            res = hill(rank, world, dist, int(mode[4:]))
        elif mode.startswith("life"):
            res = life(rank, world, dist, int(mode[4:]))
        elif mode == "zonal":
            res = zonal(rank, world, dist)
        else:
            res = zones(rank, world, dist)
        print(json.dumps(dict(res, rank=rank)), flush=True)
        MG.finish(dist)
    except Exception as e:
        print(json.dumps({"rank": rank, "error": "%s: %s" % (type(e).__name__, e)}), flush=True)
        sys.exit(3)


if __name__ == "__main__":
    main()
