"""Benchmark: fused hillshade (python/hill.py) on a 16384 x 16384 float32 fBm DEM.

One step = one pass of the hot path over one batch: the hillshade program
(one fused focal kernel) over the whole DEM. Per rank the DEM is its own
independent raster (weak scaling, no data-path collective).

  value  -- Gcells/s with the DEM and the output resident in HBM (all ranks,
            units / max-over-ranks device time), CUDA events on the engine's stream;
  e2e    -- the same metric through the public C ABI with pinned HOST buffers:
            every step uploads the DEM, runs the program and downloads the result;
  roofline -- algorithmic 8 B/cell (4 B read + 4 B written) per launch over the
            measured kernel duration, against the measured HBM copy bandwidth;
  cpu_baseline -- the C oracle (restatement of the reference semantics) on the
            host cores, on a bounded window of the same DEM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--size S]
"""
import argparse
import concurrent.futures as cf
import faulthandler
import ctypes as ct
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL = 8          # fused hillshade: read 4 B + write 4 B per cell
METRIC = "hillshade Gcells/s & %HBM peak (fused/batched vs plain); tile p50/p99 ms"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--size", type=int, default=16384)
    p.add_argument("--block", type=int, default=256)
    p.add_argument("--e2e-steps", type=int, default=0, help="steps of the host-buffer e2e run (0: --steps)")
    p.add_argument("--no-clocks", action="store_true")
    p.add_argument("--no-mix", action="store_true", help="skip the batched-mix, zonal and serving sections")
    p.add_argument("--sections", default="plain,wsum,batched,life,zonal_stats,serving",
                   help="comma-separated extra sections, each printed as its own JSON line before the headline "
                        "(plain, wsum, batched, life, zonal_stats, serving; the parity section always runs)")
    p.add_argument("--zonal-size", type=int, default=16384)
    p.add_argument("--literal-chain", action="store_true",
                   help="generate hillshade as the literal operator chain (no algebraic rewrite)")
    p.add_argument("--one-cell", action="store_true", help="one cell per thread step (no paired f32x2 cells)")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- CPU baseline

class CpuHillshade:
    """The C oracle (restatement of the reference semantics), -O3 -march=native,
    computing row bands of one raster on all host threads (ctypes releases the
    GIL). The thread pool is created once, outside any timed region."""

    def __init__(self, threads=None):
        from oracle import oracle as O
        self.O = O
        self.L = O.lib_native()
        self.threads = threads or os.cpu_count() or 1
        self.pool = cf.ThreadPoolExecutor(max_workers=self.threads)
        list(self.pool.map(lambda _: None, range(self.threads)))   # start the workers

    def run(self, dem, out, rows, bs=(256, 256), border=0):
        """Computes rows [0, rows) of the hillshade of the whole `dem` into `out`."""
        n = self.threads * 4
        cuts = [rows * i // n for i in range(n + 1)]
        list(self.pool.map(lambda i: self.O.hillshade_rows(self.L, dem, out, bs, border, cuts[i], cuts[i + 1]),
                           range(n)))

    def close(self):
        self.pool.shutdown()


def cpu_baseline(dem_host, seconds_budget=10.0, rows=2048):
    """Times whole passes over rows [0, rows) of the full DEM (borders decided by
    the whole raster) on all host threads, repeating passes up to the budget."""
    import numpy as np
    cpu = CpuHillshade()
    out = np.empty_like(dem_host)
    rows = min(rows, dem_host.shape[0])
    cpu.run(dem_host, out, rows)    # warm (page faults, library load)
    passes, t0 = 0, time.perf_counter()
    while True:
        cpu.run(dem_host, out, rows)
        passes += 1
        if time.perf_counter() - t0 > seconds_budget or passes >= 200:
            break
    dt = time.perf_counter() - t0
    cpu.close()
    cells = rows * dem_host.shape[1]
    return {"value": round(cells * passes / dt / 1e9, 6), "unit": "Gcells/s", "cores": cpu.threads, "kind": "port",
            "sample": "rows 0-%d of the %dx%d DEM (all columns) x %d passes, oracle/oracle.c hillshade "
                      "(-O3 -march=native, -ffp-contract=off) in row bands on %d threads" % (
                          rows, dem_host.shape[1], dem_host.shape[0], passes, cpu.threads)}


# ---------------------------------------------------------------- clocks

class Clocks:
    """Samples the GPU's SM clock and clock-event (throttle) reasons during a
    timed region: NVML read in-process every 2 ms on a thread (so that regions of
    a few tens of ms get samples), else `nvidia-smi -lms 100` into a CSV file.
    Only reads; changes no setting."""

    def __init__(self, index, enabled=True, device=None):
        self.enabled = enabled
        self.index = index
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None
        # the nvidia-smi fallback's CSV: MAP_B200_CLOCKS_DIR, else the temporary directory
        import tempfile
        cdir = os.environ.get("MAP_B200_CLOCKS_DIR", tempfile.gettempdir())
        self.path = os.path.join(cdir, "map_b200_clocks_rank%d.csv" % index) if enabled else None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device if self.device is not None else self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        if not self.enabled:
            return self
        import threading
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap,
                    "hw_power_brake_slowdown": nv.nvmlClocksEventReasonHwPowerBrakeSlowdown}
            self.stop = threading.Event()

            def run():
                while not self.stop.is_set():
                    try:
                        sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.rows.append((sm, [k for k, b in bits.items() if rs & b]))
                    except Exception:
                        pass
                    self.stop.wait(0.002)
            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.thread is not None:
            if not self.rows:
                return None
            sm = [r[0] for r in self.rows]
            reasons = sorted({k for r in self.rows for k in r[1]})
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(self.rows), "source": "nvml, 2 ms"}
        if self.proc is None or self.path is None:
            return None
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, 100 ms"}


# ---------------------------------------------------------------- reference arm

def run_reference(args, rank, world):
    """The reference's CPU implementation of the path: its OpenCL pipeline cannot
    be built here, so the oracle port (a C restatement of its semantics,
    -O3 -march=native) runs on all host cores. One step = the hillshade of the
    whole size^2 DEM (rank 0's DEM of the GPU arm: same generator and seed),
    computed in row bands by a thread pool created before the timed steps."""
    if rank != 0:
        return
    import numpy as np
    from map_b200 import synth
    S = args.size
    threads = os.cpu_count() or 1
    dem = synth.fbm_dem(S, S, seed=1000, threads=threads)
    out = np.empty_like(dem)
    cpu = CpuHillshade(threads)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cpu.run(dem, out, S)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    cpu.close()
    ms = statistics.median(times) * 1e3
    v = S * S / (ms * 1e-3) / 1e9
    sample = "the whole %dx%d DEM per step (%d warm-up + %d timed passes, median), oracle/oracle.c hillshade " \
             "(-O3 -march=native) in row bands on %d threads" % (S, S, args.warmup, args.steps, threads)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 6), "unit": "Gcells/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "fused hillshade (hill.py), %dx%d F32 fBm DEM (8 octaves, persistence 0.5, "
                                   "0-3000 m), %dx%d blocks, block-mirror border" % (S, S, args.block, args.block),
                       "sample": "whole raster per step"},
            "cpu_baseline": {"value": round(v, 6), "unit": "Gcells/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(v, 6), "unit": "Gcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- mixes

def bench_batched(M, W, synth, torch, dev, n_rasters=512, steps=5, seed=5):
    """512 rasters, sides log-uniform in [64, 2048], aspect uniform in [0.5, 2],
    each running fused hillshade + a 6-layer weighted overlay, three ways: the
    plain path (one launch per group per 256x256 block, the reference's launch
    order), the fused path (one launch per group per raster) and the batched
    persistent launch (graph replay). Raster-edge mirror border. Every output of
    every raster is compared between the three."""
    import numpy as np
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    weights = [0.1, 0.2, 0.3, 0.15, 0.15, 0.1]
    M.set_border(M.BORDER_RASTER_MIRROR)
    keep, progs = [], []
    cells = 0
    for i in range(n_rasters):
        side = float(np.exp(rng.uniform(np.log(64), np.log(2048))))
        asp = float(rng.uniform(0.5, 2.0))
        w = max(8, int(round(side * np.sqrt(asp))))
        h = max(8, int(round(side / np.sqrt(asp))))
        pw = (w + 31) // 32 * 32
        dem = torch.zeros((h, pw), dtype=torch.float32, device=dev)
        dem[:, :w] = synth.fbm_dem(h, w, seed=seed * 1000 + i, xp=torch, device=dev)
        lay = [torch.rand((h, pw), generator=gen, device=dev) for _ in range(6)]
        outs = [torch.zeros((h, pw), dtype=torch.float32, device=dev) for _ in range(6)]   # plain, fused, batched x 2
        bs = [256, 256]
        dn = M.from_device(dem.data_ptr(), pw * 4, [w, h], M.F32, bs)
        ln = [M.from_device(l.data_ptr(), pw * 4, [w, h], M.F32, bs) for l in lay]
        progs.append((W.hillshade(dn), W.wsum(ln, weights), outs, pw * 4, w))
        keep.append((dem, lay, dn, ln))
        cells += w * h
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(M.stream(), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def per_raster(mode, slot):
        M.set_exec_mode(mode)
        try:
            for hs, ov, outs, pitch, _ in progs[:8]:      # warm (compiles)
                M.to_device(hs, outs[slot].data_ptr(), pitch, sync=False)
                M.to_device(ov, outs[slot + 1].data_ptr(), pitch, sync=False)
            M.sync()
            n0 = M._lib.ma_totalLaunchCount()
            e0.record(stream)
            for hs, ov, outs, pitch, _ in progs:
                M.to_device(hs, outs[slot].data_ptr(), pitch, sync=False)
                M.to_device(ov, outs[slot + 1].data_ptr(), pitch, sync=False)
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1), M._lib.ma_totalLaunchCount() - n0
        finally:
            M.set_exec_mode(M.EXEC_FUSED)

    plain_ms, plain_launches = per_raster(M.EXEC_PLAIN, 0)
    fused_ms, fused_launches = per_raster(M.EXEC_FUSED, 2)
    # batched path
    b = M.Batch()
    for hs, ov, outs, pitch, _ in progs:
        b.add([hs, ov], [(outs[4].data_ptr(), pitch), (outs[5].data_ptr(), pitch)])
    t0 = time.perf_counter()
    b.prepare(autotune=True)
    prep_s = time.perf_counter() - t0
    b.run()
    e0.record(stream)
    for _ in range(steps):
        b.run(sync=False)
    e1.record(stream)
    e1.synchronize()
    M.sync()
    batch_ms = e0.elapsed_time(e1) / steps
    plain_same = fused_same = True
    for hs, ov, outs, pitch, w in progs:
        for k in (0, 1):
            bo = outs[4 + k][:, :w]
            plain_same &= bool(torch.equal(outs[k][:, :w], bo))
            fused_same &= bool(torch.equal(outs[2 + k][:, :w], bo))
    M.set_border(M.BORDER_BLOCK_MIRROR)
    info = b.info()
    return {"rasters": n_rasters, "cells": cells, "value": round(cells / (batch_ms * 1e-3) / 1e9, 3),
            "fused_value": round(cells / (fused_ms * 1e-3) / 1e9, 3),
            "plain_value": round(cells / (plain_ms * 1e-3) / 1e9, 3), "unit": "Gcells/s",
            "speedup_vs_plain": round(plain_ms / batch_ms, 2), "speedup_vs_fused_per_raster": round(fused_ms / batch_ms, 2),
            "ms_per_step": round(batch_ms, 3), "fused_ms": round(fused_ms, 3), "plain_ms": round(plain_ms, 3),
            "plain_launches": plain_launches, "fused_launches": fused_launches,
            "batched_launches_per_step": info["launches"], "prepare_s": round(prep_s, 2), "kinds": info["kinds"],
            "all_outputs_plain_equal_batched": plain_same, "all_outputs_fused_equal_batched": fused_same,
            "programs": "fused hillshade + 6-layer weighted overlay per raster"}


def bench_serving(M, synth, torch, dev, size=32768, rates=(200, 1000, 2000, 5000, 10000), outstanding=(4, 16, 64),
                  seconds=3.0):
    """Requests over a device-resident size^2 DEM: windows 256^2/512^2/1024^2 at
    uniform offsets, mix 50% hillshade / 20% slope / 15% viewshed (observer
    height 10 m, radius 167 cells = 5 km at 30 m) / 15% D8 + flow accumulation;
    admission by an HBM budget of 8 GiB. Open loop: Poisson arrivals at each
    rate (up to past saturation); closed loop: a fixed number of requests kept
    in flight (the throughput ceiling). mean_batch is per run."""
    dem = synth.fbm_dem(size, size, seed=4242, xp=torch, device=dev).contiguous()
    torch.cuda.synchronize()
    srv = M.Server(dem.data_ptr(), size * 4, size, size, budget_bytes=8 << 30, max_batch=512)
    srv.load(rate=200, seconds=0.5, seed=99)            # warm-up: compiles every program kind
    out = {"dem": "%dx%d F32 fBm, resident" % (size, size), "mix": [0.5, 0.2, 0.15, 0.15], "runs": []}
    keys = ("mode", "requests", "throughput_req_s", "gcells_s", "p50_ms", "p99_ms", "batches", "mean_batch",
            "by_window", "by_program")
    for r in rates:
        res = srv.load(rate=r, seconds=seconds, seed=r)
        out["runs"].append({"rate_req_s": r} | {k: res[k] for k in keys})
    for n in outstanding:
        res = srv.load_closed(n, seconds, seed=1000 + n)
        out["runs"].append({"outstanding": n} | {k: res[k] for k in keys})
    srv.close()
    del dem
    return out


def bench_life(M, W, synth, torch, dev, size=4096, gens=100, steps=5, warmup=3, block=512):
    """Game of Life (life.py: 3x3 Moore neighbourhood, B3/S23): a size^2 U8 grid,
    Bernoulli(0.3) live cells, dead border, `gens` generations per step, fused
    (one launch per generation) vs plain (one launch per generation per block);
    the fused result is checked bit-exact against the oracle."""
    import numpy as np
    grid = synth.bernoulli_u8(size, size, 0.3, seed=2024)
    g_t = torch.from_numpy(grid).to(dev)
    out = torch.empty_like(g_t)
    torch.cuda.synchronize()   # the engine's stream does not wait for torch's
    M.set_border(M.BORDER_DEAD)
    try:
        src = M.from_device(g_t.data_ptr(), size, [size, size], M.U8, [block, block])
        prog = W.life(src, gens)
        st = torch.cuda.ExternalStream(M.stream(), device=dev)
        for _ in range(warmup):
            M.to_device(prog, out.data_ptr(), size, sync=False)
        M.sync()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = M._lib.ma_totalLaunchCount()
        ev0.record(st)
        for _ in range(steps):
            M.to_device(prog, out.data_ptr(), size, sync=False)
        ev1.record(st)
        ev1.synchronize()
        launches = M._lib.ma_totalLaunchCount() - l0
        ms = ev0.elapsed_time(ev1) / steps
        got = out.cpu().numpy()
        M.set_exec_mode(M.EXEC_PLAIN)
        M.to_device(prog, out.data_ptr(), size, sync=True)    # compile / warm
        t0 = time.perf_counter()
        M.to_device(prog, out.data_ptr(), size, sync=True)
        plain_ms = (time.perf_counter() - t0) * 1e3
        plain_same = bool(np.array_equal(out.cpu().numpy(), got))
    finally:
        M.set_exec_mode(M.EXEC_FUSED)
        M.set_border(M.BORDER_BLOCK_MIRROR)
    from oracle import oracle as O
    ref = O.life(grid, (block, block), gens, border=2)
    updates = size * size * gens
    peak, peak_kind = peaks()
    gbs = updates * 2 / (ms * 1e-3) / 1e9
    return {"workload": "Game of Life (life.py, B3/S23), %dx%d U8 Bernoulli(0.3), dead border, %d generations, %dx%d blocks"
                        % (size, size, gens, block, block),
            "value": round(updates / (ms * 1e-3) / 1e9, 2), "unit": "Gcell-updates/s", "ms_per_step": round(ms, 3),
            "steps": steps, "warmup": warmup, "launches_per_step": launches // steps,
            "plain_value": round(updates / (plain_ms * 1e-3) / 1e9, 3), "plain_ms": round(plain_ms, 2),
            "speedup_vs_plain": round(plain_ms / ms, 1), "plain_equals_fused": plain_same,
            "bit_exact_vs_oracle": bool(np.array_equal(got, ref)),
            "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s", "frac": round(gbs / peak, 4),
                         "bytes_per_cell_update": 2, "note": "the 16 MiB grid stays in L2 between generations"}}


def bench_zonal_stats(M, synth, torch, dev, size=16384, nzones=1024, steps=10, warmup=3):
    """Per-zone count/min/max/sum/mean: size^2 F32 lognormal(0, 1) values over a
    size^2 S32 Voronoi partition of `nzones` uniform seeds (8 B/cell read)."""
    import numpy as np
    g = torch.Generator(device=dev)
    g.manual_seed(31)
    val = torch.empty((size, size), dtype=torch.float32, device=dev).log_normal_(0.0, 1.0, generator=g)
    zone = synth.voronoi_s32(size, size, nzones, seed=32, xp=torch, device=dev).contiguous()
    outs = torch.zeros(nzones * 6, dtype=torch.float32, device=dev)
    cnt = torch.zeros(nzones, dtype=torch.int64, device=dev)
    st = torch.cuda.current_stream(dev)
    o = outs.data_ptr()

    def call():
        M.zonal_stats_device(val.data_ptr(), size * 4, zone.data_ptr(), size * 4, size, size, nzones, cnt.data_ptr(),
                             o, o + 4 * nzones, o + 8 * nzones, o + 12 * nzones, stream=st.cuda_stream)

    for _ in range(warmup):
        call()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(st)
    for _ in range(steps):
        call()
    ev1.record(st)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    cells = size * size
    peak, peak_kind = peaks()
    gbs = cells * 8 / (ms * 1e-3) / 1e9
    # accuracy against the FP64 oracle at full size
    from oracle import oracle as O
    v_h = val.cpu().numpy()
    z_h = zone.cpu().numpy()
    t0 = time.perf_counter()
    ref = O.zone_stats(v_h, z_h, nzones)
    cpu_s = time.perf_counter() - t0
    oh = outs.cpu().numpy()
    c_h = cnt.cpu().numpy().astype(np.uint64)
    exact = bool((c_h == ref["count"]).all() and (oh[:nzones].view(np.uint32) == ref["min"].view(np.uint32)).all()
                 and (oh[nzones:2 * nzones].view(np.uint32) == ref["max"].view(np.uint32)).all())
    rel_sum = float(np.max(np.abs(oh[2 * nzones:3 * nzones] - ref["sum64"]) / ref["sum64"]))
    mean64 = ref["sum64"] / ref["count"].astype(np.float64)
    rel_mean = float(np.max(np.abs(oh[3 * nzones:4 * nzones] - mean64) / mean64))
    del val, zone
    return {"workload": "per-zone count/min/max/sum/mean, %dx%d F32 lognormal(0,1) over %dx%d S32 Voronoi(%d)"
                        % (size, size, size, size, nzones),
            "value": round(cells / (ms * 1e-3) / 1e9, 3), "unit": "Gcells/s", "ms_per_step": round(ms, 4),
            "steps": steps, "warmup": warmup, "l2": "inputs larger than L2 (2 GiB per step)",
            "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(gbs / peak, 4), "bytes_per_cell": 8, "peak_kind": peak_kind},
            "count_min_max_bit_exact": exact, "max_rel_err_sum_vs_fp64": rel_sum,
            "max_rel_err_mean_vs_fp64": rel_mean,
            "cpu_baseline": {"value": round(cells / cpu_s / 1e9, 4), "unit": "Gcells/s", "cores": 1, "kind": "port",
                             "sample": "the whole %dx%d raster, oracle restatement (1 thread)" % (size, size)}}


# ---------------------------------------------------------------- hillshade sections

def bench_parity(M, W, torch, dem_t, out_t, block, win=2048):
    """Hillshade error statement on a win^2 window of the DEM (cells whose 3x3
    neighbourhood lies inside the window, so the window's own borders do not
    matter): the GPU result of the timed program against the FP32 oracle under the
    test tolerance, and both against the FP64 oracle; then the literal operator
    chain (rewrite off) on the same window."""
    import numpy as np
    from oracle import oracle as O
    S = dem_t.shape[0]
    y0, x0 = S // 2 - win // 2, S // 3
    dem_win = dem_t[y0:y0 + win, x0:x0 + win].cpu().numpy()
    bs = (block, block)
    ref32 = O.hillshade_f32(dem_win, bs, 0)[1:-1, 1:-1]
    ref64 = O.hillshade_f64(dem_win, bs, 0)[1:-1, 1:-1]
    bound = O.hillshade_bound(dem_win, bs, 0)[1:-1, 1:-1]

    def stats(got):
        ok, d, only = O.hill_tolerance(got, ref32, bound)
        e = np.abs(got.astype(np.float64) - ref64)
        ulp = O.ulp_f32(ref64)
        well = np.abs(ref64) >= 0.05
        return {"within_tolerance": bool(ok.all()), "max_abs_diff_vs_fp32_oracle": float(d.max()),
                "bit_identical_fraction": float((got == ref32).mean()),
                "cells_only_via_cancellation_clause": int(only.sum()),
                "max_abs_err_vs_fp64": float(e.max()), "max_ulp_err_vs_fp64_where_abs_ge_0.05": float((e / ulp)[well].max()),
                "max_rel_err_vs_fp64_where_abs_ge_0.05": float((e / np.abs(ref64))[well].max())}

    got = out_t[y0 + 1:y0 + win - 1, x0 + 1:x0 + win - 1].cpu().numpy()
    e32 = np.abs(ref32.astype(np.float64) - ref64)
    res = {"window": "%dx%d interior cells of a %dx%d window of the headline DEM" % (win - 2, win - 2, win, win),
           "tolerance": "4 ulp or 1e-5 rel of the FP32 oracle, or 4x the FP32 chain's first-order rounding-error "
                        "scale where its two terms cancel (oracle.hill_tolerance)",
           "fp32_oracle": {"max_abs_err_vs_fp64": float(e32.max()),
                           "max_ulp_err_vs_fp64_where_abs_ge_0.05": float((e32 / O.ulp_f32(ref64))[np.abs(ref64) >= 0.05].max())},
           "gpu": stats(got), "gpu_rewrite": M.get_algebraic_rewrite()}
    prev = M.get_algebraic_rewrite()
    try:
        M.set_algebraic_rewrite(not prev)
        wt = torch.from_numpy(dem_win).to(dem_t.device)
        torch.cuda.synchronize()
        d = M.from_device(wt.data_ptr(), win * 4, [win, win], M.F32, [block, block])
        other = M.to_numpy(W.hillshade(d))[1:-1, 1:-1]
        res["gpu_rewrite_off" if prev else "gpu_rewrite_on"] = stats(other)
    finally:
        M.set_algebraic_rewrite(prev)
    return res


def bench_plain(M, W, synth, torch, dev, block=256, steps=10, warmup=3):
    """The plain path (one launch per fusion group per block, in the reference's
    scheduler order) against the fused path (one launch per group): hillshade
    on the 1024^2 DEM in 256^2 blocks (the reference's CPU-runnable
    configuration) and on the 16384^2 DEM."""
    out = {}
    st = torch.cuda.ExternalStream(M.stream(), device=dev)
    for S, k in ((1024, steps * 5), (16384, 3)):
        dem_t = synth.fbm_dem(S, S, seed=77, xp=torch, device=dev).contiguous()
        o_t = torch.empty_like(dem_t)
        torch.cuda.synchronize()   # the engine's stream does not wait for torch's
        dem = M.from_device(dem_t.data_ptr(), S * 4, [S, S], M.F32, [block, block])
        hs = W.hillshade(dem)
        r = {}
        for mode, name in ((M.EXEC_FUSED, "fused"), (M.EXEC_PLAIN, "plain")):
            M.set_exec_mode(mode)
            try:
                for _ in range(warmup):
                    M.to_device(hs, o_t.data_ptr(), S * 4, sync=False)
                M.sync()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                l0 = M._lib.ma_totalLaunchCount()
                t0 = time.perf_counter()
                e0.record(st)
                for _ in range(k):
                    M.to_device(hs, o_t.data_ptr(), S * 4, sync=False)
                e1.record(st)
                e1.synchronize()
                host_ms = (time.perf_counter() - t0) * 1e3 / k
                ms = e0.elapsed_time(e1) / k
                r[name] = {"ms_per_step": round(ms, 4), "value": round(S * S / (ms * 1e-3) / 1e9, 3),
                           "launches_per_step": (M._lib.ma_totalLaunchCount() - l0) // k,
                           "host_ms_per_step": round(host_ms, 4), "steps": k}
                r[name + "_out"] = o_t.clone()
            finally:
                M.set_exec_mode(M.EXEC_FUSED)
        same = bool(torch.equal(r.pop("fused_out"), r.pop("plain_out")))
        out["%dx%d" % (S, S)] = dict(r, plain_equals_fused=same,
                                     fused_vs_plain=round(r["plain"]["ms_per_step"] / r["fused"]["ms_per_step"], 2))
        del dem_t, o_t, dem, hs
    out["unit"] = "Gcells/s"
    out["workload"] = "hillshade (hill.py), fBm DEM, %dx%d blocks, block-mirror border" % (block, block)
    return out


def bench_wsum(M, W, torch, dev, size=16384, steps=10, warmup=3):
    """Weighted overlay (wsum.py generalised to 6 layers): 6 F32 uniform[0,1)
    layers, weights summing to 1, one fused Local launch; 28 B/cell."""
    import numpy as np
    from oracle import oracle as O
    weights = [0.1, 0.2, 0.3, 0.15, 0.15, 0.1]
    g = torch.Generator(device=dev)
    g.manual_seed(17)
    lay = [torch.rand((size, size), generator=g, device=dev) for _ in range(6)]
    o_t = torch.empty((size, size), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()   # the engine's stream does not wait for torch's
    ln = [M.from_device(l.data_ptr(), size * 4, [size, size], M.F32, [256, 256]) for l in lay]
    prog = W.wsum(ln, weights)
    st = torch.cuda.ExternalStream(M.stream(), device=dev)
    for _ in range(warmup):
        M.to_device(prog, o_t.data_ptr(), size * 4, sync=False)
    M.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = M._lib.ma_totalLaunchCount()
    e0.record(st)
    for _ in range(steps):
        M.to_device(prog, o_t.data_ptr(), size * 4, sync=False)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    launches = (M._lib.ma_totalLaunchCount() - l0) // steps
    cells = size * size
    peak, peak_kind = peaks()
    gbs = cells * 28 / (ms * 1e-3) / 1e9
    # bit-exact against the oracle on a 1024-row window (element-wise: any window is exact)
    rows = 1024
    ls_h = [np.ascontiguousarray(l[:rows].cpu().numpy()) for l in lay]
    ref = O.wsum_f32(ls_h, np.array(weights, np.float32))
    got = o_t[:rows].cpu().numpy()
    exact = bool(np.array_equal(got.view(np.uint32), ref.view(np.uint32)))
    # CPU baseline: the native oracle on the same window, passes up to ~5 s, all threads
    L = O.lib_native()
    n = rows * size
    threads = os.cpu_count() or 1
    outc = np.empty_like(ls_h[0])
    cut = [n * i // threads for i in range(threads + 1)]
    wv = np.array(weights, np.float32)

    def part(i):
        ptrs = (ct.c_void_p * 6)(*[l.ctypes.data + 4 * cut[i] for l in ls_h])
        L.orc_wsum_f32(ptrs, wv, 6, cut[i + 1] - cut[i], outc.ctypes.data + 4 * cut[i])

    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(part, range(threads)))
        passes, t0 = 0, time.perf_counter()
        while passes < 100 and time.perf_counter() - t0 < 5.0:
            list(ex.map(part, range(threads)))
            passes += 1
        cdt = time.perf_counter() - t0
    del lay, o_t
    return {"workload": "weighted overlay (wsum.py) of 6 F32 uniform[0,1) layers, %dx%d, weights %s" % (size, size, weights),
            "value": round(cells / (ms * 1e-3) / 1e9, 3), "unit": "Gcells/s", "ms_per_step": round(ms, 4),
            "steps": steps, "warmup": warmup, "launches_per_step": launches,
            "l2": "inputs larger than L2 (7 GiB per step)",
            "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(gbs / peak, 4), "bytes_per_cell": 28, "peak_kind": peak_kind},
            "bit_exact_vs_oracle": exact,
            "cpu_baseline": {"value": round(n * passes / cdt / 1e9, 4), "unit": "Gcells/s", "cores": threads,
                             "kind": "port", "sample": "%d rows x %d columns x %d passes, oracle wsum (-O3 -march=native)"
                                                       % (rows, size, passes)}}


# ---------------------------------------------------------------- our arm

def main():
    faulthandler.enable()
    args = parse()
    from map_b200 import multigpu as MG
    rank, local, world = MG.rank_info()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = MG.init("nccl", world)

    from map_b200 import map as M
    from map_b200 import synth
    from map_b200 import workloads as W
    M._lib.ma_setDevice(local)
    M.set_algebraic_rewrite(not args.literal_chain)
    M.set_paired_cells(not args.one_cell)

    S = args.size
    cells = S * S
    dev = torch.device("cuda", local)
    dem_t = synth.fbm_dem(S, S, seed=1000 + rank, xp=torch, device=dev).contiguous()
    out_t = torch.empty_like(dem_t)
    torch.cuda.synchronize()
    pitch = S * 4
    dem = M.from_device(dem_t.data_ptr(), pitch, [S, S], M.F32, [args.block, args.block])
    hs = W.hillshade(dem)
    stream = torch.cuda.ExternalStream(M.stream(), device=dev)

    def barrier():
        MG.barrier(dist)

    # warm-up (compiles and loads the kernel)
    for _ in range(args.warmup):
        M.to_device(hs, out_t.data_ptr(), pitch, sync=False)
    M.sync()
    torch.cuda.synchronize()

    # timed: K steps, inputs resident in HBM, events on the engine's stream
    launches0 = M._lib.ma_totalLaunchCount()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with Clocks(local, enabled=not args.no_clocks, device=local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            M.to_device(hs, out_t.data_ptr(), pitch, sync=False)
        ev1.record(stream)
        while not ev1.query():   # poll (not a blocking wait) so the clock sampler keeps running
            time.sleep(0.0005)
    M.sync()
    torch.cuda.synchronize()
    barrier()
    launches = M._lib.ma_totalLaunchCount() - launches0
    ms = MG.max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist, dev)
    value = MG.job_throughput(cells, world, ms) / 1e9

    # end to end through the public API with pinned host buffers, every step
    # uploading the DEM and downloading the result
    e2e_steps = args.e2e_steps or args.steps
    nbytes = cells * 4
    h_in = M._lib.ma_hostAlloc(nbytes)
    h_out = M._lib.ma_hostAlloc(nbytes)
    dem_host = dem_t.cpu().numpy()
    ct.memmove(h_in, dem_host.ctypes.data, nbytes)
    dem_h = M.Raster(M._lib.ma_fromHost(ct.c_void_p(h_in), M.Array([S, S]), M.F32, M.Array([args.block, args.block]), 0))
    hs_h = W.hillshade(dem_h)
    M._lib.ma_toHost(hs_h, ct.c_void_p(h_out), nbytes)  # warm
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        M._lib.ma_toHost(hs_h, ct.c_void_p(h_out), nbytes)
    e2e_ms = MG.max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps, dist, dev)
    e2e_value = MG.job_throughput(cells, world, e2e_ms) / 1e9
    e2e_same = bool(np.array_equal(np.ctypeslib.as_array(ct.cast(h_out, ct.POINTER(ct.c_float)), shape=(S, S)),
                                   out_t.cpu().numpy()))
    del hs_h, dem_h
    M._lib.ma_hostFree(ct.c_void_p(h_in))
    M._lib.ma_hostFree(ct.c_void_p(h_out))

    if rank == 0:
        peak, peak_kind = peaks()
        achieved = cells * BYTES_PER_CELL / (ms * 1e-3) / 1e9
        traffic, traffic_src = None, None
        tpath = os.path.join(ROOT, "profiles", "hillshade_focal_traffic.json")
        if os.path.exists(tpath):
            try:
                with open(tpath) as f:
                    tj = json.load(f)
                key = "dram_bytes_per_launch_scaled_to_%d" % S
                if tj.get("rewrite") == M.get_algebraic_rewrite() and key in tj:
                    traffic = tj[key]
                    traffic_src = tj.get("captured")
            except Exception:
                traffic = None
        sections = [x for x in args.sections.split(",") if x] if (world == 1 and not args.no_mix) else []
        runners = {"parity": lambda: bench_parity(M, W, torch, dem_t, out_t, args.block),
                   "plain": lambda: bench_plain(M, W, synth, torch, dev, args.block),
                   "wsum": lambda: bench_wsum(M, W, torch, dev),
                   "batched": lambda: bench_batched(M, W, synth, torch, dev),
                   "life": lambda: bench_life(M, W, synth, torch, dev),
                   "zonal_stats": lambda: bench_zonal_stats(M, synth, torch, dev, size=args.zonal_size),
                   "serving": lambda: bench_serving(M, synth, torch, dev)}
        summary = {}
        for name in ["parity"] + sections:
            try:
                res = runners[name]()
            except Exception as e:   # reported, not fatal: the headline line still prints
                res = {"error": str(e)[:300]}
            print(json.dumps({"section": name} | res), flush=True)
            if name == "parity":
                parity = res
            elif isinstance(res, dict) and "value" in res:
                summary[name] = {k: res[k] for k in ("value", "unit") if k in res}
        cpu = cpu_baseline(dem_t.cpu().numpy(), seconds_budget=10.0)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Gcells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "fused hillshade (hill.py), %dx%d F32 fBm DEM (8 octaves, persistence 0.5, "
                                   "0-3000 m) per GPU, %dx%d blocks, block-mirror border" % (S, S, args.block, args.block),
                       "l2": "inputs larger than L2 (%.2f GiB in + %.2f GiB out per step)" % (nbytes / 2 ** 30, nbytes / 2 ** 30),
                       "parallelism": "independent raster per GPU (weak scaling)",
                       "algebraic_rewrite": M.get_algebraic_rewrite(), "paired_cells": M.get_paired_cells()},
            "e2e": {"value": round(e2e_value, 3), "unit": "Gcells/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "steps": e2e_steps, "equals_device_result": e2e_same},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_source": traffic_src,
                         "note": "achieved = 8 B/cell x cells / kernel time; peak %s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind},
            "cpu_baseline": cpu,
            "parity": {k: parity.get("gpu", {}).get(k) for k in ("within_tolerance", "max_abs_diff_vs_fp32_oracle",
                                                                 "max_abs_err_vs_fp64")} if isinstance(parity, dict) else None,
            "sections": summary,
        }
        ck = clk.summary()
        if ck:
            line["clocks"] = ck
        print(json.dumps(line), flush=True)
    MG.finish(dist)


if __name__ == "__main__":
    main()
