"""Seeded synthetic rasters for tests and benchmarks.

No public dataset is used by the reference or its benchmark plan, so inputs are
generated with the shapes and value distributions the workloads name:
  * fBm DEM: `octaves` octaves of value noise (lattice values uniform in [0,1),
    smoothstep-interpolated), persistence 0.5, rescaled to [lo, hi] metres;
  * Bernoulli grids (U8 0/1);
  * lognormal value rasters;
  * uniform [0,1) layers;
  * Voronoi zone rasters (nearest of `n` uniform seed points).
All generators take an explicit seed. `xp` may be numpy or torch (arrays on the
device the torch tensors live on) for large rasters.
"""
import numpy as np


def _axis_weights(n, cells, xp, device=None):
    if xp is np:
        u = (np.arange(n, dtype=np.float64) + 0.5) * (cells / n)
        i = np.minimum(np.floor(u).astype(np.int64), cells - 1)
    else:
        u = (xp.arange(n, dtype=xp.float64, device=device) + 0.5) * (cells / n)
        i = xp.clamp(xp.floor(u).long(), max=cells - 1)
    f = u - i
    f = f * f * (3.0 - 2.0 * f)
    return i, f


def fbm_dem(h, w, seed, octaves=8, persistence=0.5, lo=0.0, hi=3000.0, base_cells=4, xp=np, device=None, threads=1):
    """float32 (h, w) fractal Brownian value-noise DEM rescaled to [lo, hi], row-major.
    threads > 1 (numpy only) computes row bands in parallel, with the same result."""
    if xp is np and threads > 1 and h >= 64 * threads:
        return _fbm_dem_bands(h, w, seed, octaves, persistence, lo, hi, base_cells, threads)
    rng = np.random.default_rng(seed)
    side = max(h, w)
    total = None
    amp = 1.0
    for o in range(octaves):
        cells = base_cells * (2 ** o)
        cx = max(1, int(round(cells * w / side)))
        cy = max(1, int(round(cells * h / side)))
        lat = rng.random((cy + 1, cx + 1))
        if xp is np:
            L = lat
        else:
            L = xp.as_tensor(lat, dtype=xp.float64, device=device)
        iy, fy = _axis_weights(h, cy, xp, device)
        ix, fx = _axis_weights(w, cx, xp, device)
        if xp is np:
            top = L[iy][:, ix] * (1 - fx)[None, :] + L[iy][:, ix + 1] * fx[None, :]
            bot = L[iy + 1][:, ix] * (1 - fx)[None, :] + L[iy + 1][:, ix + 1] * fx[None, :]
            noise = top * (1 - fy)[:, None] + bot * fy[:, None]
        else:
            Ly0, Ly1 = L[iy], L[iy + 1]
            top = Ly0[:, ix] * (1 - fx)[None, :] + Ly0[:, ix + 1] * fx[None, :]
            del Ly0
            bot = Ly1[:, ix] * (1 - fx)[None, :] + Ly1[:, ix + 1] * fx[None, :]
            del Ly1
            noise = top * (1 - fy)[:, None] + bot * fy[:, None]
            del top, bot
        total = noise * amp if total is None else total + noise * amp
        del noise
        amp *= persistence
    mn, mx = total.min(), total.max()
    out = (total - mn) / (mx - mn) * (hi - lo) + lo
    # row-major (C-contiguous) like every raster the engine reads through raw pointers
    return np.ascontiguousarray(out, dtype=np.float32) if xp is np else out.float().contiguous()


def _fbm_dem_bands(h, w, seed, octaves, persistence, lo, hi, base_cells, threads):
    import concurrent.futures as cf
    rng = np.random.default_rng(seed)
    side = max(h, w)
    lats = []
    for o in range(octaves):
        cells = base_cells * (2 ** o)
        cx = max(1, int(round(cells * w / side)))
        cy = max(1, int(round(cells * h / side)))
        lats.append((rng.random((cy + 1, cx + 1)), cx, cy))
    total = np.empty((h, w), np.float64)

    def band(r0, r1):
        amp = 1.0
        acc = None
        for lat, cx, cy in lats:
            iy, fy = _axis_weights(h, cy, np)
            ix, fx = _axis_weights(w, cx, np)
            iy, fy = iy[r0:r1], fy[r0:r1]
            top = lat[iy][:, ix] * (1 - fx)[None, :] + lat[iy][:, ix + 1] * fx[None, :]
            bot = lat[iy + 1][:, ix] * (1 - fx)[None, :] + lat[iy + 1][:, ix + 1] * fx[None, :]
            noise = top * (1 - fy)[:, None] + bot * fy[:, None]
            acc = noise * amp if acc is None else acc + noise * amp
            amp *= persistence
        total[r0:r1] = acc
        return acc.min(), acc.max()

    step = (h + threads * 4 - 1) // (threads * 4)
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        mm = list(ex.map(lambda r: band(r, min(h, r + step)), range(0, h, step)))
    mn = min(m[0] for m in mm)
    mx = max(m[1] for m in mm)
    out = np.empty((h, w), np.float32)

    def rescale(r0):
        r1 = min(h, r0 + step)
        out[r0:r1] = (total[r0:r1] - mn) / (mx - mn) * (hi - lo) + lo

    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(rescale, range(0, h, step)))
    return out


def bernoulli_u8(h, w, p, seed):
    rng = np.random.default_rng(seed)
    return (rng.random((h, w)) < p).astype(np.uint8)


def lognormal_f32(h, w, seed, mu=0.0, sigma=1.0):
    rng = np.random.default_rng(seed)
    return rng.lognormal(mu, sigma, size=(h, w)).astype(np.float32)


def uniform_f32(h, w, seed):
    rng = np.random.default_rng(seed)
    return rng.random((h, w), dtype=np.float32)


def voronoi_s32(h, w, n, seed, xp=np, device=None):
    """int32 (h, w) zone ids: index of the nearest of n uniform seed points
    (distance from cell centres; ties go to the lowest index).

    Cells are processed in square tiles; a seed can own a cell of a tile only if
    its distance to the tile is at most the smallest, over all seeds, of the
    distance to the tile's farthest corner, so each tile compares its cells
    with those candidate seeds only."""
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2)) * np.array([w, h])
    T = max(16, int(2 * np.sqrt(h * w / max(n, 1))))
    if xp is np:
        out = np.empty((h, w), np.int32)
    else:
        out = xp.empty((h, w), dtype=xp.int32, device=device)
        P = xp.as_tensor(pts, dtype=xp.float64, device=device)
    for y0 in range(0, h, T):
        y1 = min(h, y0 + T)
        for x0 in range(0, w, T):
            x1 = min(w, x0 + T)
            # distances from every seed to the tile's cell-centre rectangle
            dx_near = np.maximum(np.maximum(x0 + 0.5 - pts[:, 0], pts[:, 0] - (x1 - 0.5)), 0.0)
            dy_near = np.maximum(np.maximum(y0 + 0.5 - pts[:, 1], pts[:, 1] - (y1 - 0.5)), 0.0)
            dx_far = np.maximum(np.abs(x0 + 0.5 - pts[:, 0]), np.abs(x1 - 0.5 - pts[:, 0]))
            dy_far = np.maximum(np.abs(y0 + 0.5 - pts[:, 1]), np.abs(y1 - 0.5 - pts[:, 1]))
            r2 = np.min(dx_far ** 2 + dy_far ** 2)
            cand = np.nonzero(dx_near ** 2 + dy_near ** 2 <= r2)[0]
            if xp is np:
                ys = np.arange(y0, y1) + 0.5
                xs = np.arange(x0, x1) + 0.5
                c = pts[cand]
                d = (ys[None, :, None] - c[:, 1, None, None]) ** 2 + (xs[None, None, :] - c[:, 0, None, None]) ** 2
                out[y0:y1, x0:x1] = cand[np.argmin(d, axis=0)]
            else:
                ys = xp.arange(y0, y1, device=device, dtype=xp.float64) + 0.5
                xs = xp.arange(x0, x1, device=device, dtype=xp.float64) + 0.5
                ci = xp.as_tensor(cand, device=device)
                c = P[ci]
                d = (ys[None, :, None] - c[:, 1, None, None]) ** 2 + (xs[None, None, :] - c[:, 0, None, None]) ** 2
                out[y0:y1, x0:x1] = ci[xp.argmin(d, dim=0)].to(xp.int32)
    return out

