"""The reference's example workloads expressed on the `map` API.

Each function builds the same operator graph as the corresponding reference
script, operator by operator and in the same order, so fusion, dtypes and the
floating-point evaluation order match:
  hillshade  -- python/hill.py:15-50   (Sobel /8/dist, slope, aspect, hillshade)
  life       -- python/life.py:24-34   (B3/S23 with a 3x3 Moore correlation)
  stats      -- python/stats.py:13-34  (global zonal statistics)
  wsum       -- python/wsum.py:11      (weighted overlay, left to right)
  viewshed   -- python/view.py:18-37   (radial max of slopes from an observer)
"""
from . import map as M

PI = 3.141593   # the constant the reference scripts use


def hori(dem, dist=1):
    h = [[-1, 0, 1],
         [-2, 0, 2],
         [-1, 0, 1]]
    return M.convolve(dem, h) / (8 * dist)


def vert(dem, dist=1):
    v = [[-1, -2, -1],
         [0, 0, 0],
         [1, 2, 1]]
    return M.convolve(dem, v) / (8 * dist)


def slope(dem, zf=1, dist=1):
    x = hori(dem, dist)
    y = vert(dem, dist)
    return M.atan(zf * M.sqrt(x * x + y * y))


def aspect(dem, dist=1):
    x = hori(dem, dist)
    y = vert(dem, dist)
    z1 = (x != 0) * M.atan2(y, -x)
    z1 = z1 + (z1 < 0) * (PI * 2)
    z0 = (x == 0) * ((y > 0) * (PI / 2) + (y < 0) * (PI * 2 - PI / 2))
    return z1 + z0


def hillshade(dem, zenith=45, azimuth=315):
    zr = (90 - float(zenith)) / 180 * PI
    ar = 360 - float(azimuth) + 90
    ar = ar - 360 if (ar > 360) else ar
    ar = ar / 180 * PI
    return (M.cos(zr) * M.cos(slope(dem)) +
            M.sin(zr) * M.sin(slope(dem)) * M.cos(ar - aspect(dem)))


def life_step(state):
    S = [[1, 1, 1],
         [1, 0, 1],
         [1, 1, 1]]
    nbh = M.convolve(state, S)
    return (nbh == 3) + (nbh == 2) * state


def life(state, generations):
    for _ in range(generations):
        state = life_step(state)
    return state


def life_initial(ds, bs, seed=16):
    """The reference script's initial state: rand(N, ds, U8, ROW+BLK, bs) > 128."""
    return M.rand(seed, ds, M.U8, M.ROW + M.BLK, bs) > 128


def stats(dem):
    """Returns the named scalar rasters of python/stats.py (evaluate with M.eval)."""
    N = M.prod(dem.datasize())
    maxv = M.zmax(dem)
    minv = M.zmin(dem)
    rang = maxv - minv
    mean = M.zsum(dem) / N
    geom = M.zprod(dem) ** (1.0 / N)
    harm = N / M.zsum(1.0 / dem)
    quam = M.sqrt(M.zsum(dem ** 2) / N)
    cubm = M.cbrt(M.zsum(dem ** 3) / N)
    dev = (dem - mean) ** 2
    var = M.zsum(dev) / N
    std = M.sqrt(var)
    norm = (dev - minv) / rang
    nstd = M.sqrt(M.zsum(norm) / N)
    return dict(maxv=maxv, minv=minv, rang=rang, mean=mean, geom=geom, harm=harm, quam=quam, cubm=cubm,
                std=std, nstd=nstd)


def wsum(layers, weights):
    """0 + w0*r0 + r1*w1 + ... + 0, as python/wsum.py writes it for four layers."""
    out = 0
    for i, (r, w) in enumerate(zip(layers, weights)):
        out = out + (w * r if i % 2 == 0 else r * w)
    return out + 0


def distance(raster, coord):
    x = coord[0] - M.index(raster, M.D1)
    y = coord[1] - M.index(raster, M.D2)
    return M.sqrt(x * x + y * y + 0.0)


def viewshed(dem, obs, h):
    shift = dem - h
    dist = distance(dem, obs)
    slope_ = shift / dist
    maxr = M.rmax(slope_, obs)
    return (maxr * dist + h) - dem
