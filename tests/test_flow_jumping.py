"""The pointer-jumping flow accumulation (codegen.cpp gen_spread, _pj_* kernels)
replayed on the CPU: the Euler-tour successor function built from the 3 x 3 D8
codes around each cell, Wyllie's rounds with double buffers, and the final
subtraction, in NumPy with the kernels' int32 wrap-around arithmetic, against
the oracle's accumulation (oracle.c orc_flowacc_s32) on random acyclic direction
rasters with pits, invalid codes and codes that leave the raster."""
import numpy as np
import pytest

from oracle import oracle as O

DX = [1, 1, 0, -1, -1, -1, 0, 1]     # E, SE, S, SW, W, NW, N, NE
DY = [0, 1, 1, 1, 0, -1, -1, -1]
END = -1


def d8_index(c):
    c = int(c)
    if c == 0 or (c & (c - 1)) != 0:
        return -1
    return c.bit_length() - 1


def down(D, x, y):
    d = d8_index(D[y, x])
    if d < 0:
        return -1
    nx, ny = x + DX[d], y + DY[d]
    H, W = D.shape
    if not (0 <= nx < W and 0 <= ny < H):
        return -1
    return ny * W + nx


def child(D, x, y, j0):
    H, W = D.shape
    for j in range(j0, 8):
        nx, ny = x + DX[j], y + DY[j]
        if 0 <= nx < W and 0 <= ny < H and d8_index(D[ny, nx]) == ((j + 4) & 7):
            return ny * W + nx
    return -1


def after_up(D, x, y, d):
    H, W = D.shape
    px, py = x + DX[d], y + DY[d]
    sib = child(D, px, py, ((d + 4) & 7) + 1)
    if sib >= 0:
        return 2 * sib
    return 2 * (py * W + px) + 1 if down(D, px, py) >= 0 else END


def rounds(N):
    r = 1
    while (1 << r) <= 2 * N:
        r += 1
    return r


def jump(D, water):
    H, W = D.shape
    N = W * H
    nxt = np.full(2 * N, END, np.int64)
    sm = np.zeros(2 * N, np.int64)
    for c in range(N):
        x, y = c % W, c // W
        if down(D, x, y) >= 0:
            fc = child(D, x, y, 0)
            nxt[2 * c] = 2 * fc if fc >= 0 else 2 * c + 1
            nxt[2 * c + 1] = after_up(D, x, y, d8_index(D[y, x]))
            sm[2 * c] = water[y, x]
    R = rounds(N)
    for _ in range(R):                       # double-buffered: read old, write new
        live = nxt != END
        s2 = sm.copy()
        n2 = nxt.copy()
        s2[live] = sm[live] + sm[nxt[live]]
        n2[live] = nxt[nxt[live]]
        sm, nxt = s2 & 0xFFFFFFFF, n2          # u32 sums
    out = np.zeros((H, W), np.int64)
    for c in range(N):
        x, y = c % W, c // W
        if down(D, x, y) < 0:
            fc = child(D, x, y, 0)
            acc = sm[2 * fc] if fc >= 0 else 0
        else:
            assert nxt[2 * c] == END         # no cycle
            nu = after_up(D, x, y, d8_index(D[y, x]))
            acc = sm[2 * c] - (0 if nu == END else sm[nu]) - water[y, x]
        out[y, x] = acc & 0xFFFFFFFF
    return out.astype(np.uint32).view(np.int32)


@pytest.mark.parametrize("shape,seed", [((9, 13), 1), ((17, 11), 2), ((24, 24), 3), ((7, 40), 4)])
def test_jumping_equals_the_oracle(shape, seed):
    rng = np.random.default_rng(seed)
    # E, SE, S, SW never decrease y and E alone keeps it: acyclic
    codes = np.array([0, 1, 2, 4, 8, 1, 2, 4, 8, 3], np.uint8)
    D = codes[rng.integers(0, len(codes), shape)]
    water = rng.integers(-1000, 1000, shape).astype(np.int64)
    ref, cyclic = O.flowacc_s32(water.astype(np.int32), D)
    assert not cyclic
    assert np.array_equal(jump(D, water), ref)


def test_jumping_on_a_dem_drainage():
    from map_b200 import synth
    dem = synth.fbm_dem(20, 23, seed=9).astype(np.float64)
    H, W = dem.shape
    D = np.zeros((H, W), np.uint8)
    for y in range(H):                        # steepest strict descent, E..NE order
        for x in range(W):
            best, code = 0.0, 0
            for d in range(8):
                nx, ny = x + DX[d], y + DY[d]
                if 0 <= nx < W and 0 <= ny < H:
                    drop = (dem[y, x] - dem[ny, nx]) / (1.0 if d % 2 == 0 else 1.414213)
                    if drop > best:
                        best, code = drop, 1 << d
            D[y, x] = code
    water = np.ones((H, W), np.int64)
    ref, cyclic = O.flowacc_s32(water.astype(np.int32), D)
    assert not cyclic
    assert np.array_equal(jump(D, water), ref)
