"""Staged edge tiles under the reference's block mirror (skeleton/common.cuh):
the staged box holds the raster mirror's value for every out-of-raster cell,
and block_exception names the cells whose taps differ from it; those cells are
recomputed through the border rule. Checked exhaustively on the CPU over many
raster, block and halo sizes: every cell with a differing tap is named (the
recomputation is then exact), and the named cells stay few."""
import itertools

import pytest


def reflect(i, d):
    """reflect_idx: invert(i, d) of runtime/skeleton/util.cpp:493, clamped."""
    r = -i - 1 if i < 0 else (d - (i - d + 1) if i >= d else i)
    return min(max(r, 0), d - 1)


def block_mirror(W, H, B0, B1, x, y, dx, dy):
    """focal_src with the block-mirror rule (the reading cell's block)."""
    nx, ny = x + dx, y + dy
    if 0 <= nx < W and 0 <= ny < H:
        return nx, ny
    bx0, by0 = (x // B0) * B0, (y // B1) * B1
    bw, bh = min(B0, W - bx0), min(B1, H - by0)
    return bx0 + reflect(nx - bx0, bw), by0 + reflect(ny - by0, bh)


def raster_mirror(W, H, x, y, dx, dy):
    """What stage_fix_border writes for an out-of-raster staged cell."""
    nx, ny = x + dx, y + dy
    if 0 <= nx < W and 0 <= ny < H:
        return nx, ny
    return reflect(nx, W), reflect(ny, H)


def block_exception(W, H, B0, B1, x, y, hx, hy):
    bx, by = x % B0, y % B1
    near_bx = bx < hx or bx >= B0 - hx or x >= W - hx
    near_by = by < hy or by >= B1 - hy or y >= H - hy
    edge_y = y < hy or y >= H - hy
    edge_x = x < hx or x >= W - hx
    lastx, lasty = (W - 1) // B0, (H - 1) // B1
    inner_last_x = x >= W - hx and (x // B0 != lastx or W - lastx * B0 < hx)
    inner_last_y = y >= H - hy and (y // B1 != lasty or H - lasty * B1 < hy)
    return (edge_y and near_bx) or (edge_x and near_by) or inner_last_x or inner_last_y


GEOMS = [(W, H, B0, B1, hx, hy)
         for (W, H) in [(64, 48), (65, 47), (100, 61), (33, 90), (49, 50), (97, 34)]
         for (B0, B1) in [(16, 16), (32, 8), (20, 12), (64, 48)]
         for (hx, hy) in [(1, 1), (2, 1), (1, 3), (3, 2)]
         if B0 > hx and B1 > hy]


@pytest.mark.parametrize("W,H,B0,B1,hx,hy", GEOMS)
def test_every_differing_cell_is_recomputed(W, H, B0, B1, hx, hy):
    named = 0
    for y in range(H):
        for x in range(W):
            exc = block_exception(W, H, B0, B1, x, y, hx, hy)
            named += exc
            if exc:
                continue
            for dx, dy in itertools.product(range(-hx, hx + 1), range(-hy, hy + 1)):
                assert block_mirror(W, H, B0, B1, x, y, dx, dy) == raster_mirror(W, H, x, y, dx, dy), (x, y, dx, dy)
    # the named cells lie along the raster's edges only
    assert named <= 2 * (hy * W + hx * H) + 4 * hx * hy
