"""The packed byte-cell form of focal groups (four cells of a row as 16-bit
lanes, interior tiles) on the GPU: bit-identical to the one-cell form and to
the oracle, for Life under every border rule and on ragged rasters, for an
assortment of integer bodies on byte rasters (weighted correlations, relations,
selects, logical and bitwise operations, minimum / maximum, products), and for
outputs written to device buffers whose rows are not 4-byte aligned (those
tiles take the one-cell form)."""
import numpy as np
import pytest
import torch

from map_b200 import synth
from map_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def both_forms(M, build, arrays, bs):
    out = []
    for packed in (True, False):
        M.set_paired_cells(packed)
        rs = [M.from_numpy(a, bs=list(bs)) for a in arrays]
        r = build(*rs)
        assert ("focal_cell4(" in M.generated_source(r)) == packed
        out.append(M.to_numpy(r))
    M.set_paired_cells(True)
    return out


@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("shape,bs", [((512, 1024), (256, 256)), ((300, 517), (128, 128)), ((129, 131), (64, 64))])
def test_life_packed_equals_one_cell_and_oracle(fresh, border, shape, bs):
    M = fresh
    M.set_border(border)
    st = synth.bernoulli_u8(shape[0], shape[1], 0.3, seed=21)
    packed, single = both_forms(M, lambda s: W.life(s, 5), [st], bs)
    assert np.array_equal(packed, single)
    assert np.array_equal(packed, O.life(st, bs, 5, border))


BODIES = {
    "life": lambda a, b: W.life_step(a),
    "weighted": lambda a, b: M_.convolve(a, [[1, 2, 1], [2, 4, 2], [1, 2, 1]]) > 600,
    "select": lambda a, b: M_.con(M_.convolve(a, [[0, 1, 0], [1, 1, 1], [0, 1, 0]]) >= 300, a, b),
    "logic": lambda a, b: (M_.convolve(a, [[1, 1, 1], [1, 1, 1], [1, 1, 1]]) < 1000) * (b != 7) + (a <= b),
    "minmax": lambda a, b: (M_.max(M_.convolve(a, [[1, 0, 1], [0, 0, 0], [1, 0, 1]]), b * 3) + 255 - M_.min(a, b)) > 500,
    "bitwise": lambda a, b: ((M_.convolve(a, [[0, 0, 0], [1, 0, 1], [0, 0, 0]]).astype(M_.U16) & b.astype(M_.U16)) ^
                             (a.astype(M_.U16) | b.astype(M_.U16))) > 50,
    "wrap": lambda a, b: (M_.convolve(a, [[0, 1, 0], [1, 0, 1], [0, 1, 0]]) + b).astype(M_.U8),
    "product": lambda a, b: M_.min(M_.convolve(a, [[0, 0, 0], [0, 1, 0], [0, 0, 0]]), 127) * M_.min(b, 200) > 9000,
    "logical": lambda a, b: M_.con((a > 10) * (b < 200), M_.convolve(a, [[1, 1, 1], [1, 1, 1], [1, 1, 1]]) > 1100, a < 3),
}
M_ = None


@pytest.mark.parametrize("name", sorted(BODIES))
def test_integer_bodies_packed_equals_one_cell(fresh, name):
    global M_
    M = M_ = fresh
    rng = np.random.default_rng(31)
    a = rng.integers(0, 256, (260, 700), dtype=np.uint8)
    b = rng.integers(0, 256, (260, 700), dtype=np.uint8)
    build = BODIES[name]
    out = []
    for packed in (True, False):
        M.set_paired_cells(packed)
        r = build(M.from_numpy(a, bs=[128, 128]), M.from_numpy(b, bs=[128, 128]))
        out.append((M.to_numpy(r), "focal_cell4(" in M.generated_source(r)))
    M.set_paired_cells(True)
    assert out[0][0].dtype == out[1][0].dtype and np.array_equal(out[0][0], out[1][0])
    assert out[0][1] and not out[1][1]


def test_life_into_unaligned_device_rows(fresh):
    M = fresh
    st = synth.bernoulli_u8(256, 512, 0.35, seed=22)
    want = O.life(st, (256, 256), 1, 0)
    pitch = 512 + 3                                     # rows start at every byte offset mod 4
    buf = torch.zeros(256 * pitch + 1, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    r = W.life_step(M.from_numpy(st, bs=[256, 256]))
    assert "focal_cell4(" in M.generated_source(r)
    M.to_device(r, buf.data_ptr() + 1, pitch)
    got = buf[1:].reshape(256, pitch)[:, :512].cpu().numpy()
    assert np.array_equal(got, want)
