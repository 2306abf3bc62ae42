"""The Local skeleton's 16-byte vector form (full tiles whose rows start on
16-byte boundaries load and store whole vectors; other tiles take the scalar
path): results equal NumPy restatements bit for bit for element sizes 1, 2, 4
and 8 bytes, with cell-index nodes (each lane keeps its own x), ragged raster
edges and device inputs whose pitch rules the vector form out."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.float32, np.float64])
@pytest.mark.parametrize("shape", [(64, 256), (97, 203), (32, 64), (200, 1030)])
def test_vector_local_matches_numpy(M, dtype, shape):
    rng = np.random.default_rng(7)
    h, w = shape
    if np.issubdtype(dtype, np.floating):
        a_np = rng.standard_normal(shape).astype(dtype)
        b_np = rng.standard_normal(shape).astype(dtype)
    else:
        a_np = rng.integers(0, 100, size=shape).astype(dtype)
        b_np = rng.integers(0, 100, size=shape).astype(dtype)
    a, b = M.from_numpy(a_np), M.from_numpy(b_np)
    got = M.to_numpy(a * b + a)
    assert np.array_equal(got, a_np * b_np + a_np)
    # each lane of a vector keeps its own column index
    xs = M.to_numpy(M.index(a, M.D1).astype(M._dt_of_np[np.dtype(dtype).name]) + b)
    want = (np.arange(w, dtype=np.int64)[None, :] + np.zeros((h, 1), np.int64)).astype(dtype) + b_np
    assert np.array_equal(xs, want)


def test_mixed_element_sizes_take_the_scalar_path(M):
    rng = np.random.default_rng(8)
    a_np = rng.standard_normal((70, 130)).astype(np.float32)
    k_np = rng.integers(0, 5, size=(70, 130)).astype(np.uint8)
    got = M.to_numpy(M.from_numpy(a_np) * M.from_numpy(k_np))
    assert np.array_equal(got, a_np * k_np.astype(np.float32))


def test_unaligned_device_pitch_takes_the_scalar_path(M):
    rng = np.random.default_rng(9)
    h, w = 96, 128
    base = torch.from_numpy(rng.standard_normal((h, w + 1)).astype(np.float32)).cuda()   # pitch 516 bytes
    torch.cuda.synchronize()   # the engine's stream does not wait for torch's
    a = M.from_device(base.data_ptr(), (w + 1) * 4, [w, h], M.F32)
    got = M.to_numpy(a * 3.0 + 1.0)
    ref = base[:, :w].cpu().numpy() * np.float32(3.0) + np.float32(1.0)
    assert np.array_equal(got, ref)
