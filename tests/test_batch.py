"""Packing of independent tissues into one atlas grid (mb_batch_pack, CPU):
every tissue inside the atlas, no two tissues overlapping or sharing a face,
and the batching configuration's 256 tissues packed at > 85 % occupancy."""
import numpy as np
import pytest


def _check(sizes):
    from monoalg3d_c_b200 import batch
    W, H, x0, y0 = batch.pack(sizes)
    owner = np.full((H, W), -1, dtype=np.int64)
    for q, (nx, ny) in enumerate(sizes):
        assert 1 <= x0[q] and x0[q] + nx <= W - 1 and 1 <= y0[q] and y0[q] + ny <= H - 1
        blk = owner[y0[q]:y0[q] + ny, x0[q]:x0[q] + nx]
        assert (blk == -1).all(), "tissues overlap"
        blk[...] = q
    # no face between cells of two different tissues
    for a, b in ((owner[:, 1:], owner[:, :-1]), (owner[1:, :], owner[:-1, :])):
        both = (a >= 0) & (b >= 0)
        assert (a[both] == b[both]).all(), "two tissues share a face"
    return W, H


def test_pack_random_sizes():
    rng = np.random.default_rng(4)
    sizes = [(int(rng.integers(1, 60)), int(rng.integers(1, 40))) for _ in range(70)]
    _check(sizes)


def test_pack_single_and_degenerate():
    assert _check([(5, 1)]) >= (7, 3)
    _check([(1, 1), (1, 1), (3, 1)])


def test_pack_rejects_bad_sizes():
    from monoalg3d_c_b200 import MonoAlgError, batch
    with pytest.raises(MonoAlgError):
        batch.pack([(0, 3)])


def test_batching_configuration_occupancy():
    from monoalg3d_c_b200 import workloads
    sizes, scales, kw = workloads.config2()
    assert len(sizes) == 256 and scales.shape == (256, 5)
    W, H = _check(sizes)
    assert sum(a * b for a, b in sizes) / (W * H) > 0.85
