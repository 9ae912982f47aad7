"""The reference's numbering of a cuboid's cells (mb_reference_cell_order, the
Hilbert order of its octree that save_simulation_state's files and its state
vector follow) against the numbering read from the reference's own grid
builder (tests/golden/cell_order.npz, written by make_cell_order.py): the
active cells' order and the number of octree leaves, for small and ragged
cuboids whole and for the benchmark tissues' shapes by hash.  Host code only."""
import hashlib
import os

import numpy as np
import pytest

from monoalg3d_c_b200.monodomain import reference_cell_order

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "cell_order.npz"))
SMALL = sorted({k[len("order_"):] for k in GOLD.files if k.startswith("order_")})
LARGE = sorted({k[len("sha256_"):] for k in GOLD.files if k.startswith("sha256_")})


def _shape(key):
    return tuple(int(x) for x in key.split("x"))


@pytest.mark.parametrize("key", SMALL)
def test_small_cuboids(key):
    order, leaves = reference_cell_order(*_shape(key))
    np.testing.assert_array_equal(order, GOLD[f"order_{key}"])
    assert leaves == int(GOLD[f"leaves_{key}"])


@pytest.mark.parametrize("key", LARGE)
def test_benchmark_shapes(key):
    order, leaves = reference_cell_order(*_shape(key))
    assert leaves == int(GOLD[f"leaves_{key}"])
    assert order.size == int(GOLD[f"active_{key}"])
    assert hashlib.sha256(order.tobytes()).hexdigest() == GOLD[f"sha256_{key}"].item().decode()


def test_mask_keeps_the_order_of_the_remaining_cells():
    nx, ny, nz = 30, 20, 6
    full, leaves = reference_cell_order(nx, ny, nz)
    mask = (np.random.default_rng(5).random(nx * ny * nz) > 0.3).astype(np.uint8)
    order, leaves_m = reference_cell_order(nx, ny, nz, mask)
    np.testing.assert_array_equal(order, full[mask[full] == 1])
    assert leaves_m == leaves   # removed cells stay leaves of the octree


def test_bad_sizes_are_refused():
    with pytest.raises(Exception):
        reference_cell_order(0, 4, 4)
