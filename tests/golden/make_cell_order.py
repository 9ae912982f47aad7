"""Writes tests/golden/cell_order.npz: the reference's numbering of the active
cells of several cuboids (grid indices in the order of its octree's leaves,
which save_simulation_state and the reference's state vector follow) and the
number of leaves, read from the reference's own grid builder through
oracle/ref/hilbert_probe.c (built by `make -C oracle/ref`).  Small cuboids are
stored whole; the benchmark tissues' shapes as a SHA-256 of the int64 order.

    python tests/golden/make_cell_order.py
"""
import hashlib
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PROBE = os.path.join(HERE, "..", "..", "oracle", "_ref", "bin", "hilbert_probe")
SMALL = [(1, 1, 1), (2, 2, 2), (3, 1, 1), (5, 3, 2), (7, 9, 13), (17, 4, 3), (30, 20, 6), (32, 8, 2), (33, 2, 1)]
LARGE = [(100, 100, 20), (200, 200, 50), (500, 500, 100)]


def probe(nx, ny, nz):
    """(active order as grid indices, number of leaves)."""
    p = subprocess.Popen([PROBE, "cuboid", str(nx), str(ny), str(nz)], stdout=subprocess.PIPE, text=True)
    order, leaves = [], 0
    for line in p.stdout:
        f = line.split()
        if len(f) != 4 or not all(x.lstrip("-").isdigit() for x in f):
            continue
        leaves += 1
        i, j, k, a = map(int, f)
        if a:
            order.append(i + nx * (j + ny * k))
    assert p.wait() == 0
    return np.asarray(order, dtype=np.int64), leaves


def main():
    out = {}
    for s in SMALL:
        o, n = probe(*s)
        key = "x".join(map(str, s))
        out[f"order_{key}"] = o
        out[f"leaves_{key}"] = np.int64(n)
    for s in LARGE:
        o, n = probe(*s)
        key = "x".join(map(str, s))
        out[f"sha256_{key}"] = np.bytes_(hashlib.sha256(o.tobytes()).hexdigest())
        out[f"leaves_{key}"] = np.int64(n)
        out[f"active_{key}"] = np.int64(o.size)
        print(key, n, o.size)
    np.savez_compressed(os.path.join(HERE, "cell_order.npz"), **out)


if __name__ == "__main__":
    main()
