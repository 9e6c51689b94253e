"""Generates the LBVH golden fixtures in this directory from the reference's
own CPU code (oracle/_ref/libehgp_ref.so: CanonicalPointCloud::rejecting_duplicates
+ MortonLbvhIndex::build, compiled from morsehgp3d/src/cpu against the
project-written Boost shim).  Run here, where the reference tree exists:

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "e-hgp_b200")]

from oracle import pyoracle  # noqa: E402
import workloads  # noqa: E402

TINY = np.nextafter(0.0, 1.0)
BIG = np.finfo(np.float64).max


def cases():
    yield "uniform256_s0", workloads.uniform_cube(256, 0)
    yield "uniform256_s1", workloads.uniform_cube(256, 1)
    yield "lattice5_f32", workloads.jittered_lattice(5, 3).astype(np.float64)
    # known-answer clouds of morsehgp3d/tests/unit/test_spatial_lbvh.cpp:641-744
    yield "collision4", np.array([[1, 1, 1], [2 * TINY, 0, 0], [0, 0, 0], [TINY, 0, 0]], float)
    yield "extrema4", np.array([[-BIG, -TINY, 0], [TINY, BIG, -BIG], [BIG, 0, TINY], [0, -BIG, BIG]], float)
    rng = np.random.Generator(np.random.PCG64(7))
    p = rng.random((600, 3))
    p[::3] = np.round(p[::3] * 7) / 7 + rng.random((200, 3)) * 1e-9  # many Morton collisions
    yield "collisions600", p
    q = rng.random((300, 3)) * 1e-300  # tiny exponents + a far point
    q[0] = [1e300, -1e300, 3.0]
    yield "spread300", q


def main():
    for name, pts in cases():
        r = pyoracle.lbvh_build(pts, "reference")
        np.savez_compressed(os.path.join(HERE, f"lbvh_{name}.npz"), points=pts,
                            **{k: r[k] for k in ("source_index", "leaves", "nodes", "counters", "root_aabb")},
                            root=np.uint64(r["root"]))
        print(name, len(pts), r["counters"])


if __name__ == "__main__":
    main()
