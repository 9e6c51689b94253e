"""The allocation-free LBVH entry point (ehgp_lbvh_build_noalloc).

It serves callers that may not call cudaMalloc, such as a host framework that
owns all device memory through its own pool, or a latency-critical caller that
cannot accept cudaMalloc's device-wide synchronisation.  It must give exactly
the result of the context-based entry point (ehgp_lbvh_build): the work is
integer and index work, so the tolerance is zero.  Two calls in a row on
different clouds show that the shared scratch array keeps no stale state
between calls.  This file is collected last on purpose, and it also passes
alone in a fresh process.
"""
import numpy as np
import pytest

import ehgp
import workloads

pytestmark = pytest.mark.gpu

FIELDS = ("source_index", "leaves", "nodes", "counters", "root_aabb")


def _collided(n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = rng.random((n, 3))
    pts[: n // 2] = np.round(pts[: n // 2] * 5) / 5 + rng.random((n // 2, 3)) * 1e-10
    return pts


def test_noalloc_matches_context_entry_point_two_calls_in_a_row():
    lib = ehgp.load()
    cap = int(lib.ehgp_lbvh_noalloc_max_points())
    assert cap == 16384
    clouds = [workloads.uniform_cube(cap, 21), _collided(5000, 22)]
    # the allocation-free calls first, so that in a fresh process the first
    # call also does the per-device set-up
    got = [ehgp.lbvh_build_noalloc(p) for p in clouds]
    with ehgp.Context(max_points=cap) as ctx:
        want = [ctx.lbvh_build(p) for p in clouds]
    for g, w in zip(got, want):
        for k in FIELDS:
            assert np.array_equal(getattr(g, k), getattr(w, k)), k
        assert g.root == w.root
    assert got[1].counters[3] > 0  # the second cloud exercises equal-code groups


def test_noalloc_rejects_sizes_and_bad_input():
    lib = ehgp.load()
    cap = int(lib.ehgp_lbvh_noalloc_max_points())
    with pytest.raises(ehgp.CapacityError):
        ehgp.lbvh_build_noalloc(workloads.uniform_cube(cap + 1, 1))
    with pytest.raises(ehgp.DuplicatePoint):
        ehgp.lbvh_build_noalloc(np.array([[0.0, 0, 0], [-0.0, 0, 0]]))
    # still correct after a rejected call
    p = workloads.uniform_cube(300, 2)
    with ehgp.Context(max_points=300) as ctx:
        w = ctx.lbvh_build(p)
    g = ehgp.lbvh_build_noalloc(p)
    for k in FIELDS:
        assert np.array_equal(getattr(g, k), getattr(w, k)), k
