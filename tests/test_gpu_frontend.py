"""Python front end (e-hgp_b200/ehgp.py): CUDA arrays in place, `fit`, and cuts.

* `Context.lbvh_build_dlpack` reads a CUDA tensor (binary64 in place, binary32 widened on the
  device) or a DLPack capsule, and builds the same snapshot as the host path.
* `fit` from a CUDA tensor equals `fit` from the host array, array for array.
* `HierarchyResult.cut(k, a)` on the normative hgp_reduced definition forests: the exact node
  levels recovered from the level supports equal the definition's levels, and the cut at
  every level equals the cut of the definition forest under the same rule.
"""
import glob
import json
import os
from fractions import Fraction

import numpy as np
import pytest

import ehgp
import workloads

pytestmark = pytest.mark.gpu

SNAP = ("source_index", "leaves", "nodes", "counters", "root_aabb")


def test_gpu_dlpack_input_matches_host(ctx):
    import torch
    pts = workloads.uniform_cube(3000, 17)
    want = ctx.lbvh_build(pts)
    t = torch.from_numpy(pts).cuda()
    got = ctx.lbvh_build_dlpack(t, outputs=True)
    for k in SNAP:
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
    got = ctx.lbvh_build_dlpack(torch.utils.dlpack.to_dlpack(t), outputs=True)
    for k in SNAP:
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
    lat = workloads.jittered_lattice(10, 3)  # binary32
    want = ctx.lbvh_build(lat)
    got = ctx.lbvh_build_dlpack(torch.from_numpy(lat).cuda(), outputs=True)
    for k in SNAP:
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
    with pytest.raises(ehgp.InvalidArgument):
        ctx.lbvh_build_dlpack(torch.zeros((10, 2), dtype=torch.float64, device="cuda"))


def test_gpu_fit_from_tensor_equals_fit_from_host():
    import torch
    pts = workloads.mixture_cloud(1500, np.random.Generator(np.random.PCG64(8)))
    a = ehgp.fit(pts, K=10)
    b = ehgp.fit(torch.from_numpy(pts).cuda(), K=10)
    for k in ("nodes", "children", "batches", "roots", "vertical", "node_supports", "emst_u", "emst_v", "points"):
        assert np.array_equal(a[k], b[k]), k
    assert a["counts"]["final_roots"] == 10


DEFINITION = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "definition_*.json")))


def _definition_cut(forest, a):
    lev = [Fraction(int(nd[1]), int(nd[2])) for nd in forest["nodes"]]
    parent = {}
    for i, nd in enumerate(forest["nodes"]):
        for c in nd[3]:
            parent[c] = i
    return sorted(i for i, x in enumerate(lev) if x <= a and (i not in parent or lev[parent[i]] > a))


@pytest.mark.parametrize("path", DEFINITION, ids=[os.path.basename(p)[11:-5] for p in DEFINITION])
def test_gpu_cut_matches_definition(path):
    d = json.load(open(path))
    res = ehgp.fit(np.array(d["points"]), K=d["K"])
    nodes = res["nodes"]
    for f in d["forests"]:
        k = f["order"]
        idx = np.nonzero(nodes["order"] == k)[0]
        local = {int(g): i for i, g in enumerate(idx)}
        lev = res.node_levels(k)
        assert [lev[int(g)] for g in idx] == [Fraction(int(nd[1]), int(nd[2])) for nd in f["nodes"]]
        for a in sorted({Fraction(int(nd[1]), int(nd[2])) for nd in f["nodes"]}):
            got = [local[g] for g in res.cut(k, a)]
            assert got == _definition_cut(f, a), (k, a)
