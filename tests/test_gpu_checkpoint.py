"""Checkpoint and resume after the support stages (ehgp_checkpoint_save / _load).

A checkpoint written after the supports of a cloud, loaded into a fresh context, lets the
hierarchy run without enumerating the supports again (the context's counters show no pair
or triple/quad run) and gives the same records as the uninterrupted run.  A corrupted,
truncated or foreign file is refused and the loading context keeps no state of it."""
import numpy as np
import pytest

import ehgp
import workloads

pytestmark = pytest.mark.gpu

ARRAYS = ("events", "journal_batches", "roles", "families", "arm_removed", "nodes", "children", "births", "bindings",
          "saddles", "groups", "batches", "roots", "vertical")


def test_gpu_checkpoint_resumes_the_hierarchy(ctx, tmp_path):
    pts = workloads.uniform_cube(1500, 31)
    ctx.lbvh_build(pts, outputs=False)
    want = ctx.hierarchy(10)
    path = str(tmp_path / "cloud.ckp")
    ctx.checkpoint_save(path, 10)
    with ehgp.Context(max_points=4096) as c2:
        assert c2.checkpoint_load(path) == 10
        before = c2.counters()
        got = c2.hierarchy(10)
        after = c2.counters()
    assert (after["pair_runs"], after["higher_runs"]) == (before["pair_runs"], before["higher_runs"])
    for k in ARRAYS:
        assert np.array_equal(got[k], want[k]), k


def test_gpu_checkpoint_refuses_damaged_files(ctx, tmp_path):
    pts = workloads.jittered_lattice(8, 2)
    ctx.lbvh_build(pts, outputs=False)
    path = tmp_path / "good.ckp"
    ctx.checkpoint_save(str(path), 4)
    data = path.read_bytes()
    bad = {"flipped": data[:200] + bytes([data[200] ^ 1]) + data[201:], "truncated": data[:-7],
           "foreign": b"NOTACKPT" + data[8:], "longer": data + b"\0"}
    with ehgp.Context(max_points=4096) as c2:
        for name, blob in bad.items():
            p = tmp_path / f"{name}.ckp"
            p.write_bytes(blob)
            with pytest.raises(ehgp.InvalidArgument):
                c2.checkpoint_load(str(p))
        assert c2.checkpoint_load(str(path)) == 4
        c2.hierarchy(4)
