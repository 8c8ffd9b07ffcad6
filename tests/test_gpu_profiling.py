"""Stage timing (ao_tree_set_profiling / ao_tree_stage_times).

The CUDA-event counterpart of the reference's NVTX ranges behind
ADAPTIVE_OCTREE_PROFILING (config.hpp:20-28): with profiling on, build() and
update() record events at their stage boundaries and around every near-field
launch; calls under stream capture record nothing.
"""
import numpy as np
import pytest

from tests import scenarios as S
from tests.gpu_util import to_dev, tree_config

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_stage_times_of_build_and_update():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import adaptive_trees_b200 as ab
    xyz = S.plummer_sphere(200_000, seed=5, dtype=np.float32)
    xs = [to_dev(a) for a in xyz]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        t = ab.Tree(0, *xs, tree_config(bucket=512, nf=True, hilbert=True), stream=s)
        assert t.stageTimes() is None
        t.setProfiling(True)
        t.build()
        b = t.stageTimes()
        assert b is not None and b["call"] == "build"
        assert b["near_field_launches"] >= 1 and b["near_field_ms"] > 0
        parts = b["keys_and_sort_ms"] + b["refresh_ms"] + b["passes_ms"] + b["finish_ms"]
        assert b["refresh_ms"] < 0.05  # two back-to-back events: a build has no full refresh
        assert parts == pytest.approx(b["total_ms"], rel=1e-3, abs=1e-3)
        assert b["near_field_ms"] <= b["passes_ms"] + 1e-3

        t.update()
        u = t.stageTimes()
        assert u["call"] == "update"
        # the full refresh plus one launch per pass
        assert u["near_field_launches"] == 1 + 2  # octree default: 2 passes
        assert 0 < u["near_field_first_ms"] <= u["refresh_ms"]
        assert u["near_field_first_ms"] <= u["near_field_ms"] <= u["refresh_ms"] + u["passes_ms"] + 1e-3
        parts = u["keys_and_sort_ms"] + u["refresh_ms"] + u["passes_ms"] + u["finish_ms"]
        assert parts == pytest.approx(u["total_ms"], rel=1e-3, abs=1e-3)

        # under capture nothing is recorded, and replay works as without profiling
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            t.update()
        assert t.stageTimes() is None
        g.replay()
        s.synchronize()
        del g
        t.setProfiling(False)
        t.update()
        assert t.stageTimes() is None


def test_stage_times_without_near_field():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import adaptive_trees_b200 as ab
    xyz = S.uniform_cube(50_000, seed=2)
    t = ab.Tree(0, *[to_dev(a) for a in xyz], tree_config(bucket=16))
    t.setProfiling(True)
    t.build()
    t.update()
    u = t.stageTimes()
    assert u["near_field_launches"] == 0 and u["near_field_ms"] == 0.0
    assert u["total_ms"] > 0
