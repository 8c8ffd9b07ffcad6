"""Opt-in convergence-checked update (ao_tree_update_until_converged).

The reference's update() runs a fixed number of passes (octree.cu:471-481,
kdtree3d.cu:259-270), which leaves overfull or mergeable leaves behind when
the particles move far between steps.  updateUntilConverged(M) passes until a
pass changes nothing, at most M.  Its tree must equal the oracle's update()
with update_iterations = M, bit for bit, through the same resize protocol; a
second call on unchanged coordinates must change nothing.
"""
import numpy as np
import pytest

from tests import scenarios as S
from tests.gpu_util import compare, oracle_config, to_dev, tree_config

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAX_PASSES = 48


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from adaptive_trees_b200 import _capi
    _capi.load()


def _converge_both(g, o, max_resizes=64):
    """The resize protocol around updateUntilConverged; returns the changed passes of each call."""
    changed = [g.updateUntilConverged(MAX_PASSES)]
    o.update()
    k = 0
    while True:
        gn = g.doBuffersNeedResize()
        assert gn == o.needs_resize()
        if not gn:
            return changed
        k += 1
        assert k < max_resizes
        g.resizeBuffers()
        o.resize_buffers()
        changed.append(g.updateUntilConverged(MAX_PASSES))
        o.update()


# (kind, bucket, nf, hilbert, dtype, default fixed pass count)
CASES = [
    (0, 16, False, False, np.float64, 2),
    (0, 16, False, True, np.float32, 2),
    (0, 256, True, True, np.float32, 2),
    (1, 16, False, False, np.float64, 6),
]


@pytest.mark.parametrize("case", CASES, ids=["oct-lc-morton", "oct-lc-hilbert", "oct-nf-hilbert", "binary"])
def test_update_until_converged_matches_oracle_with_max_passes(oracle_mod, case):
    O = oracle_mod
    kind, bucket, nf, hilbert, dtype, fixed = case
    n = 40_000
    xyz = S.plummer_sphere(n, seed=11, scale=0.02, centre=(0.3, 0.3, 0.3), dtype=dtype)
    cfg = dict(bucket=bucket, nf=nf, hilbert=hilbert, views=(1, 1, 1))
    import adaptive_trees_b200 as ab
    xs = [to_dev(a) for a in xyz]
    g = ab.Tree(kind, *xs, tree_config(**cfg))
    o = O.OracleTree(kind, *xyz, oracle_config(iters=MAX_PASSES, **cfg))
    g.build()
    o.build()
    compare(g, o)
    # the cluster jumps across the box and spreads out: far more than a
    # fixed pass count can follow
    far = S.plummer_sphere(n, seed=12, scale=0.08, centre=(0.7, 0.6, 0.65), dtype=dtype)
    for t, a in zip(xs, far):
        t.copy_(torch.from_numpy(np.ascontiguousarray(a)).to("cuda"))
    torch.cuda.synchronize()
    o.set_coordinates(*far)
    changed = _converge_both(g, o)
    compare(g, o)
    assert sum(changed) > fixed, changed  # the fixed policy would have stopped early
    assert changed[-1] < MAX_PASSES
    # converged: the same coordinates again change nothing
    before = {name: g.get(name + "_d").clone() for name in ("cornerstone", "leafCounts", "perm")}
    assert g.updateUntilConverged(MAX_PASSES) == 0
    assert not g.doBuffersNeedResize()
    for name, t in before.items():
        assert torch.equal(g.get(name + "_d"), t), name


def test_update_until_converged_equals_fixed_update_with_as_many_passes(oracle_mod):
    """The same tree as the library's own update() configured with M passes."""
    import adaptive_trees_b200 as ab
    xyz = S.gaussian_mixture(30_000, seed=21, dtype=np.float64)
    moved = S.gaussian_mixture(30_000, seed=22, dtype=np.float64)
    trees = []
    for iters in (-1, 12):
        xs = [to_dev(a) for a in xyz]
        t = ab.Tree(0, *xs, tree_config(bucket=32, iters=iters, views=(1, 1, 1)))
        t.build()
        for d, a in zip(xs, moved):
            d.copy_(torch.from_numpy(np.ascontiguousarray(a)).to("cuda"))
        torch.cuda.synchronize()
        trees.append((t, xs))
    (a, _), (b, _) = trees
    changed = a.updateUntilConverged(12)
    b.update()
    assert a.doBuffersNeedResize() == b.doBuffersNeedResize()
    assert 0 < changed <= 12
    for name in ("particleKeys", "perm", "cornerstone", "leafCounts", "sfcBoxIndex", "parentIndex"):
        assert torch.equal(a.get(name + "_d"), b.get(name + "_d")), name


def test_update_until_converged_rejects_bad_arguments():
    import adaptive_trees_b200 as ab
    xyz = S.uniform_cube(1000, seed=3)
    t = ab.Tree(0, *[to_dev(a) for a in xyz], tree_config(bucket=16))
    with pytest.raises(Exception):
        t.updateUntilConverged(1)  # before build()
    t.build()
    with pytest.raises(Exception):
        t.updateUntilConverged(0)
    assert t.updateUntilConverged(4) == 0


def test_batch_update_until_converged_matches_single_trees():
    """Every system of a batch equals a Tree updated until converged alone,
    through the resize-and-retry step of the systems that need it."""
    import adaptive_trees_b200 as ab

    from tests.gpu_util import to_np
    rng = np.random.default_rng(31)
    sizes = [1, 700, 5_000, 20_000, 60_000]
    host = [S.plummer_sphere(n, seed=40 + k, scale=0.01, centre=(0.25, 0.3, 0.35)) for k, n in enumerate(sizes)]
    moved = [S.plummer_sphere(n, seed=60 + k, scale=0.06 + 0.02 * k, centre=tuple(rng.uniform(0.4, 0.7, 3)))
             for k, n in enumerate(sizes)]
    dev = [[to_dev(a) for a in sysx] for sysx in host]
    cfg = tree_config(bucket=16, hilbert=True)
    batch = ab.Batch([d[0] for d in dev], [d[1] for d in dev], [d[2] for d in dev], cfg)
    trees = [ab.Tree(0, *d, cfg) for d in dev]
    batch.build()
    for t in trees:
        t.build()
    for d, m in zip(dev, moved):
        for t_, a in zip(d, m):
            t_.copy_(torch.from_numpy(np.ascontiguousarray(a)).to("cuda"))
    torch.cuda.synchronize()
    changed = batch.updateUntilConverged(MAX_PASSES)
    tree_changed = [t.updateUntilConverged(MAX_PASSES) for t in trees]
    assert changed == max(tree_changed) and changed > 2, (changed, tree_changed)
    for rounds in range(20):
        flags = [t.doBuffersNeedResize() for t in trees]
        assert batch.doBuffersNeedResize() == any(flags)
        assert [bool(batch.info(s).needs_resize) for s in range(len(trees))] == flags
        for s, t in enumerate(trees):
            for name in ("particleKeys_d", "perm_d", "cornerstone_d", "leafCounts_d"):
                assert np.array_equal(to_np(batch.get(s, name)), to_np(t.get(name))), (rounds, s, name)
            assert batch.info(s).leaf_capacity == t.info().leaf_capacity
        if not any(flags):
            break
        for t, f in zip(trees, flags):
            if f:
                t.resizeBuffers()
                t.updateUntilConverged(MAX_PASSES)
        batch.resizeBuffers()
        batch.updateUntilConverged(MAX_PASSES, frozen=[not f for f in flags])
    else:
        pytest.fail("resize loop did not settle")
    assert batch.updateUntilConverged(MAX_PASSES) == 0
    batch.close()
