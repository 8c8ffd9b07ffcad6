"""The converged octree build by levels against the reference's build rounds.

build() builds the converged tree one level of internal nodes at a time
(mode 0) and derives the leaf count of every round the reference would have
run from the same cells; mode 1 runs the rounds themselves (rebalanceBuild,
octree.cu:159-180).  Both must give the same keys, permutation, cornerstone,
counts, near-field counts, leaf capacity and round count, and an update after
either must agree too.  Mode 0 must fall back to the rounds where the rounds
stop before converging (a small max_depth).
"""
import numpy as np
import pytest

from tests import scenarios as S
from tests.gpu_util import NAMES, compare, gpu_get, oracle_config, to_dev, tree_config

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _stacked(n, seed):
    """Clusters of identical points in a sparse background (deep, narrow trees)."""
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 3))
    pts[: n // 4] = 0.3 + 1e-7 * rng.random(3)
    pts[n // 4: n // 3] = [0.71, 0.2, 0.55]
    return tuple(np.ascontiguousarray(pts[:, i]) for i in range(3))


CASES = [
    ("plummer_f32", lambda: S.plummer_sphere(150_000, seed=21, dtype=np.float32)),
    ("uniform_f64", lambda: S.uniform_cube(120_000, seed=22)),
    ("mixture_f64", lambda: S.gaussian_mixture(150_000, seed=23)),
    ("stacked_f64", lambda: _stacked(40_000, 24)),
]
CONFIGS = [
    dict(bucket=512, nf=True, hilbert=True),
    dict(bucket=64, nf=True, hilbert=False),
    dict(bucket=64, nf=False, hilbert=False),
    dict(bucket=16, nf=False, hilbert=True),
    dict(bucket=1, nf=True, hilbert=False),
]


def _build(xyz, mode, **cfg):
    """Mode 0 builds twice: the second build queues only the levels the first
    one needed (and must still come out whole)."""
    import adaptive_trees_b200 as ab
    xs = [to_dev(a) for a in xyz]
    t = ab.Tree(0, *xs, tree_config(**cfg))
    t.setBuildMode(mode)
    t.build()
    if mode == 0:
        t.build()
    return t, xs


def _same(a, b, nf):
    for name in NAMES:
        if name == "nearFieldCounts" and not nf:
            continue
        x, y = gpu_get(a, name), gpu_get(b, name)
        assert x.size == y.size, name
        bad = np.nonzero(x != y)[0]
        assert bad.size == 0, f"{name}: {bad.size} mismatches at {bad[:5]}"
    ia, ib = a.info(), b.info()
    assert ia.num_leaves == ib.num_leaves
    assert ia.leaf_capacity == ib.leaf_capacity, (ia.leaf_capacity, ib.leaf_capacity)
    assert a.buildPath()[1] == b.buildPath()[1], (a.buildPath(), b.buildPath())


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: f"b{c['bucket']}_{'nf' if c['nf'] else 'lc'}"
                                                      f"_{'hil' if c['hilbert'] else 'mor'}")
def test_levels_equal_rounds(case, cfg):
    xyz = case[1]()
    lv, xs_l = _build(xyz, 0, **cfg)
    rd, xs_r = _build(xyz, 1, **cfg)
    assert lv.buildPath()[0] is True
    assert rd.buildPath()[0] is False
    _same(lv, rd, cfg["nf"])
    # an update after either build
    moved = S.jitter(xyz, 2e-3, seed=5)
    for xs in (xs_l, xs_r):
        for d, a in zip(xs, moved):
            d.copy_(torch.from_numpy(np.ascontiguousarray(a)).to("cuda"))
    for t in (lv, rd):
        t.update()
        while t.doBuffersNeedResize():
            t.resizeBuffers()
            t.update()
    _same(lv, rd, cfg["nf"])
    lv.close()
    rd.close()


def test_levels_match_oracle_with_views():
    from oracle import oracle as O
    xyz = S.plummer_sphere(60_000, seed=31, dtype=np.float32)
    cfg = dict(bucket=256, nf=True, hilbert=True, views=(1, 1, 1))
    t, _ = _build(xyz, 0, **cfg)
    o = O.OracleTree(0, *xyz, oracle_config(**cfg))
    o.build()
    assert t.buildPath()[0]
    compare(t, o)
    t.close()


@pytest.mark.parametrize("max_depth", [1, 2, 3])
def test_round_limit_falls_back_to_rounds(max_depth):
    from oracle import oracle as O
    xyz = S.plummer_sphere(50_000, seed=32, dtype=np.float32)
    cfg = dict(bucket=64, nf=True, hilbert=False, max_depth=max_depth)
    t, _ = _build(xyz, 0, **cfg)
    o = O.OracleTree(0, *xyz, oracle_config(**cfg))
    o.build()
    compare(t, o)
    by_levels, rounds = t.buildPath()
    assert not by_levels and rounds == max_depth
    t.close()


@pytest.mark.parametrize("n", [1, 7, 600])
def test_small_trees(n):
    from oracle import oracle as O
    xyz = S.uniform_cube(n, seed=33)
    for cfg in (dict(bucket=4, nf=False), dict(bucket=4, nf=True, hilbert=True)):
        t, _ = _build(xyz, 0, **cfg)
        o = O.OracleTree(0, *xyz, oracle_config(**cfg))
        o.build()
        compare(t, o)
        t.close()


def test_escaped_particles_sort_last():
    from oracle import oracle as O
    x, y, z = S.uniform_cube(5_000, seed=34)
    x, y, z = x.copy(), y.copy(), z.copy()
    esc = np.finfo(np.float64).max
    for a in (x, y, z):
        a[::7] = esc
    cfg = dict(bucket=8, nf=True, hilbert=True)
    t, _ = _build((x, y, z), 0, **cfg)
    o = O.OracleTree(0, x, y, z, oracle_config(**cfg))
    o.build()
    assert t.buildPath()[0]
    compare(t, o)
    t.close()


@pytest.mark.parametrize("first,second", [("uniform", "stacked"), ("stacked", "uniform"), ("plummer", "mixture")])
@pytest.mark.parametrize("nf", [True, False])
def test_second_build_of_another_tree(first, second, nf):
    """The second build queues the levels the first tree needed; a tree of
    another shape (deeper, shallower, denser) must still come out equal to
    the rounds."""
    import adaptive_trees_b200 as ab
    gen = {"uniform": lambda: S.uniform_cube(60_000, seed=41), "stacked": lambda: _stacked(60_000, 42),
           "plummer": lambda: S.plummer_sphere(80_000, seed=43), "mixture": lambda: S.gaussian_mixture(80_000, seed=44)}
    a, b = gen[first](), gen[second]()
    cfg = dict(bucket=16, nf=nf, hilbert=True)
    trees = []
    for mode in (0, 1):  # the same two builds by levels and by rounds (leafCapacity keeps its history)
        xs = [to_dev(v) for v in a]
        t = ab.Tree(0, *xs, tree_config(**cfg))
        t.setBuildMode(mode)
        t.build()
        for d, v in zip(xs, b):
            d.copy_(torch.from_numpy(np.ascontiguousarray(v)).to("cuda"))
        t.build()
        trees.append(t)
    assert trees[0].buildPath()[0]
    _same(trees[0], trees[1], nf)
    for t in trees:
        t.close()


def test_deeper_tree_after_a_shallow_one():
    """The level build queues as many levels as the tree's last build needed;
    a deeper tree on the same object must still come out complete."""
    import adaptive_trees_b200 as ab
    from oracle import oracle as O
    shallow = S.uniform_cube(20_000, seed=35)
    deep = _stacked(20_000, 36)
    xs = [to_dev(a) for a in shallow]
    cfg = dict(bucket=32, nf=True, hilbert=True)
    t = ab.Tree(0, *xs, tree_config(**cfg))
    t.build()
    for d, a in zip(xs, deep):
        d.copy_(torch.from_numpy(np.ascontiguousarray(a)).to("cuda"))
    t.build()
    # the same two builds in the oracle: the second keeps the first's
    # buffer capacities, as the reference's vectors do
    o = O.OracleTree(0, *shallow, oracle_config(**cfg))
    o.build()
    o.set_coordinates(*deep)
    o.build()
    assert t.buildPath()[0]
    compare(t, o)
    t.close()


# ---------------------------------------------------------------------------
# binary (k-d) trees: the converged tree a depth at a time against the passes
# ---------------------------------------------------------------------------
BIN_CASES = [
    ("mixture_f64", lambda: S.gaussian_mixture(200_000, seed=51)),
    ("uniform_f64", lambda: S.uniform_cube(150_000, seed=52)),
    ("plummer_f32", lambda: S.plummer_sphere(150_000, seed=53, dtype=np.float32)),
    ("stacked_f64", lambda: _stacked(40_000, 54)),
]


def _binary(xyz, mode, builds=1, **cfg):
    import adaptive_trees_b200 as ab
    xs = [to_dev(a) for a in xyz]
    t = ab.Tree(1, *xs, tree_config(**cfg))
    t.setBuildMode(mode)
    for _ in range(builds):
        t.build()
    return t, xs


def _same_binary(a, b):
    for name in ("particleKeys", "perm", "cornerstone", "leafCounts"):
        x, y = gpu_get(a, name), gpu_get(b, name)
        assert x.size == y.size and np.array_equal(x, y), name
    ia, ib = a.info(), b.info()
    assert (ia.num_leaves, ia.num_nodes, ia.leaf_capacity, ia.max_achieved_depth) == \
        (ib.num_leaves, ib.num_nodes, ib.leaf_capacity, ib.max_achieved_depth)
    assert a.buildPath()[1] == b.buildPath()[1]
    assert a.doBuffersNeedResize() == b.doBuffersNeedResize()


@pytest.mark.parametrize("case", BIN_CASES, ids=[c[0] for c in BIN_CASES])
@pytest.mark.parametrize("bucket,max_depth", [(32, -1), (1, -1), (64, 12), (8, 5)])
def test_binary_levels_equal_passes(case, bucket, max_depth):
    xyz = case[1]()
    lv, xs_l = _binary(xyz, 0, builds=2, bucket=bucket, max_depth=max_depth)
    rd, xs_r = _binary(xyz, 1, builds=2, bucket=bucket, max_depth=max_depth)
    assert lv.buildPath()[0] and not rd.buildPath()[0]
    _same_binary(lv, rd)
    moved = S.jitter(xyz, 2e-3, seed=9)
    for xs in (xs_l, xs_r):
        for d, a in zip(xs, moved):
            d.copy_(torch.from_numpy(np.ascontiguousarray(a)).to("cuda"))
    for t in (lv, rd):
        t.update()
        while t.doBuffersNeedResize():
            t.resizeBuffers()
            t.update()
    _same_binary(lv, rd)
    lv.close()
    rd.close()


@pytest.mark.parametrize("n", [1, 7, 33, 600])
def test_binary_small_trees(n):
    xyz = S.uniform_cube(n, seed=55)
    lv, _ = _binary(xyz, 0, bucket=4)
    rd, _ = _binary(xyz, 1, bucket=4)
    _same_binary(lv, rd)
    lv.close()
    rd.close()


def test_binary_escaped_and_views():
    from oracle import oracle as O
    x, y, z = S.gaussian_mixture(30_000, seed=56)
    x, y, z = x.copy(), y.copy(), z.copy()
    esc = np.finfo(np.float64).max
    for a in (x, y, z):
        a[::9] = esc
    cfg = dict(bucket=16, views=(1, 1, 1))
    t, _ = _binary((x, y, z), 0, **cfg)
    o = O.OracleTree(1, x, y, z, oracle_config(**cfg))
    o.build()
    assert t.buildPath()[0]
    compare(t, o)
    t.close()
