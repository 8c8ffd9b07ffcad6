"""GPU parity of the CUDA path against the CPU oracle and the reference's golden vectors.

Every call goes through the C ABI (adaptive_trees_b200 -> libadaptive_trees_b200.so).
The bar is bit-exact equality of every integer output: keys, Perm, K, N, NF,
all view arrays, sizes, counters and the leaf capacity.
"""
import hashlib

import numpy as np
import pytest

from tests import scenarios as S
from tests.golden.make_golden import load_expected, load_snapshots
from tests.gpu_util import compare, gpu_get, oracle_config, to_dev, to_np, tree_config

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from adaptive_trees_b200 import _capi
    _capi.load()


def _ab():
    import adaptive_trees_b200 as ab
    return ab


def make_pair(O, kind, xyz, **cfg):
    ab = _ab()
    xs = [to_dev(a) for a in xyz]
    g = ab.Tree(kind, *xs, tree_config(**cfg))
    o = O.OracleTree(kind, *xyz, oracle_config(**cfg))
    return g, o, xs


def set_coords(g_xs, o, xyz):
    for t, a in zip(g_xs, xyz):
        t.copy_(torch.from_numpy(np.ascontiguousarray(a)).to("cuda"))
    torch.cuda.synchronize()
    o.set_coordinates(*xyz)


def update_both(g, o, max_resizes=64):
    g.update()
    o.update()
    k = 0
    while True:
        gn = g.doBuffersNeedResize()
        on = o.needs_resize()
        assert gn == on
        if not gn:
            break
        k += 1
        assert k < max_resizes
        g.resizeBuffers()
        o.resize_buffers()
        g.update()
        o.update()


# --------------------------------------------------------------------------
# golden regression (tree_test.cu:155-209)
# --------------------------------------------------------------------------
def test_golden_regression(oracle_mod):
    ab = _ab()
    (x0, y0, z0), (x1, y1, z1) = load_snapshots()
    xs = [to_dev(a) for a in (x0, y0, z0)]
    t = ab.Tree(0, *xs, tree_config(bucket=64 * 64 * 27, nf=True, views=(1, 1, 1)))
    t.build()
    for d, a in zip(xs, (x1, y1, z1)):
        d.copy_(torch.from_numpy(a).to("cuda"))
    t.update()
    k = 0
    while t.doBuffersNeedResize():
        k += 1
        assert k < 64
        t.resizeBuffers()
        t.update()
    meta, arrays = load_expected()
    names = {"particleKeys_d": "particleKeys", "perm_d": "perm", "cornerstone_d": "cornerstone",
             "sfcBoxIndex_d": "sfcBoxIndex", "particleBeginIndex_d": "particleBeginIndex",
             "particleCounts_d": "particleCounts", "hasBoxSplit_d": "hasBoxSplit", "boxDepth_d": "boxDepth",
             "parentIndex_d": "parentIndex", "childIndex_d": "childIndex", "sfcParticleIndex_d": "sfcParticleIndex",
             "levelOffset_d": "levelOffset"}
    for ref, ours in names.items():
        a = gpu_get(t, ours)
        spec = meta["arrays"][ref]
        assert a.size == spec["len"], ours
        if ref in arrays:
            bad = np.nonzero(a != arrays[ref])[0]
            assert bad.size == 0, f"{ours}: mismatches at {bad[:5]}"
        assert hashlib.sha256(a.tobytes()).hexdigest() == spec["sha256"], ours
    assert t.maxAchievedDepth() == meta["maxAchievedDepth"]


# --------------------------------------------------------------------------
# keys (computeSfcKeys) against the oracle
# --------------------------------------------------------------------------
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("box", [(0, 1, 0, 1, 0, 1), (0.1, 2.3, -1.0, 1.0, 0.5, 0.75), (-3, 5, -3, 5, -3, 5)])
def test_keys_match_oracle(oracle_mod, dtype, box):
    O = oracle_mod
    ab = _ab()
    rng = np.random.default_rng(11)
    n = 100_003
    lo, hi = np.array(box[0::2]), np.array(box[1::2])
    pts = lo + rng.random((n, 3)) * (hi - lo)
    pts[:50] = lo  # domain corners and edges
    pts[50:100] = hi
    pts[100:200] = np.finfo(dtype).max  # escaped
    xyz = tuple(np.ascontiguousarray(pts[:, i].astype(dtype)) for i in range(3))
    xs = [to_dev(a) for a in xyz]
    for hilbert in (False, True):
        got = to_np(ab.compute_sfc_keys(0, *xs, box=box, sfc_kind=int(hilbert)))
        exp = O.octree_keys(*xyz, box=box, hilbert=hilbert)
        bad = np.nonzero(got != exp)[0]
        assert bad.size == 0, (hilbert, bad[:5], got[bad[:5]], exp[bad[:5]])
    got = to_np(ab.compute_sfc_keys(1, *xs, box=box))
    exp = O.binary_keys(*xyz, box=box)
    assert np.array_equal(got, exp)
    # unaligned coordinate pointers take the scalar load path
    xs2 = [to_dev(np.concatenate([[dtype(0.5)], a]))[1:] for a in xyz]
    got = to_np(ab.compute_sfc_keys(0, *xs2, box=box, sfc_kind=1))
    assert np.array_equal(got, O.octree_keys(*xyz, box=box, hilbert=True))


# --------------------------------------------------------------------------
# octree build + updates vs oracle
# --------------------------------------------------------------------------
OCT_CASES = [
    # (name, generator, dtype, bucket, nf, hilbert, n)
    ("uniform-lc-morton-f64", "uniform", np.float64, 64, False, False, 60_000),
    ("uniform-lc-hilbert-f32", "uniform", np.float32, 16, False, True, 40_000),
    ("plummer-nf-hilbert-f32", "plummer", np.float32, 512, True, True, 60_000),
    ("plummer-nf-morton-f64", "plummer", np.float64, 512, True, False, 30_000),
    ("plummer-lc-morton-f32", "plummer", np.float32, 8, False, False, 50_000),
    ("uniform-nf-morton-f64", "uniform", np.float64, 64 * 64 * 27, True, False, 80_000),
]


def gen(kind, n, dtype, seed):
    if kind == "uniform":
        return S.uniform_cube(n, seed=seed, dtype=dtype)
    return S.plummer_sphere(n, seed=seed, dtype=dtype)


@pytest.mark.parametrize("case", OCT_CASES, ids=[c[0] for c in OCT_CASES])
def test_octree_build_update_matches_oracle(oracle_mod, case):
    O = oracle_mod
    name, dist, dtype, bucket, nf, hilbert, n = case
    xyz = gen(dist, n, dtype, seed=7)
    g, o, xs = make_pair(O, 0, xyz, bucket=bucket, nf=nf, hilbert=hilbert, views=(1, 1, 1))
    g.build()
    o.build()
    compare(g, o)
    for step in range(3):
        xyz = S.jitter(xyz, 2e-3, seed=100 + step)
        set_coords(xs, o, xyz)
        update_both(g, o)
        compare(g, o)


def test_octree_many_duplicate_keys_stable_perm(oracle_mod):
    """fp32 points on a coarse lattice: long runs of equal keys; Perm must ascend inside each run."""
    O = oracle_mod
    rng = np.random.default_rng(3)
    pts = (rng.integers(0, 40, size=(200_000, 3)) / 40.0).astype(np.float32)
    xyz = tuple(np.ascontiguousarray(pts[:, i]) for i in range(3))
    g, o, _ = make_pair(O, 0, xyz, bucket=4096, views=(1, 1, 1))
    g.build()
    o.build()
    compare(g, o)
    keys, perm = gpu_get(g, "particleKeys"), gpu_get(g, "perm")
    same = keys[1:] == keys[:-1]
    assert same.sum() > 100_000
    assert np.all(perm[1:][same] > perm[:-1][same])


def test_octree_capacity_resize_loop(oracle_mod):
    """Large displacement between updates forces capacity rejection and resizes."""
    O = oracle_mod
    xyz = S.uniform_cube(20_000, seed=4)
    g, o, xs = make_pair(O, 0, xyz, bucket=8, views=(1, 1, 1), iters=3)
    g.build()
    o.build()
    compare(g, o)
    rng = np.random.default_rng(5)
    clustered = tuple(np.ascontiguousarray(np.clip(0.3 + 0.01 * rng.normal(size=20_000), 0, 0.999999))
                      for _ in range(3))
    set_coords(xs, o, clustered)
    update_both(g, o)
    compare(g, o)
    set_coords(xs, o, xyz)
    update_both(g, o)
    compare(g, o)


@pytest.mark.parametrize("max_depth", [0, 1, 2, 5])
def test_octree_build_round_limit(oracle_mod, max_depth):
    """OctreeConfig::maxDepth caps the build rounds (octree.cu:164)."""
    O = oracle_mod
    xyz = S.plummer_sphere(30_000, seed=9, dtype=np.float64)
    g, o, _ = make_pair(O, 0, xyz, bucket=4, max_depth=max_depth, views=(1, 1, 1))
    g.build()
    o.build()
    compare(g, o)


# --------------------------------------------------------------------------
# escaped slots (tree_test.cu:411-504)
# --------------------------------------------------------------------------
@pytest.mark.parametrize("hilbert", [False, True])
@pytest.mark.parametrize("nf", [False, True])
@pytest.mark.parametrize("mask", [0, 0x08, 0xB7])
def test_escaped_slots_match_oracle(oracle_mod, hilbert, nf, mask):
    O = oracle_mod
    xyz = S.slot_coordinates(mask)
    g, o, _ = make_pair(O, 0, xyz, bucket=27 if nf else 1, iters=4, nf=nf, hilbert=hilbert, views=(1, 1, 1))
    g.build()
    o.build()
    assert not g.doBuffersNeedResize()
    compare(g, o)
    backing_p, n, cap, _ = g.buffer_info("sfcParticleIndex_d")
    assert cap >= 8


@pytest.mark.parametrize("hilbert", [False, True])
@pytest.mark.parametrize("nf", [False, True])
def test_graph_replay_matches_direct_through_escape_and_reactivation(oracle_mod, hilbert, nf):
    """One captured update() graph replayed across escape/reactivation equals direct updates."""
    O = oracle_mod
    ab = _ab()
    xyz = S.slot_coordinates(0xFF)
    xs = [to_dev(a) for a in xyz]
    s = torch.cuda.Stream()
    cfg = tree_config(bucket=27 if nf else 1, iters=4, nf=nf, hilbert=hilbert, views=(1, 1, 1))
    with torch.cuda.stream(s):
        direct = ab.Tree(0, *xs, cfg, stream=s)
        captured = ab.Tree(0, *xs, cfg, stream=s)
        direct.build()
        captured.build()
    o = O.OracleTree(0, *xyz, oracle_config(bucket=27 if nf else 1, iters=4, nf=nf, hilbert=hilbert, views=(1, 1, 1)))
    o.build()
    keys_ptr = captured.buffer_info("particleKeys_d")[0]
    map_ptr = captured.buffer_info("sfcParticleIndex_d")[0]
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        captured.update()
    for mask in (0xFF, 0xFF ^ 0x08, 0x91, 0, 0x04, 0xFF, 0, 0xFF):
        nxt = S.slot_coordinates(mask)
        with torch.cuda.stream(s):
            for t, a in zip(xs, nxt):
                t.copy_(torch.from_numpy(a).to("cuda"))
            direct.update()
            graph.replay()
        s.synchronize()
        o.set_coordinates(*nxt)
        o.update()
        assert not direct.doBuffersNeedResize()
        assert not captured.doBuffersNeedResize()
        assert not o.needs_resize()
        compare(direct, o)
        compare(captured, o)
        assert captured.buffer_info("particleKeys_d")[0] == keys_ptr
        assert captured.buffer_info("sfcParticleIndex_d")[0] == map_ptr
    del graph


# --------------------------------------------------------------------------
# binary k-d tree
# --------------------------------------------------------------------------
BIN_BOXES = [(0, 1, 0, 1, 0, 1), (-0.5, 0.5, 1, 2.25, -2, -0.25), (0, 1, 0, 1, 0, 64), (0, 1, 0, 1, 0, 2.0 ** 40)]


@pytest.mark.parametrize("box", BIN_BOXES)
def test_binary_lattice_matches_oracle(oracle_mod, box):
    O = oracle_mod
    pts = S.lattice_particles(box)
    pts[7] = S.escaped_point()
    g, o, _ = make_pair(O, 1, S.to_xyz(pts), bucket=3, box=box, views=(1, 1, 1))
    g.build()
    o.build()
    assert not g.doBuffersNeedResize()
    compare(g, o)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_binary_mixture_build_update_matches_oracle(oracle_mod, dtype):
    O = oracle_mod
    xyz = S.gaussian_mixture(80_000, seed=5, dtype=dtype)
    g, o, xs = make_pair(O, 1, xyz, bucket=32, views=(1, 1, 1))
    g.build()
    o.build()
    compare(g, o)
    for step in range(3):
        xyz = S.jitter(xyz, 5e-4, seed=200 + step)
        set_coords(xs, o, xyz)
        update_both(g, o)
        compare(g, o)


def test_binary_key_bits_and_depth(oracle_mod):
    O = oracle_mod
    box = (0, 1, 0, 1, 0, 2.0 ** 40)
    pts = [(0, 0, 0), (0, 0, 1), (0, 0, 2.0 ** 39)]
    for depth in (1, 63):
        g, o, _ = make_pair(O, 1, S.to_xyz(pts), bucket=1, box=box, max_depth=depth)
        g.build()
        o.build()
        compare(g, o)
        keys = gpu_get(g, "particleKeys")
        assert int(keys[1]) == 1 << 23 and int(keys[2]) == 1 << 62
        if depth == 63:
            assert g.maxAchievedDepth() == 40


@pytest.mark.parametrize("depth", [0, 1, 2, 63])
def test_binary_duplicate_depth_limit(oracle_mod, depth):
    O = oracle_mod
    pts = [(0.5, 0.5, 0.5)] * 3
    g, o, _ = make_pair(O, 1, S.to_xyz(pts), bucket=1, max_depth=depth, views=(1, 1, 1))
    g.build()
    o.build()
    compare(g, o)
    assert gpu_get(g, "leafCounts").size == depth + 1


def test_binary_domain_edges_and_escaped(oracle_mod):
    O = oracle_mod
    box = (0, 1, 0, 1, 0, 2.0 ** 80)
    pts = [(0, 0, 0), (1, 1, 2.0 ** 80), (-1, -1, -1), (2, 2, 2.0 ** 81), S.escaped_point()]
    g, o, _ = make_pair(O, 1, S.to_xyz(pts), bucket=3, max_depth=0, box=box, views=(1, 1, 1))
    g.build()
    o.build()
    compare(g, o)
    assert [int(k) for k in gpu_get(g, "particleKeys")] == [0, 0, S.ROOT_END - 1, S.ROOT_END - 1, (1 << 64) - 1]


@pytest.mark.parametrize("slots", [0, 9])
def test_binary_empty_and_escaped_inputs(oracle_mod, slots):
    O = oracle_mod
    pts = [S.escaped_point()] * slots
    xyz = S.to_xyz(pts) if slots else tuple(np.zeros(0) for _ in range(3))
    g, o, _ = make_pair(O, 1, xyz, bucket=3, views=(1, 1, 1))
    g.build()
    o.build()
    compare(g, o)
    for _ in range(3):
        update_both(g, o)
        compare(g, o)


def test_binary_graph_replay_with_resize(oracle_mod):
    """Captured binary updates equal direct ones through split, merge, resize and re-capture."""
    O = oracle_mod
    ab = _ab()
    box = (0, 1, 0, 1.25, 0, 1.75)
    empty = [S.escaped_point()] * 65
    xs = [to_dev(a) for a in S.to_xyz(empty)]
    s = torch.cuda.Stream()
    cfg = tree_config(bucket=1, max_depth=9, iters=2, box=box, views=(1, 1, 1))
    with torch.cuda.stream(s):
        direct = ab.Tree(1, *xs, cfg, stream=s)
        captured = ab.Tree(1, *xs, cfg, stream=s)
        direct.build()
        captured.build()
    o = O.OracleTree(1, *S.to_xyz(empty), oracle_config(bucket=1, max_depth=9, iters=2, box=box, views=(1, 1, 1)))
    o.build()

    def capture():
        gph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gph, stream=s):
            captured.update()
        return gph

    graph = capture()
    resized = False
    distributed = S.lattice_particles(box)
    partial = [S.escaped_point() if i % 3 == 0 else p for i, p in enumerate(distributed)]
    clustered = [(0.25, 0.25, 0.25)] * 65
    for pts in (distributed, partial, clustered, empty, distributed):
        xyz = S.to_xyz(pts)
        for _ in range(12):
            with torch.cuda.stream(s):
                for t, a in zip(xs, xyz):
                    t.copy_(torch.from_numpy(a).to("cuda"))
                direct.update()
                graph.replay()
            s.synchronize()
            o.set_coordinates(*xyz)
            o.update()
            gd, gc, go = direct.doBuffersNeedResize(), captured.doBuffersNeedResize(), o.needs_resize()
            assert gd == gc == go
            compare(direct, o)
            compare(captured, o)
            if gc:
                resized = True
                del graph
                direct.resizeBuffers()
                captured.resizeBuffers()
                o.resize_buffers()
                graph = capture()
    assert resized


def test_late_view_request_flags_resize(oracle_mod):
    """Views requested after a build without views set needsResize first (tree_view.cu:834-845)."""
    O = oracle_mod
    ab = _ab()
    for kind in (0, 1):
        pts = S.lattice_particles((0, 1, 0, 1, 0, 1), 31)
        pts[7] = S.escaped_point()
        g, o, _ = make_pair(O, kind, S.to_xyz(pts), bucket=3)
        g.build()
        o.build()
        compare(g, o)
        for views in ((1, 0, 0), (1, 1, 0), (1, 1, 1)):
            v = ab.ViewConfig(*[bool(x) for x in views])
            g.computeViews(v)
            o.compute_views(views)
            assert g.doBuffersNeedResize() == o.needs_resize()
            g.resizeBuffers()
            o.resize_buffers()
            g.computeViews(v)
            o.compute_views(views)
            assert not g.doBuffersNeedResize()
            assert not o.needs_resize()
            compare(g, o)


# --------------------------------------------------------------------------
# near-field counts on degenerate inputs
# --------------------------------------------------------------------------
@pytest.mark.parametrize("hilbert", [False, True])
@pytest.mark.parametrize("scene", ["stacked", "cluster-in-void"])
def test_near_field_degenerate_inputs_match_oracle(oracle_mod, hilbert, scene):
    """NFCount trees whose leaves stop at the deepest level with hundreds of equal keys
    (stacked points), or whose neighbour cells lie inside much coarser leaves (a tight
    cluster in a sparse background); build and two jittered updates."""
    O = oracle_mod
    rng = np.random.default_rng(17)
    if scene == "stacked":
        spots = rng.random((5, 3))
        stacked = spots[rng.integers(0, 5, size=20_000)]
        pts = np.concatenate([stacked, rng.random((30_000, 3))])
        bucket = 512
    else:
        cluster = np.clip(np.array([0.3, 0.6, 0.2]) + 1e-4 * rng.normal(size=(30_000, 3)), 0, 0.999999)
        pts = np.concatenate([cluster, rng.random((3_000, 3))])
        bucket = 64
    xyz = tuple(np.ascontiguousarray(pts[:, i]) for i in range(3))
    g, o, xs = make_pair(O, 0, xyz, bucket=bucket, nf=True, hilbert=hilbert, views=(1, 1, 1))
    g.build()
    o.build()
    compare(g, o)
    for step in range(2):
        moved = pts.copy()
        mask = rng.random(len(pts)) < 0.5  # half the points move, the rest keep their (stacked) keys
        moved[mask] = np.clip(moved[mask] + 1e-4 * rng.normal(size=(mask.sum(), 3)), 0, 0.999999)
        xyz = tuple(np.ascontiguousarray(moved[:, i]) for i in range(3))
        set_coords(xs, o, xyz)
        update_both(g, o)
        compare(g, o)
