"""The CPU oracle against the reference's own golden vectors and test cases.

These run without a GPU.  They pin the oracle (oracle/ao_oracle.cpp) before
it is trusted as the checker of the CUDA path:
  * the "[regression]" golden vectors (tree_test.cu:155-209), bit-exact;
  * escaped-slot invariants (tree_test.cu:411-458);
  * the binary physical-bisection oracle, known-answer keys, depth limits,
    empty inputs and config validation (tree_test.cu:780-1094).
"""
import hashlib

import numpy as np
import pytest

from tests import scenarios as S
from tests.golden.make_golden import load_expected, load_snapshots

NAMES = {
    "particleKeys": "particleKeys_d", "perm": "perm_d", "cornerstone": "cornerstone_d",
    "sfcBoxIndex": "sfcBoxIndex_d", "particleBeginIndex": "particleBeginIndex_d",
    "particleCounts": "particleCounts_d", "hasBoxSplit": "hasBoxSplit_d", "boxDepth": "boxDepth_d",
    "parentIndex": "parentIndex_d", "childIndex": "childIndex_d", "sfcParticleIndex": "sfcParticleIndex_d",
    "levelOffset": "levelOffset_d",
}


def check_against_golden(get, max_depth):
    meta, arrays = load_expected()
    for ours, ref in NAMES.items():
        a = get(ours)
        spec = meta["arrays"][ref]
        assert a.size == spec["len"], ours
        assert a.dtype == np.dtype(spec["dtype"]), ours
        if ref in arrays:
            exp = arrays[ref]
            bad = np.nonzero(a != exp)[0]
            assert bad.size == 0, f"{ours}: first mismatch at {bad[:5]}"
        assert hashlib.sha256(a.tobytes()).hexdigest() == spec["sha256"], ours
    assert max_depth == meta["maxAchievedDepth"]


def test_oracle_golden_regression(oracle_mod):
    O = oracle_mod
    (x0, y0, z0), (x1, y1, z1) = load_snapshots()
    cfg = O.make_config(max_particles_per_leaf=64 * 64 * 27, split_criterion=1, views=(1, 1, 1))
    t = O.OracleTree(0, x0, y0, z0, cfg)
    t.build()
    t.set_coordinates(x1, y1, z1)
    t.update()
    attempts = 0
    while t.needs_resize():
        attempts += 1
        assert attempts < 64
        t.resize_buffers()
        t.update()
    check_against_golden(t.get, t.info()["maxAchievedDepth"])


def _escaped_cfg(O, hilbert, nf):
    return O.make_config(max_particles_per_leaf=27 if nf else 1, update_iterations=4, split_criterion=int(nf),
                         sfc_kind=int(hilbert), views=(1, 1, 1))


def check_escaped_state(t, active_mask, slots=8):
    assert not t.needs_resize()
    info = t.info()
    active = bin(active_mask).count("1")
    assert info["numParticles"] == slots and info["numActiveParticles"] == active
    keys, perm = t.get("particleKeys"), t.get("perm")
    counts, begins = t.get("particleCounts"), t.get("particleBeginIndex")
    split, mapping, leaf_counts = t.get("hasBoxSplit"), t.get("sfcParticleIndex"), t.get("leafCounts")
    assert keys.size == slots and perm.size == slots and mapping.size == active
    assert counts.size == info["numNodes"] + 1
    assert counts[0] == active and counts[-1] == active
    assert int(leaf_counts.sum()) == active
    assert np.all(keys[:-1] <= keys[1:])
    seen = set()
    for p in range(slots):
        s = int(perm[p])
        assert s < slots and s not in seen
        seen.add(s)
        if p < active:
            assert active_mask & (1 << s)
            assert int(keys[p]) < S.ROOT_END
            node = int(mapping[p])
            assert node < info["numNodes"] and split[node] == 0
            assert begins[node] <= p < begins[node] + counts[node]
        else:
            assert not active_mask & (1 << s)
            assert int(keys[p]) == (1 << 64) - 1


TREE_ARRAYS = ["cornerstone", "leafCounts", "sfcBoxIndex", "particleCounts", "particleBeginIndex", "hasBoxSplit",
               "boxDepth", "parentIndex", "childIndex", "levelOffset", "sfcParticleIndex"]


@pytest.mark.parametrize("hilbert", [False, True])
@pytest.mark.parametrize("nf", [False, True])
@pytest.mark.parametrize("mask", [0, 0x08, 0xB7])
def test_oracle_escaped_slots(oracle_mod, hilbert, nf, mask):
    O = oracle_mod
    x, y, z = S.slot_coordinates(mask)
    cfg = _escaped_cfg(O, hilbert, nf)
    t = O.OracleTree(0, x, y, z, cfg)
    t.build()
    check_escaped_state(t, mask)
    active = bin(mask).count("1")
    if active <= 1:
        assert t.get("leafCounts").size == 1
        if nf:
            assert t.get("nearFieldCounts")[0] == 27 * active
    if mask == 0:
        return
    cx, cy, cz = S.slot_coordinates(mask, compact=True)
    ref = O.OracleTree(0, cx, cy, cz, cfg)
    ref.build()
    assert not ref.needs_resize()
    names = TREE_ARRAYS + (["nearFieldCounts"] if nf else [])
    for name in names:
        assert np.array_equal(t.get(name), ref.get(name)), name
    assert np.array_equal(t.get("particleKeys")[:active], ref.get("particleKeys"))
    ids = [s for s in range(8) if mask & (1 << s)]
    perm, rperm = t.get("perm"), ref.get("perm")
    for p in range(active):
        assert perm[p] == ids[rperm[p]]


def binary_cfg(O, box=(0, 1, 0, 1, 0, 1), bucket=3, depth=-1, views=(0, 0, 0), iters=-1):
    return O.make_config(max_depth=depth, max_particles_per_leaf=bucket, update_iterations=iters, box=box,
                         views=views)


def check_binary_oracle(t, points, box, bucket, max_depth, converged=True):
    """requireOracle (tree_test.cu:780-835) on a CPU model."""
    K, keys, counts, perm = t.get("cornerstone"), t.get("particleKeys"), t.get("leafCounts"), t.get("perm")
    active_pts = [p for p in points if p[0] != S.ESC64]
    assert K.size == counts.size + 1 and K[0] == 0 and int(K[-1]) == S.ROOT_END
    info = t.info()
    assert info["numParticles"] == len(points) and info["numActiveParticles"] == len(active_pts)
    assert int(counts.sum()) == len(active_pts)
    assert np.all(keys[:-1] <= keys[1:])
    assert sorted(perm.tolist()) == list(range(len(points)))
    for i in range(len(points)):
        assert int(keys[i]) == S.physical_key(points[int(perm[i])], box)
    for i in range(counts.size):
        b, e = int(K[i]), int(K[i + 1])
        w = e - b
        assert w > 0 and w & (w - 1) == 0 and b % w == 0
        assert counts[i] == np.searchsorted(keys, np.uint64(e)) - np.searchsorted(keys, np.uint64(b))
    if not converged:
        return
    exp = S.expected_binary_leaves(box, points, bucket, max_depth)
    assert counts.size == len(exp)
    for i, (c, cnt) in enumerate(exp):
        assert int(K[i]) == c.begin and int(K[i + 1]) == c.end and counts[i] == cnt


BOXES = [(0, 1, 0, 1, 0, 1), (-0.5, 0.5, 1, 2.25, -2, -0.25), (0, 1, 0, 1, 0, 64), (0, 1, 0, 1, 0, 2.0 ** 40)]


@pytest.mark.parametrize("box", BOXES)
def test_oracle_binary_physical_bisection(oracle_mod, box):
    O = oracle_mod
    pts = S.lattice_particles(box)
    pts[7] = S.escaped_point()
    t = O.OracleTree(1, *S.to_xyz(pts), binary_cfg(O, box=box, views=(1, 1, 1)))
    t.build()
    assert not t.needs_resize()
    check_binary_oracle(t, pts, box, 3, 63)


def test_oracle_binary_key_bits_follow_longest_side(oracle_mod):
    O = oracle_mod
    box = (0, 1, 0, 1, 0, 2.0 ** 40)
    pts = [(0, 0, 0), (0, 0, 1), (0, 0, 2.0 ** 39)]
    shallow = O.OracleTree(1, *S.to_xyz(pts), binary_cfg(O, box=box, bucket=1, depth=1))
    shallow.build()
    check_binary_oracle(shallow, pts, box, 1, 1)
    keys = shallow.get("particleKeys")
    assert int(keys[0]) == 0 and int(keys[1]) == 1 << 23 and int(keys[2]) == 1 << 62
    deep = O.OracleTree(1, *S.to_xyz(pts), binary_cfg(O, box=box, bucket=1, depth=63))
    deep.build()
    check_binary_oracle(deep, pts, box, 1, 63)
    assert deep.info()["maxAchievedDepth"] == 40
    assert np.array_equal(shallow.get("particleKeys"), deep.get("particleKeys"))


@pytest.mark.parametrize("depth", [0, 1, 2, 63])
def test_oracle_binary_depth_limits_duplicates(oracle_mod, depth):
    O = oracle_mod
    pts = [(0.5, 0.5, 0.5)] * 3
    t = O.OracleTree(1, *S.to_xyz(pts), binary_cfg(O, bucket=1, depth=depth, views=(1, 1, 1)))
    t.build()
    check_binary_oracle(t, pts, (0, 1, 0, 1, 0, 1), 1, depth)
    assert t.get("leafCounts").size == depth + 1


def test_oracle_binary_domain_edges(oracle_mod):
    O = oracle_mod
    box = (0, 1, 0, 1, 0, 2.0 ** 80)
    pts = [(0, 0, 0), (1, 1, 2.0 ** 80), (-1, -1, -1), (2, 2, 2.0 ** 81), S.escaped_point()]
    t = O.OracleTree(1, *S.to_xyz(pts), binary_cfg(O, box=box, depth=0, views=(1, 1, 1)))
    t.build()
    keys = t.get("particleKeys")
    assert [int(k) for k in keys] == [0, 0, S.ROOT_END - 1, S.ROOT_END - 1, (1 << 64) - 1]
    assert t.info()["numActiveParticles"] == 4
    assert t.get("leafCounts").tolist() == [4]


@pytest.mark.parametrize("slots", [0, 9])
def test_oracle_binary_empty_and_escaped(oracle_mod, slots):
    O = oracle_mod
    pts = [S.escaped_point()] * slots
    xyz = S.to_xyz(pts) if slots else tuple(np.zeros(0) for _ in range(3))
    t = O.OracleTree(1, *xyz, binary_cfg(O, views=(1, 1, 1)))
    t.build()
    check_binary_oracle(t, pts, (0, 1, 0, 1, 0, 1), 3, 63)
    for _ in range(3):
        t.update()
        assert not t.needs_resize()
        check_binary_oracle(t, pts, (0, 1, 0, 1, 0, 1), 3, 63)


def test_oracle_config_validation(oracle_mod):
    O = oracle_mod
    z = np.zeros(0)
    with pytest.raises(O.OracleError):
        O.OracleTree(1, z, z, z, binary_cfg(O, depth=64))
    with pytest.raises(O.OracleError):
        O.OracleTree(1, z, z, z, binary_cfg(O, box=(0, 0, 0, 1, 0, 1)))
    with pytest.raises(O.OracleError):
        O.OracleTree(1, z, z, z, O.make_config(split_criterion=1))
    with pytest.raises(O.OracleError):
        O.OracleTree(1, z, z, z, O.make_config(sfc_kind=1))
    with pytest.raises(O.OracleError):
        O.OracleTree(0, z, z, z, O.make_config(update_iterations=0))
    with pytest.raises(O.OracleError):
        O.OracleTree(0, z, z, z, O.make_config(max_particles_per_leaf=0))


def test_oracle_octree_leafcount_fixpoint(oracle_mod):
    """The converged LeafCount octree splits exactly the cells holding more than
    the bucket (cstone_check.cu:17-18 semantics), checked on a uniform cube."""
    O = oracle_mod
    x, y, z = S.uniform_cube(1 << 14, seed=5)
    t = O.OracleTree(0, x, y, z, O.make_config(max_particles_per_leaf=16))
    t.build()
    K, N, P = t.get("cornerstone"), t.get("leafCounts"), t.get("particleKeys")
    assert int(N.sum()) == x.size
    for i in range(N.size):
        b, e = int(K[i]), int(K[i + 1])
        assert N[i] <= 16
        w = e - b
        level = 21 - (w.bit_length() - 1) // 3
        if level > 0:
            parent_w = w << 3
            pb = b - b % parent_w
            cnt = np.searchsorted(P, np.uint64(pb + parent_w)) - np.searchsorted(P, np.uint64(pb))
            assert cnt > 16
