"""The batch's converged build by levels (one persistent launch) against its
build rounds and against single trees.

Batch.build() in mode 0 builds every system's converged tree by levels in
one cooperative launch; mode 1 runs the reference's rounds over all systems
(rebalanceBuild, octree.cu:159-180).  Both must give every system the same
keys, permutation, cornerstone, counts, leaf capacity and needsResize, and
an update after either must agree too.  Mode 0 falls back to the rounds when
a system's rounds would stop at max_depth before converging.
"""
import numpy as np
import pytest

from .gpu_util import to_np, tree_config
from .scenarios import plummer_sphere

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


NAMES = ("particleKeys_d", "perm_d", "cornerstone_d", "leafCounts_d")


def _system(rng, k, n, real):
    kind = k % 4
    if kind == 0:
        x, y, z = (rng.random(n).astype(real) for _ in range(3))
    elif kind == 1:
        x, y, z = plummer_sphere(n, int(rng.integers(1 << 30)), dtype=real)
    elif kind == 2:
        # stacked points in a sparse background: deep, narrow subtrees
        x, y, z = (rng.random(n).astype(real) for _ in range(3))
        x[: n // 3], y[: n // 3], z[: n // 3] = real(0.3), real(0.6), real(0.2)
    else:
        x, y, z = (np.clip(0.5 + 0.01 * rng.normal(size=n), 0, 0.999).astype(real) for _ in range(3))
    if n > 20 and k % 5 == 3:
        x[: n // 7] = real(2.0)  # escaped: outside the box
    return x, y, z


def _batch(host, cfg, mode):
    import adaptive_trees_b200 as ab
    dev = [[torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in s] for s in host]
    b = ab.Batch([d[0] for d in dev], [d[1] for d in dev], [d[2] for d in dev], cfg)
    b.setBuildMode(mode)
    b.build()
    return b, dev


def _same(a, b, S, label):
    for s in range(S):
        for name in NAMES:
            x, y = to_np(a.get(s, name)), to_np(b.get(s, name))
            assert x.shape == y.shape and np.array_equal(x, y), f"{label}: system {s} {name}"
        ia, ib = a.info(s), b.info(s)
        assert (ia.num_leaves, ia.num_active_particles, ia.leaf_capacity, ia.needs_resize) == \
            (ib.num_leaves, ib.num_active_particles, ib.leaf_capacity, ib.needs_resize), f"{label}: system {s}"


@pytest.mark.parametrize("real,hilbert,bucket,S", [(np.float32, False, 64, 300),
                                                  (np.float64, True, 16, 40),
                                                  (np.float32, True, 1, 12),
                                                  (np.float64, False, 8, 700)])
def test_levels_equal_rounds(real, hilbert, bucket, S):
    rng = np.random.default_rng(100 + S)
    sizes = [0, 1, 2, 7, 65, 4096] + list(np.floor(10.0 ** rng.uniform(1.0, 4.7, S - 6)).astype(int))
    host = [_system(rng, k, int(n), real) for k, n in enumerate(sizes)]
    cfg = tree_config(bucket=bucket, hilbert=hilbert)
    lv, dl = _batch(host, cfg, 0)
    rd, dr = _batch(host, cfg, 1)
    assert lv.buildPath() and not rd.buildPath()
    assert lv.doBuffersNeedResize() == rd.doBuffersNeedResize()
    _same(lv, rd, S, "build")
    # a jittered update (with the resize-and-retry step) after either build
    jr = np.random.default_rng(7)
    for s in range(S):
        for i in range(3):
            a = host[s][i]
            if a.size:
                moved = np.clip(a + real(0.003) * jr.normal(size=a.size).astype(real), 0, 0.999).astype(real)
                moved[a > 1] = a[a > 1]
                dl[s][i].copy_(torch.from_numpy(moved))
                dr[s][i].copy_(torch.from_numpy(moved))
    for b in (lv, rd):
        b.update()
        for _ in range(16):
            if not b.doBuffersNeedResize():
                break
            b.resizeBuffers()
            b.update()
    _same(lv, rd, S, "update")
    lv.close()
    rd.close()


def test_levels_match_single_trees():
    import adaptive_trees_b200 as ab
    rng = np.random.default_rng(5)
    sizes = [0, 3, 500, 33_333, 120_000, 9]
    host = [_system(rng, k, n, np.float32) for k, n in enumerate(sizes)]
    cfg = tree_config(bucket=32, hilbert=True)
    b, dev = _batch(host, cfg, 0)
    assert b.buildPath()
    b.doBuffersNeedResize()
    for s, d in enumerate(dev):
        t = ab.Tree(0, *d, cfg)
        t.setBuildMode(1)  # the reference's rounds
        t.build()
        for name in NAMES:
            assert np.array_equal(to_np(b.get(s, name)), to_np(t.get(name))), f"system {s} {name}"
        assert b.info(s).leaf_capacity == t.info().leaf_capacity
        t.close()
    b.close()


@pytest.mark.parametrize("max_depth", [1, 2])
def test_round_limit_falls_back_to_rounds(max_depth):
    rng = np.random.default_rng(9)
    host = [_system(rng, k, n, np.float32) for k, n in enumerate([50_000, 10, 80_000])]
    cfg = tree_config(bucket=16, hilbert=False, max_depth=max_depth)
    lv, _ = _batch(host, cfg, 0)
    rd, _ = _batch(host, cfg, 1)
    assert not lv.buildPath()
    lv.doBuffersNeedResize()
    rd.doBuffersNeedResize()
    _same(lv, rd, len(host), "build")
    lv.close()
    rd.close()


def test_second_build_grows_buffers():
    """A deeper forest on the same batch: the arena and the leaf arrays grow
    (a relaunch of the level build), and the result still equals the rounds."""
    rng = np.random.default_rng(12)
    small = [_system(rng, 0, n, np.float32) for n in (1000, 2000, 500)]
    big = [_system(rng, 2, n, np.float32) for n in (1000, 2000, 500)]
    cfg = tree_config(bucket=2, hilbert=False)
    lv, dl = _batch(small, cfg, 0)
    rd, dr = _batch(small, cfg, 1)
    for s in range(3):
        for i in range(3):
            dl[s][i].copy_(torch.from_numpy(big[s][i]))
            dr[s][i].copy_(torch.from_numpy(big[s][i]))
    lv.build()
    rd.build()
    assert lv.buildPath()
    lv.doBuffersNeedResize()
    rd.doBuffersNeedResize()
    _same(lv, rd, 3, "second build")
    lv.close()
    rd.close()


def test_build_is_three_launches():
    """Keys, the persistent sort and the persistent level build: three kernel
    launches for the whole batch (after the first build has tuned the sort)."""
    import adaptive_trees_b200 as ab
    rng = np.random.default_rng(21)
    host = [_system(rng, k, n, np.float32) for k, n in enumerate([30_000, 5, 70_000, 0, 12_345])]
    cfg = tree_config(bucket=64, hilbert=False)
    b, dev = _batch(host, cfg, 0)
    probe = ab.Tree(0, *dev[0], cfg)  # the launch counter is process-wide
    b.build()
    torch.cuda.synchronize()
    before = probe.info().kernel_launches
    b.build()
    torch.cuda.synchronize()
    assert b.buildPath()
    assert probe.info().kernel_launches - before == 3
    rd, _ = _batch(host, cfg, 1)
    b.doBuffersNeedResize()
    rd.doBuffersNeedResize()
    _same(b, rd, len(host), "build")
    probe.close()
    b.close()
    rd.close()
