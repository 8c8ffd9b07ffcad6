"""Batched octrees (Batch / ao_batch_*) against one plain Tree per system.

Every system of a batch must hold exactly what a Tree built and updated on
that system alone holds: particleKeys_d, perm_d, cornerstone_d,
leafCounts_d, the active count, leafCapacity and needsResize, through build,
updates, and the resize-and-retry step of the systems that need it.
"""
import ctypes

import numpy as np
import pytest

from adaptive_trees_b200 import _capi as C

from .gpu_util import to_np, tree_config
from .scenarios import plummer_sphere


def _systems(rng, real, sizes):
    out = []
    for k, n in enumerate(sizes):
        if k % 3 == 2:
            x, y, z = plummer_sphere(n, int(rng.integers(1 << 30)), dtype=real)
        else:
            x, y, z = (rng.random(n).astype(real) for _ in range(3))
        if n > 10 and k % 4 == 1:
            x[: n // 10] = real(1.5)  # escaped: outside the box
        out.append((x, y, z))
    return out


def _compare(batch, trees, label):
    for s, t in enumerate(trees):
        for name in ("particleKeys_d", "perm_d", "cornerstone_d", "leafCounts_d"):
            a, b = to_np(batch.get(s, name)), to_np(t.get(name))
            assert a.shape == b.shape and np.array_equal(a, b), f"{label}: system {s} {name}"
        bi, ti = batch.info(s), t.info()
        assert bi.num_leaves == ti.num_leaves, f"{label}: system {s} leaves"
        assert bi.num_active_particles == ti.num_active_particles, f"{label}: system {s} active"
        assert bi.leaf_capacity == ti.leaf_capacity, f"{label}: system {s} leafCapacity"


def _flags(batch, trees):
    tree_flags = [t.doBuffersNeedResize() for t in trees]
    any_flag = batch.doBuffersNeedResize()
    batch_flags = [bool(batch.info(s).needs_resize) for s in range(len(trees))]
    assert batch_flags == tree_flags and any_flag == any(tree_flags)
    return tree_flags


@pytest.mark.gpu
# (n, sigma) of the system whose first update needs a resize, checked with the
# oracle for each configuration: built uniform, then compressed into a
# Gaussian cluster of width sigma, whose leaves split past the capacity
@pytest.mark.parametrize("real,hilbert,bucket,clustered", [(np.float32, False, 64, (50_000, 0.01)),
                                                           (np.float64, True, 16, (50_000, 0.01)),
                                                           (np.float32, True, 8, (100_000, 0.02))])
def test_batch_matches_single_trees(real, hilbert, bucket, clustered):
    import torch

    import adaptive_trees_b200 as ab
    rng = np.random.default_rng(17 + bucket)
    sizes = [0, 1, 7, 100, 4095, 4096, 4097, 20_000, 3_000, 150_000, 9_999, 60_000]
    host = _systems(rng, real, sizes)
    point = len(sizes)
    crng = np.random.default_rng(11)
    nc, sigma = clustered
    host.append(tuple(crng.random(nc).astype(real) for _ in range(3)))
    squeezed = tuple(np.clip(0.3 + sigma * crng.normal(size=nc), 0, 0.999).astype(real) for _ in range(3))
    dev = [[torch.from_numpy(a.copy()).cuda() for a in sysx] for sysx in host]
    cfg = tree_config(bucket=bucket, hilbert=hilbert)
    torch.cuda.synchronize()
    batch = ab.Batch([d[0] for d in dev], [d[1] for d in dev], [d[2] for d in dev], cfg)
    trees = [ab.Tree(0, *d, cfg) for d in dev]
    batch.build()
    for t in trees:
        t.build()
    _flags(batch, trees)
    _compare(batch, trees, "build")

    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    upper = float(np.nextafter(real(1.0), real(0.0)))
    for step in range(3):
        for s, d in enumerate(dev):
            if step == 0 and s == point:
                for t_, h in zip(d, squeezed):
                    t_.copy_(torch.from_numpy(h))
                continue
            for t_ in d:
                t_.add_(torch.randn(t_.shape, generator=gen, device="cuda", dtype=t_.dtype) * 1e-3)
                t_.clamp_(0.0, upper)
        batch.update()
        for t in trees:
            t.update()
        flags = _flags(batch, trees)
        _compare(batch, trees, f"update {step}")
        if step == 0:
            assert flags[point], "compressing the uniform system must exceed its capacity"
        rounds = 0
        while any(flags):
            rounds += 1
            assert rounds < 20
            for t, f in zip(trees, flags):
                if f:
                    t.resizeBuffers()
                    t.update()
            batch.resizeBuffers()
            batch.update(frozen=[not f for f in flags])
            flags = _flags(batch, trees)
            _compare(batch, trees, f"update {step} resize {rounds}")
    batch.close()


@pytest.mark.gpu
def test_batch_update_replays_from_a_graph():
    import torch

    import adaptive_trees_b200 as ab
    rng = np.random.default_rng(3)
    host = _systems(rng, np.float32, [5_000, 70_000, 1, 30_000])
    dev = [[torch.from_numpy(a.copy()).cuda() for a in sysx] for sysx in host]
    cfg = tree_config(bucket=32)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        batch = ab.Batch([d[0] for d in dev], [d[1] for d in dev], [d[2] for d in dev], cfg, stream=s)
        trees = [ab.Tree(0, *d, cfg, stream=s) for d in dev]
        batch.build()
        for t in trees:
            t.build()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            batch.update()
        gen = torch.Generator(device="cuda")
        gen.manual_seed(9)
        for _ in range(3):
            for d in dev:
                for t_ in d:
                    t_.add_(torch.randn(t_.shape, generator=gen, device="cuda") * 2e-3).clamp_(0.0, 0.99999994)
            g.replay()
            for t in trees:
                t.update()
            s.synchronize()
            assert not any(_flags(batch, trees))
            _compare(batch, trees, "graph replay")
        del g
    batch.close()


def test_batch_create_validates_arguments_without_a_gpu():
    lib = C.load()
    cfg = C.AoConfig()
    cfg.max_depth, cfg.max_particles_per_leaf, cfg.update_iterations = -1, 64, -1
    for i, v in enumerate((0, 1, 0, 1, 0, 1)):
        cfg.box[i] = v
    P = ctypes.c_void_p * 2
    counts = (ctypes.c_size_t * 2)(10, 0)
    h = ctypes.c_void_p()
    # null coordinates of a non-empty system
    st = lib.ao_batch_create(0, 2, P(None, None), P(None, None), P(None, None), counts, ctypes.byref(cfg), None,
                             ctypes.byref(h))
    assert st == 1 and "null" in lib.ao_last_error().decode()
    # NFCount is not batched
    cfg.split_criterion = 1
    st = lib.ao_batch_create(0, 2, P(1, None), P(1, None), P(1, None), counts, ctypes.byref(cfg), None,
                             ctypes.byref(h))
    assert st == 1 and "LeafCount" in lib.ao_last_error().decode()
    cfg.split_criterion = 0
    # no systems
    st = lib.ao_batch_create(0, 0, P(), P(), P(), counts, ctypes.byref(cfg), None, ctypes.byref(h))
    assert st == 1
