"""Serving (Server / ao_serve_*): results alone and in the mix, admission, errors.

A request must give the same result whether it runs alone (one worker,
submitted after the previous request finished) or among many overlapping
requests (eight workers, everything submitted at once): the digest of the
tree's keys, permutation, cornerstone and counts after every build and
update is compared.
"""
import numpy as np
import pytest

from adaptive_trees_b200 import _capi as C

from .gpu_util import tree_config
from .scenarios import gaussian_mixture, plummer_sphere


def _coords(kind, n, seed, real):
    if kind == "plummer":
        return plummer_sphere(n, seed, dtype=real)
    if kind == "mixture":
        return gaussian_mixture(n, seed, dtype=real)
    rng = np.random.default_rng(seed)
    return tuple(rng.random(n).astype(real) for _ in range(3))


def _script():
    """(op, tree, payload) requests; payload = (coordinate key) for builds and updates."""
    f32, f64 = np.float32, np.float64
    trees = {
        0: (0, tree_config(bucket=64), "uniform", 20_000, f32),
        1: (0, tree_config(bucket=64, nf=True, hilbert=True), "plummer", 50_000, f32),
        2: (0, tree_config(bucket=16, hilbert=True), "mixture", 100_000, f64),
        3: (1, tree_config(bucket=32), "mixture", 30_000, f64),
        4: (0, tree_config(bucket=128, nf=True), "uniform", 8_000, f64),
        5: (0, tree_config(bucket=64), "plummer", 200_000, f32),
        6: (0, tree_config(bucket=64), "uniform", 50_000, f32),
    }
    ops = [("build", t, 0) for t in trees]
    ops += [("update", 0, 1), ("update", 1, 1), ("update", 2, 1), ("update", 3, 1), ("release", 4, None),
            ("update", 5, 1), ("update", 6, "cluster"), ("update", 0, 2), ("build", 4, 10), ("update", 1, 2),
            ("update", 4, 11), ("release", 0, None), ("release", 2, None), ("build", 2, 20), ("update", 5, 2),
            ("update", 3, 2), ("update", 2, 21), ("update", 6, 1), ("build", 0, 30), ("update", 0, 31)]
    return trees, ops


def _tensors(trees, ops):
    """Device coordinates of every (tree, version); versions > 0 are jittered copies."""
    import torch
    out = {}
    base = {}
    for op, t, v in ops:
        if op == "release":
            continue
        kind, cfg, dist, n, real = trees[t]
        if v == "cluster":
            rng = np.random.default_rng(11)
            xyz = tuple(np.clip(0.3 + 0.01 * rng.normal(size=n), 0, 0.999).astype(real) for _ in range(3))
        else:
            root = v - v % 10
            if (t, root) not in base:
                base[(t, root)] = _coords(dist, n, 1000 * t + root, real)
            xyz = base[(t, root)]
            if v % 10:
                rng = np.random.default_rng(7 * t + v)
                upper = np.nextafter(real(1.0), real(0.0))
                xyz = tuple(np.clip(a + rng.normal(0, 1e-3, n).astype(real), 0, upper).astype(real) for a in xyz)
        out[(t, v)] = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in xyz]
    return out


def _submit(server, trees, op, t, v, xyz):
    if op == "build":
        kind, cfg, _, _, _ = trees[t]
        return server.build(t, *xyz[(t, v)], config=cfg, kind=kind, digest=True)
    if op == "update":
        return server.update(t, *xyz[(t, v)], digest=True)
    return server.release(t)


@pytest.mark.gpu
def test_serve_results_alone_equal_results_in_the_mix():
    import torch

    import adaptive_trees_b200 as ab
    trees, ops = _script()
    xyz = _tensors(trees, ops)
    torch.cuda.synchronize()

    alone = ab.Server(slots=1)
    res_alone = []
    for op, t, v in ops:
        res_alone.append(alone.wait(_submit(alone, trees, op, t, v, xyz)))
    alone.close()

    mixed = ab.Server(slots=8)
    tickets = [_submit(mixed, trees, op, t, v, xyz) for op, t, v in ops]
    res_mixed = [mixed.wait(k) for k in tickets]
    stats = mixed.stats()
    mixed.close()

    for (op, t, v), a, m in zip(ops, res_alone, res_mixed):
        assert a["status"] == 0, (op, t, v, a["message"])
        assert m["status"] == 0, (op, t, v, m["message"])
        assert (a["digest"], a["num_leaves"], a["resizes"]) == (m["digest"], m["num_leaves"], m["resizes"]), \
            (op, t, v)
    cluster = ops.index(("update", 6, "cluster"))
    assert res_alone[cluster]["resizes"] > 0, "the clustered update must go through the resize retry"
    assert stats["completed"] == len(ops) and stats["failed"] == 0
    assert stats["p99_ms"] >= stats["p50_ms"] > 0

    # a served build is the plain tree's build
    kind, cfg, _, _, _ = trees[5]
    plain = ab.Tree(kind, *xyz[(5, 0)], cfg)
    plain.build()
    assert plain.info().num_leaves == res_alone[5]["num_leaves"]


@pytest.mark.gpu
def test_serve_admission_under_a_small_budget_and_errors():
    import torch

    import adaptive_trees_b200 as ab
    n = 1 << 20
    rng = np.random.default_rng(2)
    big = [[torch.from_numpy(rng.random(n, dtype=np.float32)).cuda() for _ in range(3)] for _ in range(3)]
    budget = 96 << 20  # room for one of these trees at a time (about 64 MB estimated, 71 MB held)
    s = ab.Server(slots=4, memory_budget_bytes=budget)
    cfg = tree_config(bucket=64)
    tickets = [s.build(0, *big[0], config=cfg), s.build(1, *big[1], config=cfg), s.release(0),
               s.build(2, *big[2], config=cfg), s.release(1), s.release(2)]
    results = [s.wait(k) for k in tickets]
    assert all(r["status"] == 0 for r in results), [r["message"] for r in results]
    st = s.stats()
    assert st["peak_bytes"] <= budget and st["resident_trees"] == 0

    huge = [torch.zeros(4 << 20, dtype=torch.float32, device="cuda") for _ in range(3)]
    r = s.wait(s.build(9, *huge, config=cfg))
    assert r["status"] == 3 and "budget" in r["message"]
    t0 = s.wait(s.build(5, *big[0], config=cfg))
    assert t0["status"] == 0
    assert s.wait(s.build(5, *big[1], config=cfg))["status"] == 1          # id already resident
    assert s.wait(s.update(77, *big[0]))["status"] == 1                      # no such tree
    assert s.wait(s.update(5, *[a[:1000] for a in big[0]]))["status"] == 1  # particle count changed
    assert s.wait(s.release(5))["status"] == 0
    s.close()


def test_serve_create_validates_arguments_without_a_gpu():
    import ctypes
    lib = C.load()
    h = ctypes.c_void_p()
    assert lib.ao_serve_create(0, 1 << 30, ctypes.byref(h)) == 1
    assert lib.ao_serve_create(4, 0, ctypes.byref(h)) == 1
