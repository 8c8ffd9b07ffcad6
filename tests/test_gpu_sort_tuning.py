"""The sort tuner: every compiled radix sort configuration sorts identically.

The engine's radix sort is compiled for several digit widths and keys per
thread, and the tuner picks one per device and size class by timing them on
the first build.  The trees must not depend on that choice: for each forced
configuration, ao_sort_pairs must equal a stable numpy sort, and the keys,
permutation and cornerstone of an octree and of a batch must equal those of
the default configuration.  Tuning must record a choice and keep the trees
unchanged.
"""
import ctypes

import numpy as np
import pytest

from adaptive_trees_b200 import _capi as C

from .gpu_util import to_np, tree_config
from .scenarios import plummer_sphere

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _restore_tuner():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import adaptive_trees_b200 as ab
    yield
    ab.force_sort_config(None)
    ab.set_sort_autotune(True)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _pair_sort(keys, vals, n, begin, end):
    lib = C.load()
    out_k = torch.empty_like(keys)
    out_v = torch.empty(n, dtype=torch.uint32, device="cuda")
    nbytes = ctypes.c_size_t()
    C.check(lib.ao_sort_pairs(None, ctypes.byref(nbytes), None, None, None, None, n, begin, end, None))
    scratch = torch.empty(max(1, nbytes.value), dtype=torch.uint8, device="cuda")
    C.check(lib.ao_sort_pairs(_p(scratch), ctypes.byref(nbytes), _p(keys), _p(out_k), _p(vals), _p(out_v), n, begin,
                              end, None))
    torch.cuda.synchronize()
    return to_np(out_k), to_np(out_v)


def test_every_configuration_sorts_pairs_like_a_stable_sort():
    import adaptive_trees_b200 as ab
    rng = np.random.default_rng(7)
    configs = ab.sort_configs()
    assert len(configs) >= 4 and {b for b, _ in configs} == {7, 8}
    for n, begin, end, with_values in [(1, 0, 64, False), (2047, 0, 64, True), (100_003, 0, 64, False),
                                       (300_000, 5, 50, True), (1 << 20, 0, 64, True)]:
        k = rng.integers(0, np.iinfo(np.uint64).max, size=n, dtype=np.uint64, endpoint=True)
        k[rng.integers(0, n, size=n // 3)] = k[rng.integers(0, n, size=n // 3)]  # runs of equal keys
        keys = torch.from_numpy(k.view(np.int64)).cuda().view(torch.uint64)
        v = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
        vals = torch.from_numpy(v.view(np.int32)).cuda().view(torch.uint32) if with_values else None
        mask = np.uint64(((1 << (end - begin)) - 1) << begin) if end - begin < 64 else np.uint64(~np.uint64(0))
        order = np.argsort((k & mask) >> np.uint64(begin), kind="stable")
        want_v = v[order] if with_values else order.astype(np.uint32)
        for c in range(len(configs)):
            ab.force_sort_config(c)
            got_k, got_v = _pair_sort(keys, vals, n, begin, end)
            assert np.array_equal(got_k, k[order]), (n, c)
            assert np.array_equal(got_v, want_v), (n, c)


def test_trees_and_batches_do_not_depend_on_the_configuration():
    import adaptive_trees_b200 as ab
    xyz = plummer_sphere(150_000, 9, dtype=np.float32)
    moved = np.clip(xyz[0] + np.random.default_rng(8).normal(0, 1e-3, xyz[0].size), 0, 0.99999994).astype(np.float32)
    rng = np.random.default_rng(5)
    sizes = [1, 3000, 70_000, 12_345, 0, 250_000]
    host = [tuple(rng.random(n).astype(np.float32) for _ in range(3)) for n in sizes]
    dev = [[torch.from_numpy(a).cuda() for a in h] for h in host]
    want = None
    for c in range(len(ab.sort_configs())):
        ab.force_sort_config(c)
        xs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in xyz]
        t = ab.Tree(0, *xs, tree_config(bucket=512, nf=True, hilbert=True))
        t.build()
        xs[0].copy_(torch.from_numpy(moved))
        torch.cuda.synchronize()
        t.update()
        t.doBuffersNeedResize()
        b = ab.Batch([d[0] for d in dev], [d[1] for d in dev], [d[2] for d in dev], tree_config(bucket=32))
        b.build()
        got = [to_np(t.get(name)) for name in ("particleKeys_d", "perm_d", "cornerstone_d", "nearFieldCounts_d")]
        for s in range(len(sizes)):
            got += [to_np(b.get(s, name)) for name in ("particleKeys_d", "perm_d", "cornerstone_d")]
        b.close()
        if want is None:
            want = got
        else:
            for a, e in zip(got, want):
                assert np.array_equal(a, e), c


def test_first_build_tunes_and_later_builds_reuse_the_choice():
    import adaptive_trees_b200 as ab
    ab.force_sort_config(None)
    ab.set_sort_autotune(False)
    n = 300_001
    xyz = plummer_sphere(n, 3, dtype=np.float32)
    xs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in xyz]
    t = ab.Tree(0, *xs, tree_config(bucket=64))
    t.build()
    plain = [to_np(t.get(name)) for name in ("particleKeys_d", "perm_d", "cornerstone_d")]
    assert not ab.sort_tuning(n)["tuned"]

    ab.forget_sort_tuning()
    ab.set_sort_autotune(True)
    t2 = ab.Tree(0, *xs, tree_config(bucket=64))
    t2.build()
    choice = ab.sort_tuning(n)
    assert choice["tuned"] and 0 <= choice["config"] < len(ab.sort_configs())
    assert ab.sort_tuning(n + 1000)["config"] == choice["config"]  # same size class
    for a, e in zip([to_np(t2.get(name)) for name in ("particleKeys_d", "perm_d", "cornerstone_d")], plain):
        assert np.array_equal(a, e)
    t2.build()  # no second tuning: the choice stands
    assert ab.sort_tuning(n) == choice

    # a batch tunes its own (segmented) entry
    host = [tuple(np.random.default_rng(k).random(m).astype(np.float32) for _ in range(3))
            for k, m in enumerate([5000, 90_000, 1])]
    dev = [[torch.from_numpy(a).cuda() for a in h] for h in host]
    b = ab.Batch([d[0] for d in dev], [d[1] for d in dev], [d[2] for d in dev], tree_config(bucket=32))
    b.build()
    assert ab.sort_tuning(95_001, segmented=True)["tuned"]
    b.close()
