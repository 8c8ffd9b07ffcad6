"""The engine's bounded device waits end with an error status, not a hang.

Each decoupled look-back (the radix sort's digit prefixes, the rebalance
decide+scan) polls earlier tiles a bounded number of times.  The self-test
entry point runs each look-back in the one situation where its wait cannot
end by itself -- the predecessor tile is never processed, so its status word
is never published -- under a small limit.  The kernel must record the error,
return, and leave the device usable: a pair sort and a tree build afterwards
still match their references.
"""
import ctypes

import numpy as np
import pytest

from adaptive_trees_b200 import _capi as C

from .gpu_util import compare, oracle_config, to_dev, to_np, tree_config
from .scenarios import plummer_sphere

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

AO_ERR_RUNTIME = 6
K_ERR_LOOKBACK = 1


@pytest.fixture(autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@pytest.mark.parametrize("which", [0, 1], ids=["radix_sort_pass", "decide_scan"])
def test_wait_that_cannot_end_gives_up_with_error_status(which):
    lib = C.load()
    code = ctypes.c_int(-1)
    st = lib.ao_selftest_bounded_wait(which, 256, ctypes.byref(code))
    assert st == AO_ERR_RUNTIME, lib.ao_last_error().decode()
    assert code.value == K_ERR_LOOKBACK
    assert "gave up" in lib.ao_last_error().decode()


def test_selftest_rejects_bad_arguments():
    lib = C.load()
    assert lib.ao_selftest_bounded_wait(2, 256, None) == 1
    assert lib.ao_selftest_bounded_wait(0, 0, None) == 1
    assert lib.ao_selftest_bounded_wait(0, 1 << 20, None) == 1


def test_device_usable_after_a_wait_gave_up():
    import adaptive_trees_b200 as ab
    from oracle import oracle as O
    lib = C.load()
    for which in (0, 1):
        assert lib.ao_selftest_bounded_wait(which, 64, None) == AO_ERR_RUNTIME
    # a pair sort: sorted like numpy's stable sort, and its own check passes
    rng = np.random.default_rng(11)
    n = 200_003
    k = rng.integers(0, np.iinfo(np.uint64).max, size=n, dtype=np.uint64, endpoint=True)
    keys = torch.from_numpy(k.view(np.int64)).cuda().view(torch.uint64)
    ok = torch.empty_like(keys)
    ov = torch.empty(n, dtype=torch.uint32, device="cuda")
    nbytes = ctypes.c_size_t()
    C.check(lib.ao_sort_pairs(None, ctypes.byref(nbytes), None, None, None, None, n, 0, 64, None))
    scratch = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
    C.check(lib.ao_sort_pairs(_p(scratch), ctypes.byref(nbytes), _p(keys), _p(ok), None, _p(ov), n, 0, 64, None))
    C.check(lib.ao_sort_pairs_check(_p(scratch), n, None))
    order = np.argsort(k, kind="stable")
    assert np.array_equal(to_np(ok), k[order])
    assert np.array_equal(to_np(ov), order.astype(np.uint32))
    # a tree build and update: bit-exact with the oracle
    xyz = plummer_sphere(30_000, seed=12, dtype=np.float32)
    cfg = dict(bucket=64, hilbert=True)
    t = ab.Tree(0, *[to_dev(a) for a in xyz], tree_config(**cfg))
    o = O.OracleTree(0, *xyz, oracle_config(**cfg))
    t.build()
    o.build()
    compare(t, o)
    t.close()
