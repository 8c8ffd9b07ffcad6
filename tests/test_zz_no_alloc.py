"""ao_sort_pairs_noalloc (fixed device scratch, no allocation) against ao_sort_pairs.

The file name sorts last, so in a full run it executes after every other test
in the same process; it also passes on its own.  Both sorts are called
through the C ABI.
"""
import ctypes

import numpy as np
import pytest

from adaptive_trees_b200 import _capi as C

MAX = C.SORT_PAIRS_NOALLOC_MAX_ITEMS


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def test_rejects_more_items_than_the_fixed_scratch():
    """Checked before any CUDA call, so this runs without a GPU."""
    lib = C.load()
    st = lib.ao_sort_pairs_noalloc(None, None, None, None, MAX + 1, 0, 64, None)
    assert st == 1  # AO_ERR_INVALID_ARGUMENT
    msg = lib.ao_last_error().decode()
    assert str(MAX) in msg and "ao_sort_pairs_noalloc" in msg


def _reference_sort(lib, keys, vals, n, begin, end, stream):
    import torch
    out_k = torch.empty_like(keys)
    out_v = torch.empty(n, dtype=torch.uint32, device=keys.device)
    nbytes = ctypes.c_size_t()
    C.check(lib.ao_sort_pairs(None, ctypes.byref(nbytes), None, None, None, None, n, begin, end, None))
    scratch = torch.empty(max(1, nbytes.value), dtype=torch.uint8, device=keys.device)
    C.check(lib.ao_sort_pairs(_p(scratch), ctypes.byref(nbytes), _p(keys), _p(out_k), _p(vals), _p(out_v), n,
                              begin, end, ctypes.c_void_p(stream.cuda_stream)))
    C.check(lib.ao_sort_pairs_check(_p(scratch), n, ctypes.c_void_p(stream.cuda_stream)))
    return out_k, out_v


@pytest.mark.gpu
def test_matches_ao_sort_pairs_on_two_calls_in_a_row():
    import torch
    lib = C.load()
    torch.cuda.set_device(0)
    s = torch.cuda.Stream()
    rng = np.random.default_rng(2024)
    cases = [(MAX, 0, 64, False), (777_777, 3, 45, True)]
    inputs = []
    for n, begin, end, with_values in cases:
        k = rng.integers(0, np.iinfo(np.uint64).max, size=n, dtype=np.uint64, endpoint=True)
        k[rng.integers(0, n, size=n // 4)] = k[rng.integers(0, n, size=n // 4)]  # duplicate keys: stability
        keys = torch.from_numpy(k.view(np.int64)).cuda().view(torch.uint64)
        vals = None
        if with_values:
            v = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
            vals = torch.from_numpy(v.view(np.int32)).cuda().view(torch.uint32)
        inputs.append((keys, vals))
    torch.cuda.synchronize()

    # both allocation-free calls back to back on one stream
    outs = []
    with torch.cuda.stream(s):
        for (n, begin, end, _), (keys, vals) in zip(cases, inputs):
            ok = torch.empty_like(keys)
            ov = torch.empty(n, dtype=torch.uint32, device="cuda")
            C.check(lib.ao_sort_pairs_noalloc(_p(keys), _p(ok), _p(vals), _p(ov), n, begin, end,
                                              ctypes.c_void_p(s.cuda_stream)))
            # no bounded look-back wait of this call gave up
            C.check(lib.ao_sort_pairs_noalloc_check(n, ctypes.c_void_p(s.cuda_stream)))
            outs.append((ok, ov))
        refs = [_reference_sort(lib, keys, vals, n, begin, end, s)
                for (n, begin, end, _), (keys, vals) in zip(cases, inputs)]
    s.synchronize()
    for (n, begin, end, _), (ok, ov), (rk, rv), (keys, vals) in zip(cases, outs, refs, inputs):
        assert torch.equal(ok.view(torch.int64), rk.view(torch.int64)), (n, begin, end)
        assert torch.equal(ov.view(torch.int32), rv.view(torch.int32)), (n, begin, end)
        # and against numpy's stable sort of the selected bits
        k = keys.view(torch.int64).cpu().numpy().view(np.uint64)
        mask = np.uint64((1 << (end - begin)) - 1) if end - begin < 64 else np.uint64(np.iinfo(np.uint64).max)
        order = np.argsort((k >> np.uint64(begin)) & mask, kind="stable")
        expect_v = order.astype(np.uint32) if vals is None else \
            vals.view(torch.int32).cpu().numpy().view(np.uint32)[order]
        assert np.array_equal(ok.view(torch.int64).cpu().numpy().view(np.uint64), k[order])
        assert np.array_equal(ov.view(torch.int32).cpu().numpy().view(np.uint32), expect_v)


@pytest.mark.gpu
def test_repeated_calls_leave_device_memory_unchanged():
    """After the set-up call, further calls do not change the device's free
    memory: full 64-bit sorts, sorts that carry given values, and sorts of an
    empty bit range (which copy the keys and write the identity permutation
    without a radix pass)."""
    import torch
    lib = C.load()
    torch.cuda.set_device(0)
    n = 300_000
    rng = np.random.default_rng(7)
    keys = torch.from_numpy(rng.integers(0, 2 ** 63, size=n, dtype=np.int64)).cuda().view(torch.uint64)
    vals = torch.from_numpy(rng.integers(0, 2 ** 31, size=n, dtype=np.int64).astype(np.int32)).cuda()
    vals = vals.view(torch.uint32)
    ok = torch.empty_like(keys)
    ov = torch.empty(n, dtype=torch.uint32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    C.check(lib.ao_sort_pairs_noalloc(_p(keys), _p(ok), None, _p(ov), n, 0, 64, stream))  # set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        C.check(lib.ao_sort_pairs_noalloc(_p(keys), _p(ok), _p(vals), _p(ov), n, 0, 64, stream))
        C.check(lib.ao_sort_pairs_noalloc(_p(keys), _p(ok), None, _p(ov), n, 17, 17, stream))
        C.check(lib.ao_sort_pairs_noalloc_check(n, stream))
        C.check(lib.ao_sort_pairs_noalloc(_p(keys), _p(ok), None, _p(ov), n, 0, 64, stream))
        C.check(lib.ao_sort_pairs_noalloc_check(n, stream))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    k = keys.view(torch.int64).cpu().numpy()
    assert np.array_equal(ok.view(torch.int64).cpu().numpy(), np.sort(k, kind="stable"))
    assert np.array_equal(ov.view(torch.int32).cpu().numpy(), np.argsort(k, kind="stable").astype(np.int32))
