"""The radix sort tuner (ao_sort_* in include/adaptive_trees_b200.h).

The engine's radix sort is compiled in a few configurations of digit width
and keys per thread.  The first tree or batch build of a size class on a
device times them all on its own keys and keeps the fastest; these calls
report and steer that choice.  Every configuration sorts identically.
"""
from __future__ import annotations

import ctypes

from . import _capi as C


def sort_configs() -> list[tuple[int, int]]:
    """(digit bits, keys per thread) of every compiled configuration, by index."""
    lib = C.load()
    n = ctypes.c_int()
    C.check(lib.ao_sort_config_count(ctypes.byref(n)))
    out = []
    for c in range(n.value):
        b, i = ctypes.c_int(), ctypes.c_int()
        C.check(lib.ao_sort_config_info(c, ctypes.byref(b), ctypes.byref(i)))
        out.append((b.value, i.value))
    return out


def sort_tuning(n: int, segmented: bool = False) -> dict:
    """The configuration the next sort of n keys uses on the current device."""
    c, b, i, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    C.check(C.load().ao_sort_tuning(int(segmented), int(n), ctypes.byref(c), ctypes.byref(b), ctypes.byref(i),
                                    ctypes.byref(t)))
    return {"config": c.value, "digit_bits": b.value, "items_per_thread": i.value, "tile": 256 * i.value,
            "tuned": bool(t.value)}


def set_sort_autotune(on: bool):
    """Off: untuned sizes use the default configuration, with no timing runs."""
    C.check(C.load().ao_sort_set_autotune(1 if on else 0))


def force_sort_config(config: int | None):
    """Every sort uses `config` (None lifts the force)."""
    C.check(C.load().ao_sort_force_config(-1 if config is None else int(config)))


def forget_sort_tuning():
    C.check(C.load().ao_sort_forget_tuning())
