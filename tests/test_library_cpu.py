"""CPU checks of the product library: it builds for sm_100a, loads without a GPU,
and exports every entry point the C header declares."""
import ctypes
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "adaptive_trees_b200.h")


@pytest.fixture(scope="module")
def lib():
    from adaptive_trees_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ao_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "ao_tree_create" in syms and "ao_tree_update" in syms and len(syms) >= 12


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_library_exports_nothing_else(lib):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "adaptive_trees_b200", "lib",
                                                                      "libadaptive_trees_b200.so")],
                         capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    ao = {s for s in exported if s.startswith("ao_")}
    assert ao == set(declared_symbols())


def test_last_error_is_empty_string_initially(lib):
    """In a fresh process (other tests of this session leave messages behind)."""
    code = ("import ctypes, sys; L = ctypes.CDLL(sys.argv[1]); L.ao_last_error.restype = ctypes.c_char_p; "
            "assert L.ao_last_error() == b''")
    subprocess.run([sys.executable, "-c", code, lib._name], check=True, timeout=120)


def test_capi_validates_arguments_without_a_gpu(lib):
    """Invalid arguments are rejected on the host before any device work."""
    from adaptive_trees_b200 import _capi as C
    L = C.load()
    cfg = C.AoConfig()
    cfg.max_depth = -1
    cfg.update_iterations = -1
    cfg.max_particles_per_leaf = 64
    for i, v in enumerate((0, 1, 0, 1, 0, 1)):
        cfg.box[i] = v
    h = ctypes.c_void_p()
    # null output handle
    assert L.ao_tree_create(0, 1, None, None, None, 0, ctypes.byref(cfg), None, None) == 1
    # binary + NFCount (tree.hpp:127-128)
    cfg.split_criterion = 1
    assert L.ao_tree_create(1, 1, None, None, None, 0, ctypes.byref(cfg), None, ctypes.byref(h)) == 1
    assert b"Binary NFCount" in L.ao_last_error()
    cfg.split_criterion = 0
    # binary + Hilbert
    cfg.sfc_kind = 1
    assert L.ao_tree_create(1, 1, None, None, None, 0, ctypes.byref(cfg), None, ctypes.byref(h)) == 1
    cfg.sfc_kind = 0
    # -2 is not a valid "use the default" marker
    cfg.max_depth = -2
    assert L.ao_tree_create(0, 1, None, None, None, 0, ctypes.byref(cfg), None, ctypes.byref(h)) == 1
    assert b"use -1" in L.ao_last_error()
    cfg.max_depth = -1
    # null coordinates with n > 0
    assert L.ao_tree_create(0, 1, None, None, None, 5, ctypes.byref(cfg), None, ctypes.byref(h)) == 1
    assert b"must not be null" in L.ao_last_error()
    # zero bucket
    cfg.max_particles_per_leaf = 0
    assert L.ao_tree_create(0, 1, None, None, None, 0, ctypes.byref(cfg), None, ctypes.byref(h)) == 1
    cfg.max_particles_per_leaf = 64
    # zero update iterations
    cfg.update_iterations = 0
    assert L.ao_tree_create(0, 1, None, None, None, 0, ctypes.byref(cfg), None, ctypes.byref(h)) == 1
    cfg.update_iterations = -1
    # binary maxDepth beyond 63 and degenerate box
    cfg.max_depth = 64
    assert L.ao_tree_create(1, 1, None, None, None, 0, ctypes.byref(cfg), None, ctypes.byref(h)) == 1
    cfg.max_depth = -1
    cfg.box[1] = 0.0
    assert L.ao_tree_create(1, 1, None, None, None, 0, ctypes.byref(cfg), None, ctypes.byref(h)) == 1
    # null handles on every method
    assert L.ao_tree_build(None) == 1
    assert L.ao_tree_update(None) == 1
    out = ctypes.c_int()
    assert L.ao_tree_needs_resize(None, ctypes.byref(out)) == 1


def test_sort_configurations_are_listed_without_a_gpu():
    """The compiled sort configurations and the tuner's argument checks need no device."""
    from adaptive_trees_b200 import _capi as C
    from adaptive_trees_b200 import sort_configs
    configs = sort_configs()
    assert configs[0] == (8, 10)  # the default configuration
    assert len(configs) == len(set(configs)) >= 4
    for bits, items in configs:
        assert bits in (7, 8) and items % 2 == 0 and 8 <= items <= 16
        assert (64 + bits - 1) // bits % 2 == 0  # an even pass count: results stay in the first buffers
    lib = C.load()
    b, i = ctypes.c_int(), ctypes.c_int()
    assert lib.ao_sort_config_info(len(configs), ctypes.byref(b), ctypes.byref(i)) == 1
    assert lib.ao_sort_config_info(0, None, None) == 1
    assert lib.ao_sort_force_config(len(configs)) == 1
    assert lib.ao_sort_force_config(-1) == 0
    assert lib.ao_sort_set_autotune(1) == 0
