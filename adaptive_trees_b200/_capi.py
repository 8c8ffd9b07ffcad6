"""ctypes binding of the engine's C ABI (include/adaptive_trees_b200.h).

The shared library is built in-tree (python -m adaptive_trees_b200.build);
importing this module without it raises ImportError.  There is no fallback
implementation.
"""
from __future__ import annotations

import ctypes
import os
import threading

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libadaptive_trees_b200.so")

AO_OK = 0
STATUS_NAMES = {1: "invalid argument", 2: "logic error", 3: "length error", 4: "CUDA error", 5: "out of memory",
                6: "runtime error"}

# Exported entry points and their prototypes.
vp, sz, ci, cu = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint


class AoConfig(ctypes.Structure):
    _fields_ = [("max_depth", ci), ("max_particles_per_leaf", cu), ("update_iterations", ci),
                ("box", ctypes.c_double * 6), ("split_criterion", ci), ("sfc_kind", ci),
                ("views_tree_structure", ci), ("views_particle_counts", ci), ("views_particle_mapping", ci)]


class AoViewConfig(ctypes.Structure):
    _fields_ = [("tree_structure", ci), ("particle_counts_per_box", ci), ("particle_mapping", ci)]


class AoTreeInfo(ctypes.Structure):
    _fields_ = [("num_particles", sz), ("num_active_particles", sz), ("num_nodes", sz), ("num_leaves", sz),
                ("leaf_capacity", sz), ("max_achieved_depth", cu), ("split_criterion", ci), ("sfc_kind", ci),
                ("kernel_launches", ctypes.c_ulonglong)]


class AoStageTimes(ctypes.Structure):
    _fields_ = [("keys_and_sort_ms", ctypes.c_double), ("refresh_ms", ctypes.c_double),
                ("passes_ms", ctypes.c_double), ("finish_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("near_field_ms", ctypes.c_double), ("near_field_first_ms", ctypes.c_double),
                ("near_field_launches", ci), ("call", ci), ("valid", ci)]


class AoBatchSystemInfo(ctypes.Structure):
    _fields_ = [("num_particles", sz), ("num_active_particles", sz), ("num_leaves", sz), ("leaf_capacity", sz),
                ("needs_resize", ci)]


class AoRequest(ctypes.Structure):
    _fields_ = [("op", ci), ("tree", ctypes.c_longlong), ("kind", ci), ("real_type", ci), ("config", AoConfig),
                ("n", sz), ("x", vp), ("y", vp), ("z", vp), ("want_digest", ci)]


class AoRequestResult(ctypes.Structure):
    _fields_ = [("status", ci), ("queued_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("num_leaves", sz), ("resizes", ci), ("digest", ctypes.c_ulonglong)]


class AoServeStats(ctypes.Structure):
    _fields_ = [("submitted", sz), ("completed", sz), ("failed", sz), ("resident_trees", sz),
                ("resident_bytes", sz), ("peak_bytes", sz), ("particles", ctypes.c_ulonglong),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("particles_per_s", ctypes.c_double), ("span_s", ctypes.c_double)]


PROTOTYPES = {
    "ao_tree_create": [ci, ci, vp, vp, vp, sz, ctypes.POINTER(AoConfig), vp, ctypes.POINTER(vp)],
    "ao_tree_destroy": [vp],
    "ao_tree_build": [vp],
    "ao_tree_update": [vp],
    "ao_tree_update_until_converged": [vp, ci, ctypes.POINTER(ci)],
    "ao_tree_set_profiling": [vp, ci],
    "ao_tree_set_build_mode": [vp, ci],
    "ao_tree_build_path": [vp, ctypes.POINTER(ci), ctypes.POINTER(ci)],
    "ao_tree_stage_times": [vp, vp],
    "ao_tree_compute_views": [vp, ctypes.POINTER(AoViewConfig)],
    "ao_tree_needs_resize": [vp, ctypes.POINTER(ci)],
    "ao_tree_resize_buffers": [vp],
    "ao_tree_get_buffer": [vp, ci, ctypes.POINTER(vp), ctypes.POINTER(sz), ctypes.POINTER(sz)],
    "ao_tree_counters": [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp)],
    "ao_tree_get_info": [vp, ctypes.POINTER(AoTreeInfo)],
    "ao_compute_sfc_keys": [ci, ci, vp, vp, vp, sz, ctypes.POINTER(ctypes.c_double), ci, cu, vp, vp, vp],
    "ao_sort_pairs": [vp, ctypes.POINTER(sz), vp, vp, vp, vp, sz, ci, ci, vp],
    "ao_sort_pairs_noalloc": [vp, vp, vp, vp, sz, ci, ci, vp],
    "ao_sort_pairs_check": [vp, sz, vp],
    "ao_sort_pairs_noalloc_check": [sz, vp],
    "ao_selftest_bounded_wait": [ci, cu, ctypes.POINTER(ci)],
    "ao_sort_config_count": [ctypes.POINTER(ci)],
    "ao_sort_config_info": [ci, ctypes.POINTER(ci), ctypes.POINTER(ci)],
    "ao_sort_tuning": [ci, sz, ctypes.POINTER(ci), ctypes.POINTER(ci), ctypes.POINTER(ci), ctypes.POINTER(ci)],
    "ao_sort_set_autotune": [ci],
    "ao_sort_force_config": [ci],
    "ao_sort_forget_tuning": [],
    "ao_batch_create": [ci, ci, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(sz),
                        ctypes.POINTER(AoConfig), vp, ctypes.POINTER(vp)],
    "ao_batch_destroy": [vp],
    "ao_batch_build": [vp],
    "ao_batch_set_build_mode": [vp, ci],
    "ao_batch_build_path": [vp, ctypes.POINTER(ci)],
    "ao_batch_update": [vp, vp],
    "ao_batch_update_until_converged": [vp, vp, ci, ctypes.POINTER(ci)],
    "ao_batch_needs_resize": [vp, ctypes.POINTER(ci)],
    "ao_batch_resize_buffers": [vp],
    "ao_batch_set_coordinates": [vp, ci, vp, vp, vp],
    "ao_batch_get_buffer": [vp, ci, ci, ctypes.POINTER(vp), ctypes.POINTER(sz)],
    "ao_batch_get_info": [vp, ci, ctypes.POINTER(AoBatchSystemInfo)],
    "ao_serve_create": [ci, sz, ctypes.POINTER(vp)],
    "ao_serve_destroy": [vp],
    "ao_serve_submit": [vp, ctypes.POINTER(AoRequest), ctypes.POINTER(ctypes.c_longlong)],
    "ao_serve_wait": [vp, ctypes.c_longlong, ctypes.POINTER(AoRequestResult)],
    "ao_serve_drain": [vp],
    "ao_serve_get_stats": [vp, ctypes.POINTER(AoServeStats)],
    "ao_serve_reset_stats": [vp],
    "ao_release_cached_memory": [],
    "ao_tree_gather": [vp, vp, vp, sz],
    "ao_read_particles": [ctypes.c_char_p, ci, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                          ctypes.POINTER(sz)],
    "ao_free": [vp],
    "ao_read_manifest": [ctypes.c_char_p, ctypes.POINTER(vp)],
    "ao_manifest_info": [vp, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(sz), ctypes.POINTER(ctypes.c_double),
                         ctypes.POINTER(sz)],
    "ao_manifest_frame": [vp, sz, ctypes.POINTER(ci), ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ci),
                          ctypes.POINTER(ctypes.c_char_p)],
    "ao_manifest_destroy": [vp],
}

# n limit of ao_sort_pairs_noalloc (AO_SORT_PAIRS_NOALLOC_MAX_ITEMS)
SORT_PAIRS_NOALLOC_MAX_ITEMS = 1 << 20

_lock = threading.Lock()
_lib = None


class AoError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def load():
    """Load the built library (no build is attempted here)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"{LIB_PATH} is missing: build it with `python -m adaptive_trees_b200.build`")
            lib = ctypes.CDLL(LIB_PATH)
            lib.ao_last_error.restype = ctypes.c_char_p
            lib.ao_last_error.argtypes = []
            for name, args in PROTOTYPES.items():
                f = getattr(lib, name)
                f.argtypes = args
                f.restype = ci
            _lib = lib
    return _lib


def check(status: int):
    if status != AO_OK:
        raise AoError(status, load().ao_last_error().decode())
