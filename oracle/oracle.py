"""ctypes wrapper of the CPU oracle (oracle/ao_oracle.cpp).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py use this module as the checker.  The product path
(adaptive_trees_b200) never imports it.

The wrapper mirrors the shape of the product's C ABI: a tree handle created
from coordinate arrays and a config, build/update/compute_views,
needs_resize/resize_buffers, and buffer getters returning numpy arrays.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libao_oracle.so")
_lock = threading.Lock()
_lib = None

BUFFERS = {
    "particleKeys": (0, np.uint64),
    "perm": (1, np.uint32),
    "cornerstone": (2, np.uint64),
    "leafCounts": (3, np.uint32),
    "nearFieldCounts": (4, np.uint32),
    "sfcBoxIndex": (5, np.uint64),
    "hasBoxSplit": (6, np.uint8),
    "boxDepth": (7, np.uint8),
    "parentIndex": (8, np.int32),
    "childIndex": (9, np.int32),
    "levelOffset": (10, np.int32),
    "particleBeginIndex": (11, np.uint32),
    "particleCounts": (12, np.uint32),
    "sfcParticleIndex": (13, np.uint64),
}


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class AooConfig(ctypes.Structure):
    _fields_ = [
        ("max_depth", ctypes.c_int),
        ("max_particles_per_leaf", ctypes.c_uint),
        ("update_iterations", ctypes.c_int),
        ("box", ctypes.c_double * 6),
        ("split_criterion", ctypes.c_int),
        ("sfc_kind", ctypes.c_int),
        ("views_tree_structure", ctypes.c_int),
        ("views_particle_counts", ctypes.c_int),
        ("views_particle_mapping", ctypes.c_int),
    ]


def build_oracle() -> str:
    """Compile the oracle shared library (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(_LIB_PATH):
                build_oracle()
            L = ctypes.CDLL(_LIB_PATH)
            vp, sz = ctypes.c_void_p, ctypes.c_size_t
            L.aoo_last_error.restype = ctypes.c_char_p
            L.aoo_tree_create.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp, sz, ctypes.POINTER(AooConfig),
                                          ctypes.POINTER(vp)]
            L.aoo_tree_destroy.argtypes = [vp]
            L.aoo_tree_set_coordinates.argtypes = [vp, vp, vp, vp]
            L.aoo_tree_build.argtypes = [vp]
            L.aoo_tree_update.argtypes = [vp]
            L.aoo_tree_compute_views.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
            L.aoo_tree_needs_resize.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
            L.aoo_tree_resize_buffers.argtypes = [vp]
            L.aoo_tree_copy_buffer.argtypes = [vp, ctypes.c_int, vp, sz, ctypes.POINTER(sz)]
            L.aoo_tree_info.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
            L.aoo_octree_keys.argtypes = [ctypes.c_int, vp, vp, vp, sz, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_ulonglong)]
            L.aoo_binary_keys.argtypes = [ctypes.c_int, vp, vp, vp, sz, ctypes.POINTER(ctypes.c_double),
                                          ctypes.c_uint, ctypes.POINTER(ctypes.c_ulonglong)]
            L.aoo_sfc_encode.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_ulonglong)]
            L.aoo_sfc_decode.argtypes = [ctypes.c_ulonglong, ctypes.c_int, ctypes.POINTER(ctypes.c_uint)]
            _lib = L
    return _lib


def _check(code: int):
    if code != 0:
        raise OracleError(code, lib().aoo_last_error().decode())


def make_config(max_depth=-1, max_particles_per_leaf=64, update_iterations=-1, box=(0, 1, 0, 1, 0, 1),
                split_criterion=0, sfc_kind=0, views=(False, False, False)) -> AooConfig:
    c = AooConfig()
    c.max_depth = max_depth
    c.max_particles_per_leaf = max_particles_per_leaf
    c.update_iterations = update_iterations
    for i in range(6):
        c.box[i] = float(box[i])
    c.split_criterion = int(split_criterion)
    c.sfc_kind = int(sfc_kind)
    c.views_tree_structure, c.views_particle_counts, c.views_particle_mapping = (int(bool(v)) for v in views)
    return c


class OracleTree:
    """CPU model of adaptive_octree::Tree<Real, Kind> (kind 0 octree, 1 binary)."""

    def __init__(self, kind: int, x, y, z, config: AooConfig):
        self.kind = kind
        self._set_arrays(x, y, z)
        self.real = 0 if self._x.dtype == np.float32 else 1
        self.nf = kind == 0 and config.split_criterion == 1
        h = ctypes.c_void_p()
        _check(lib().aoo_tree_create(kind, self.real, self._ptr(self._x), self._ptr(self._y), self._ptr(self._z),
                                     len(self._x), ctypes.byref(config), ctypes.byref(h)))
        self.h = h

    @staticmethod
    def _ptr(a):
        return a.ctypes.data if a.size else None

    def _set_arrays(self, x, y, z):
        x, y, z = (np.ascontiguousarray(a) for a in (x, y, z))
        assert x.dtype == y.dtype == z.dtype and x.dtype in (np.float32, np.float64)
        self._x, self._y, self._z = x, y, z

    def set_coordinates(self, x, y, z):
        """Replace the borrowed coordinates (the reference mutates them in place)."""
        self._set_arrays(x, y, z)
        _check(lib().aoo_tree_set_coordinates(self.h, self._ptr(self._x), self._ptr(self._y), self._ptr(self._z)))

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            lib().aoo_tree_destroy(h)
            self.h = None

    def build(self):
        _check(lib().aoo_tree_build(self.h))

    def update(self):
        _check(lib().aoo_tree_update(self.h))

    def compute_views(self, views=None):
        if views is None:
            _check(lib().aoo_tree_compute_views(self.h, None))
        else:
            arr = (ctypes.c_int * 3)(*(int(bool(v)) for v in views))
            _check(lib().aoo_tree_compute_views(self.h, arr))

    def needs_resize(self) -> bool:
        out = ctypes.c_int()
        _check(lib().aoo_tree_needs_resize(self.h, ctypes.byref(out)))
        return bool(out.value)

    def resize_buffers(self):
        _check(lib().aoo_tree_resize_buffers(self.h))

    def get(self, name: str) -> np.ndarray:
        which, dtype = BUFFERS[name]
        n = ctypes.c_size_t()
        _check(lib().aoo_tree_copy_buffer(self.h, which, None, 0, ctypes.byref(n)))
        out = np.empty(n.value, dtype=dtype)
        _check(lib().aoo_tree_copy_buffer(self.h, which, out.ctypes.data if out.size else None, out.nbytes,
                                          ctypes.byref(n)))
        return out

    def info(self) -> dict:
        arr = (ctypes.c_ulonglong * 10)()
        _check(lib().aoo_tree_info(self.h, arr))
        v = list(arr)
        as_int = lambda u: u - (1 << 64) if u >= (1 << 63) else u  # noqa: E731
        return {
            "numParticles": v[0], "numActiveParticles": v[1], "numNodes": v[2], "maxAchievedDepth": v[3],
            "numLeaves_state": as_int(v[4]), "leafCapacity": v[5], "needsResize_state": v[6],
            "buildIterations": v[7], "activeBuffer": v[8], "numNodes_state": as_int(v[9]),
        }


def octree_keys(x, y, z, box=(0, 1, 0, 1, 0, 1), hilbert=False) -> np.ndarray:
    x, y, z = (np.ascontiguousarray(a) for a in (x, y, z))
    real = 0 if x.dtype == np.float32 else 1
    out = np.empty(len(x), dtype=np.uint64)
    b = (ctypes.c_double * 6)(*box)
    _check(lib().aoo_octree_keys(real, x.ctypes.data, y.ctypes.data, z.ctypes.data, len(x), b, int(hilbert),
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong))))
    return out


def binary_keys(x, y, z, box=(0, 1, 0, 1, 0, 1), max_depth=63) -> np.ndarray:
    x, y, z = (np.ascontiguousarray(a) for a in (x, y, z))
    real = 0 if x.dtype == np.float32 else 1
    out = np.empty(len(x), dtype=np.uint64)
    b = (ctypes.c_double * 6)(*box)
    _check(lib().aoo_binary_keys(real, x.ctypes.data, y.ctypes.data, z.ctypes.data, len(x), b, max_depth,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong))))
    return out


def sfc_encode(x: int, y: int, z: int, hilbert: bool) -> int:
    k = ctypes.c_ulonglong()
    lib().aoo_sfc_encode(x, y, z, int(hilbert), ctypes.byref(k))
    return k.value


def sfc_decode(key: int, hilbert: bool):
    xyz = (ctypes.c_uint * 3)()
    lib().aoo_sfc_decode(key, int(hilbert), xyz)
    return tuple(xyz)
