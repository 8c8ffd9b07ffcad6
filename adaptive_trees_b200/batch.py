"""Batched octrees: many independent particle systems built and updated together.

The reference's callers loop over one Tree<Real, Octree> per system.  A Batch
holds all the systems and gives each exactly what that loop would give it
(the same keys, permutation, cornerstone, counts, leafCapacity and
needsResize), while the work of all systems runs in shared kernel launches
(octree, LeafCount refinement, Morton or Hilbert keys, no views).
"""
from __future__ import annotations

import ctypes

from . import _capi as C
from .tree import TreeConfig, _torch, device_tensor

BUFFERS = {"particleKeys_d": (0, "<u8"), "perm_d": (1, "<u4"), "cornerstone_d": (2, "<u8"),
           "leafCounts_d": (3, "<u4")}


class Batch:
    """One Tree<Real, Octree>(xs[s], ys[s], zs[s], config) per system s, sharing launches."""

    def __init__(self, xs, ys, zs, config: TreeConfig | None = None, stream=None):
        torch = _torch()
        config = config or TreeConfig()
        if not (len(xs) == len(ys) == len(zs)) or len(xs) == 0:
            raise ValueError("need the same positive number of x, y and z arrays")
        dtype = xs[0].dtype
        for t in (*xs, *ys, *zs):
            if not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
                raise ValueError("coordinates must be contiguous CUDA tensors of one dtype")
        for x, y, z in zip(xs, ys, zs):
            if not (x.numel() == y.numel() == z.numel()):
                raise ValueError("x, y and z of a system must have the same length")
        if dtype not in (torch.float32, torch.float64):
            raise ValueError("coordinates must be float32 or float64")
        self.real = 0 if dtype == torch.float32 else 1
        self.config = config
        self.stream = stream or torch.cuda.current_stream()
        self._coords = [list(xs), list(ys), list(zs)]  # keep the borrowed storage alive
        S = len(xs)
        P = ctypes.c_void_p * S
        ptr = lambda t: t.data_ptr() if t.numel() else None  # noqa: E731
        px, py, pz = P(*[ptr(t) for t in xs]), P(*[ptr(t) for t in ys]), P(*[ptr(t) for t in zs])
        counts = (ctypes.c_size_t * S)(*[t.numel() for t in xs])
        cfg = config.to_c()
        h = ctypes.c_void_p()
        C.check(C.load().ao_batch_create(self.real, S, px, py, pz, counts, ctypes.byref(cfg),
                                         ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self._h = h
        self.num_systems = S

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            C.load().ao_batch_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self):
        C.check(C.load().ao_batch_build(self._h))

    def setBuildMode(self, mode: int):
        """build() path: 0 every system's converged tree by levels in one
        persistent launch (falling back to rounds where needed), 1 the rounds."""
        C.check(C.load().ao_batch_set_build_mode(self._h, int(mode)))

    def buildPath(self) -> bool:
        """True when the last build() used the level builder."""
        out = ctypes.c_int()
        C.check(C.load().ao_batch_build_path(self._h, ctypes.byref(out)))
        return bool(out.value)

    def update(self, frozen=None):
        """update() of every system; `frozen` (sequence of bools) keeps the marked systems' trees."""
        if frozen is None:
            C.check(C.load().ao_batch_update(self._h, None))
        else:
            arr = (ctypes.c_ubyte * self.num_systems)(*[1 if f else 0 for f in frozen])
            C.check(C.load().ao_batch_update(self._h, arr))

    def updateUntilConverged(self, max_passes: int = 64, frozen=None) -> int:
        """Opt-in: update passes until one changes no system, at most
        `max_passes`; returns the passes that changed some system.  Every
        system's tree equals update() with updateIterations = max_passes."""
        arr = None
        if frozen is not None:
            arr = (ctypes.c_ubyte * self.num_systems)(*[1 if f else 0 for f in frozen])
        out = ctypes.c_int()
        C.check(C.load().ao_batch_update_until_converged(self._h, arr, int(max_passes), ctypes.byref(out)))
        return out.value

    def doBuffersNeedResize(self) -> bool:
        out = ctypes.c_int()
        C.check(C.load().ao_batch_needs_resize(self._h, ctypes.byref(out)))
        return bool(out.value)

    def resizeBuffers(self):
        C.check(C.load().ao_batch_resize_buffers(self._h))

    def setCoordinates(self, s, x, y, z):
        n = x.numel()
        C.check(C.load().ao_batch_set_coordinates(self._h, int(s), x.data_ptr() if n else None,
                                                  y.data_ptr() if n else None, z.data_ptr() if n else None))
        self._coords[0][s], self._coords[1][s], self._coords[2][s] = x, y, z

    def info(self, s) -> C.AoBatchSystemInfo:
        i = C.AoBatchSystemInfo()
        C.check(C.load().ao_batch_get_info(self._h, int(s), ctypes.byref(i)))
        return i

    def get(self, s, name: str):
        which, typestr = BUFFERS[name]
        p, n = ctypes.c_void_p(), ctypes.c_size_t()
        C.check(C.load().ao_batch_get_buffer(self._h, int(s), which, ctypes.byref(p), ctypes.byref(n)))
        return device_tensor(p.value or 0, n.value, typestr)
