"""Python mirror of adaptive_octree::Tree<Real, TreeType::Octree|Binary>.

Same method names as the reference's C++ facade (tree.hpp:11-134), backed by
the engine's C ABI.  Coordinates are CUDA tensors (float32 or float64) that
the tree borrows: change them in place between update() calls, as the
reference expects.  Getters return zero-copy CUDA tensors over the engine's
buffers, sized by the last build()/doBuffersNeedResize().
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from enum import IntEnum

from . import _capi as C

OCTREE, BINARY = 0, 1


class TreeType(IntEnum):
    Octree = 0
    Binary = 1


class SplitCriterion(IntEnum):
    LeafCount = 0
    NFCount = 1


class SfcKind(IntEnum):
    Morton = 0
    Hilbert = 1


@dataclass
class ViewConfig:
    treeStructure: bool = False
    particleCountsPerBox: bool = False
    particleMapping: bool = False

    def any(self):
        return self.treeStructure or self.particleCountsPerBox or self.particleMapping


@dataclass
class TreeConfig:
    """TreeConfig<Real> (config.hpp:147-160)."""
    maxDepth: int = -1
    maxParticlesPerLeaf: int = 64
    updateIterations: int = -1
    box: tuple = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    splitCriterion: SplitCriterion = SplitCriterion.LeafCount
    sfcKind: SfcKind = SfcKind.Morton
    views: ViewConfig = field(default_factory=ViewConfig)

    def to_c(self) -> C.AoConfig:
        c = C.AoConfig()
        c.max_depth = int(self.maxDepth)
        c.max_particles_per_leaf = int(self.maxParticlesPerLeaf)
        c.update_iterations = int(self.updateIterations)
        for i in range(6):
            c.box[i] = float(self.box[i])
        c.split_criterion = int(self.splitCriterion)
        c.sfc_kind = int(self.sfcKind)
        c.views_tree_structure = int(bool(self.views.treeStructure))
        c.views_particle_counts = int(bool(self.views.particleCountsPerBox))
        c.views_particle_mapping = int(bool(self.views.particleMapping))
        return c


BUFFERS = {
    "particleKeys_d": (0, "<u8"), "perm_d": (1, "<u4"), "cornerstone_d": (2, "<u8"), "leafCounts_d": (3, "<u4"),
    "nearFieldCounts_d": (4, "<u4"), "sfcBoxIndex_d": (5, "<u8"), "hasBoxSplit_d": (6, "|u1"),
    "boxDepth_d": (7, "|u1"), "parentIndex_d": (8, "<i4"), "childIndex_d": (9, "<i4"),
    "levelOffset_d": (10, "<i4"), "particleBeginIndex_d": (11, "<u4"), "particleCounts_d": (12, "<u4"),
    "sfcParticleIndex_d": (13, "<u8"), "leafBegins_d": (14, "<u4"),
}


class _DeviceArray:
    """__cuda_array_interface__ wrapper for a device pointer."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


def _torch():
    import torch
    return torch


def device_tensor(ptr: int, n: int, typestr: str):
    """Zero-copy torch view of `n` elements at device address `ptr`."""
    torch = _torch()
    dt = {"<u8": torch.uint64, "<u4": torch.uint32, "|u1": torch.uint8, "<i4": torch.int32}[typestr]
    if n == 0 or not ptr:
        return torch.empty(0, dtype=dt, device="cuda")
    return torch.as_tensor(_DeviceArray(ptr, n, typestr), device="cuda")


class Tree:
    """Tree<Real, Kind>: kind 0 = Octree, 1 = Binary; Real from the tensor dtype."""

    def __init__(self, kind, x, y, z, config: TreeConfig | None = None, stream=None):
        torch = _torch()
        config = config or TreeConfig()
        self.kind = int(kind)
        if not (x.is_cuda and y.is_cuda and z.is_cuda):
            raise ValueError("coordinates must be CUDA tensors")
        if not (x.dtype == y.dtype == z.dtype) or x.dtype not in (torch.float32, torch.float64):
            raise ValueError("coordinates must share dtype float32 or float64")
        if not (x.is_contiguous() and y.is_contiguous() and z.is_contiguous()):
            raise ValueError("coordinates must be contiguous")
        self._coords = (x, y, z)  # keep the borrowed storage alive
        self.real = 0 if x.dtype == torch.float32 else 1
        self.config = config
        if stream is None:
            stream = torch.cuda.current_stream()
        self.stream = stream
        h = ctypes.c_void_p()
        cfg = config.to_c()
        lib = C.load()
        n = x.numel()
        C.check(lib.ao_tree_create(self.kind, self.real, x.data_ptr() if n else None, y.data_ptr() if n else None,
                                   z.data_ptr() if n else None, n, ctypes.byref(cfg),
                                   ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            C.load().ao_tree_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # --- reference methods ---
    def build(self):
        C.check(C.load().ao_tree_build(self._h))

    def update(self):
        C.check(C.load().ao_tree_update(self._h))

    def updateUntilConverged(self, max_passes: int = 64) -> int:
        """Opt-in: update passes until one changes nothing, at most
        `max_passes`; returns the passes that changed the tree.  The result
        equals update() with updateIterations = max_passes; the reference's
        update() runs a fixed pass count (octree.cu:471-481,
        kdtree3d.cu:259-270)."""
        out = ctypes.c_int()
        C.check(C.load().ao_tree_update_until_converged(self._h, int(max_passes), ctypes.byref(out)))
        return out.value

    def setBuildMode(self, mode: int):
        """Octree build() path: 0 the converged tree level by level (falling
        back to rounds where needed), 1 the reference's split/merge rounds."""
        C.check(C.load().ao_tree_set_build_mode(self._h, int(mode)))

    def buildPath(self):
        """(built by levels, build rounds that changed the tree) of the last build()."""
        lv, rounds = ctypes.c_int(), ctypes.c_int()
        C.check(C.load().ao_tree_build_path(self._h, ctypes.byref(lv), ctypes.byref(rounds)))
        return bool(lv.value), rounds.value

    def setProfiling(self, on: bool = True):
        """Stage timing of octree build() and update() with CUDA events and
        NVTX ranges (the reference's ADAPTIVE_OCTREE_PROFILING ranges,
        config.hpp:20-28)."""
        C.check(C.load().ao_tree_set_profiling(self._h, 1 if on else 0))

    def stageTimes(self) -> dict | None:
        """Stage times (ms) of the last profiled build() or update(), or None."""
        t = C.AoStageTimes()
        C.check(C.load().ao_tree_stage_times(self._h, ctypes.byref(t)))
        if not t.valid:
            return None
        out = {k: getattr(t, k) for k, _ in C.AoStageTimes._fields_ if k != "valid"}
        out["call"] = {1: "build", 2: "update"}.get(t.call, "?")
        return out

    def computeViews(self, views: ViewConfig | None = None):
        if views is None:
            C.check(C.load().ao_tree_compute_views(self._h, None))
        else:
            v = C.AoViewConfig(int(views.treeStructure), int(views.particleCountsPerBox), int(views.particleMapping))
            C.check(C.load().ao_tree_compute_views(self._h, ctypes.byref(v)))

    def doBuffersNeedResize(self) -> bool:
        out = ctypes.c_int()
        C.check(C.load().ao_tree_needs_resize(self._h, ctypes.byref(out)))
        return bool(out.value)

    def resizeBuffers(self):
        C.check(C.load().ao_tree_resize_buffers(self._h))

    def buffer_info(self, name: str):
        which, typestr = BUFFERS[name]
        p, n, cap = ctypes.c_void_p(), ctypes.c_size_t(), ctypes.c_size_t()
        C.check(C.load().ao_tree_get_buffer(self._h, which, ctypes.byref(p), ctypes.byref(n), ctypes.byref(cap)))
        return p.value or 0, n.value, cap.value, typestr

    def get(self, name: str):
        p, n, _, typestr = self.buffer_info(name)
        return device_tensor(p, n, typestr)

    def gather(self, t):
        """Per-particle data in key order: out[i] = t[perm[i]] (device tensor, first dim numParticles)."""
        torch = _torch()
        if not t.is_cuda or t.shape[0] != self.numParticles():
            raise ValueError("gather needs a CUDA tensor with numParticles rows")
        t = t.contiguous()
        out = torch.empty_like(t)
        if t.numel():
            C.check(C.load().ao_tree_gather(self._h, t.data_ptr(), out.data_ptr(), t.element_size() * t[0].numel()))
        return out

    def info(self) -> C.AoTreeInfo:
        i = C.AoTreeInfo()
        C.check(C.load().ao_tree_get_info(self._h, ctypes.byref(i)))
        return i

    def counters(self):
        a, b, c = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        C.check(C.load().ao_tree_counters(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def numParticles(self):
        return self.info().num_particles

    def numActiveParticles(self):
        return self.info().num_active_particles

    def numNodes(self):
        return self.info().num_nodes

    def maxAchievedDepth(self):
        return self.info().max_achieved_depth

    def splitCriterion(self):
        return SplitCriterion(self.info().split_criterion)

    def sfcKind(self):
        k = self.info().sfc_kind
        if k < 0:
            raise RuntimeError("Tree: SFC selection requires Octree mode")
        return SfcKind(k)


def _getter(name):
    def f(self):
        return self.get(name)
    f.__name__ = name
    return f


for _name in BUFFERS:
    setattr(Tree, _name, _getter(_name))


def compute_sfc_keys(kind, x, y, z, box=(0, 1, 0, 1, 0, 1), sfc_kind=SfcKind.Morton, max_depth=63, with_perm=False,
                     stream=None):
    """computeSfcKeys / computeSfcKeysBinary: unsorted keys (and identity perm) on the device."""
    torch = _torch()
    n = x.numel()
    keys = torch.empty(n, dtype=torch.uint64, device="cuda")
    perm = torch.empty(n, dtype=torch.uint32, device="cuda") if with_perm else None
    stream = stream or torch.cuda.current_stream()
    b = (ctypes.c_double * 6)(*[float(v) for v in box])
    real = 0 if x.dtype == torch.float32 else 1
    C.check(C.load().ao_compute_sfc_keys(int(kind), real, x.data_ptr() if n else None, y.data_ptr() if n else None,
                                         z.data_ptr() if n else None, n, b, int(sfc_kind), int(max_depth),
                                         keys.data_ptr() if n else None,
                                         perm.data_ptr() if (perm is not None and n) else None,
                                         ctypes.c_void_p(stream.cuda_stream)))
    return (keys, perm) if with_perm else keys
