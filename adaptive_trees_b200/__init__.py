"""B200-native adaptive-tree engine (octree / binary k-d cornerstone trees).

Drop-in for the tree path of nrottstegge/Adaptive_Trees: the C++ classes
(include/adaptive_octree/*.hpp), the C ABI (include/adaptive_trees_b200.h)
and this Python mirror of adaptive_octree::Tree.  Every stage runs as a
hand-written sm_100a kernel; importing `Tree` without the built library
raises ImportError.
"""
from .batch import Batch  # noqa: F401
from .serve import Server, release_cached_memory  # noqa: F401
from .sort_tuning import force_sort_config, forget_sort_tuning, set_sort_autotune, sort_configs, sort_tuning  # noqa: F401
from .tree import (BINARY, OCTREE, SfcKind, SplitCriterion, Tree, TreeConfig, TreeType, ViewConfig,  # noqa: F401
                   compute_sfc_keys, device_tensor)

__all__ = ["Tree", "Batch", "Server", "release_cached_memory", "TreeConfig", "ViewConfig", "TreeType", "SplitCriterion", "SfcKind", "OCTREE", "BINARY",
           "compute_sfc_keys", "device_tensor", "sort_configs", "sort_tuning", "set_sort_autotune",
           "force_sort_config", "forget_sort_tuning"]
