"""Helpers shared by the GPU tests: device/host conversion and oracle comparison."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

NAMES = ["particleKeys", "perm", "cornerstone", "leafCounts", "nearFieldCounts", "sfcBoxIndex", "hasBoxSplit",
         "boxDepth", "parentIndex", "childIndex", "levelOffset", "particleBeginIndex", "particleCounts",
         "sfcParticleIndex"]
NP = {"particleKeys": np.uint64, "perm": np.uint32, "cornerstone": np.uint64, "leafCounts": np.uint32,
      "nearFieldCounts": np.uint32, "sfcBoxIndex": np.uint64, "hasBoxSplit": np.uint8, "boxDepth": np.uint8,
      "parentIndex": np.int32, "childIndex": np.int32, "levelOffset": np.int32, "particleBeginIndex": np.uint32,
      "particleCounts": np.uint32, "sfcParticleIndex": np.uint64}


def to_np(t) -> np.ndarray:
    import torch
    if t.dtype == torch.uint64:
        return t.view(torch.int64).cpu().numpy().view(np.uint64)
    if t.dtype == torch.uint32:
        return t.view(torch.int32).cpu().numpy().view(np.uint32)
    return t.cpu().numpy()


def gpu_get(tree, name):
    return to_np(tree.get(name + "_d"))


def to_dev(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def tree_config(max_depth=-1, bucket=64, iters=-1, box=(0, 1, 0, 1, 0, 1), nf=False, hilbert=False,
                views=(False, False, False)):
    from adaptive_trees_b200 import SfcKind, SplitCriterion, TreeConfig, ViewConfig
    return TreeConfig(maxDepth=max_depth, maxParticlesPerLeaf=bucket, updateIterations=iters, box=tuple(box),
                      splitCriterion=SplitCriterion.NFCount if nf else SplitCriterion.LeafCount,
                      sfcKind=SfcKind.Hilbert if hilbert else SfcKind.Morton,
                      views=ViewConfig(*[bool(v) for v in views]))


def oracle_config(max_depth=-1, bucket=64, iters=-1, box=(0, 1, 0, 1, 0, 1), nf=False, hilbert=False,
                  views=(False, False, False)):
    return O.make_config(max_depth=max_depth, max_particles_per_leaf=bucket, update_iterations=iters, box=box,
                         split_criterion=int(nf), sfc_kind=int(hilbert), views=views)


def compare(gpu_tree, oracle_tree, names=None, skip=()):
    """Assert every buffer (logical contents) equal; returns the list of names compared."""
    names = names or NAMES
    done = []
    for name in names:
        if name in skip:
            continue
        try:
            e = oracle_tree.get(name)
        except O.OracleError:
            continue
        a = gpu_get(gpu_tree, name)
        assert a.dtype == e.dtype, (name, a.dtype, e.dtype)
        assert a.size == e.size, f"{name}: size {a.size} != oracle {e.size}"
        if name == "nearFieldCounts" and not getattr(oracle_tree, "nf", True):
            continue  # defined only for NFCount trees
        bad = np.nonzero(a != e)[0]
        assert bad.size == 0, f"{name}: {bad.size} mismatches, first at {bad[:5]}: gpu {a[bad[:5]]} oracle {e[bad[:5]]}"
        done.append(name)
    gi, oi = gpu_tree.info(), oracle_tree.info()
    assert gi.num_active_particles == oi["numActiveParticles"]
    assert gi.num_nodes == oi["numNodes"], (gi.num_nodes, oi["numNodes"])
    assert gi.max_achieved_depth == oi["maxAchievedDepth"], (gi.max_achieved_depth, oi["maxAchievedDepth"])
    assert gi.leaf_capacity == oi["leafCapacity"], (gi.leaf_capacity, oi["leafCapacity"])
    return done
