"""Generate the golden fixtures from the reference's own regression data.

Reads (read-only) the reference project's tests/verification_data: the two
114,537-particle Coulomb-explosion snapshots and the reference_output CSVs that
its "[regression]" test compares against (tree_test.cu:155-209), and writes:

  coulomb_snapshots.f64.xz  x0,y0,z0 (snapshot_0000) then x1,y1,z1 (snapshot_1000),
                            little-endian float64, lzma-compressed
  coulomb_expected.npz    every reference_output array used by the regression
                          test, except leafCounts_d (stale in the reference) and
                          the three 114,537-long arrays, which are pinned by digest
  coulomb_expected.json   length + sha256 of every array, and maxAchievedDepth

Usage:  python tests/golden/make_golden.py [path/to/reference/tests/verification_data]
"""
from __future__ import annotations

import hashlib
import json
import lzma
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_SRC = "/root/reference/tests/verification_data"

# name -> dtype of the reference getter (config.hpp:38-40, octree.hpp:81-120)
ARRAYS = {
    "particleKeys_d": np.uint64,
    "perm_d": np.uint32,
    "cornerstone_d": np.uint64,
    "sfcBoxIndex_d": np.uint64,
    "particleBeginIndex_d": np.uint32,
    "particleCounts_d": np.uint32,
    "hasBoxSplit_d": np.uint8,
    "boxDepth_d": np.uint8,
    "parentIndex_d": np.int32,
    "childIndex_d": np.int32,
    "sfcParticleIndex_d": np.uint64,
    "levelOffset_d": np.int32,
}
DIGEST_ONLY = {"particleKeys_d", "perm_d", "sfcParticleIndex_d"}


def read_column(path: str, dtype) -> np.ndarray:
    with open(path) as f:
        f.readline()
        vals = [int(v) for v in f.read().split()]
    if np.dtype(dtype).kind == "i":
        return np.array(vals, dtype=np.int64).astype(dtype)
    return np.array([v & 0xFFFFFFFFFFFFFFFF for v in vals], dtype=np.uint64).astype(dtype)


def read_snapshot(path: str):
    # Rows "charge x y z" after '#' comment lines (particle_io.hpp:36-140).
    d = np.loadtxt(path, comments="#")
    return (np.ascontiguousarray(d[:, 1]), np.ascontiguousarray(d[:, 2]), np.ascontiguousarray(d[:, 3]))


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main(src: str = DEFAULT_SRC):
    x0, y0, z0 = read_snapshot(os.path.join(src, "snapshot_0000.dat"))
    x1, y1, z1 = read_snapshot(os.path.join(src, "snapshot_1000.dat"))
    raw = np.concatenate([x0, y0, z0, x1, y1, z1]).astype("<f8").tobytes()
    with open(os.path.join(HERE, "coulomb_snapshots.f64.xz"), "wb") as f:
        f.write(lzma.compress(raw, preset=9 | lzma.PRESET_EXTREME))
    meta = {"source": "tests/verification_data of nrottstegge/Adaptive_Trees",
            "num_particles": int(x0.size),
            "config": {"tree": "Octree<double>", "maxParticlesPerLeaf": 64 * 64 * 27, "splitCriterion": "NFCount",
                       "sfcKind": "Morton", "box": [0, 1, 0, 1, 0, 1], "views": [True, True, True],
                       "sequence": "build(snapshot_0000); update(snapshot_1000) with resize loop"},
            "arrays": {}}
    small = {}
    for name, dtype in ARRAYS.items():
        a = read_column(os.path.join(src, "reference_output", name + ".csv"), dtype)
        meta["arrays"][name] = {"len": int(a.size), "dtype": np.dtype(dtype).name, "sha256": digest(a)}
        if name not in DIGEST_ONLY:
            small[name] = a
    with open(os.path.join(src, "reference_output", "scalars.csv")) as f:
        f.readline()
        for line in f:
            k, v = line.strip().split(",")
            meta[k] = int(v)
    np.savez_compressed(os.path.join(HERE, "coulomb_expected.npz"), **small)
    with open(os.path.join(HERE, "coulomb_expected.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
        f.write("\n")



def load_snapshots():
    """Return ((x0, y0, z0), (x1, y1, z1)) from the committed fixture."""
    with open(os.path.join(HERE, "coulomb_expected.json")) as f:
        n = json.load(f)["num_particles"]
    with open(os.path.join(HERE, "coulomb_snapshots.f64.xz"), "rb") as f:
        a = np.frombuffer(lzma.decompress(f.read()), dtype="<f8")
    parts = [np.ascontiguousarray(a[i * n:(i + 1) * n]) for i in range(6)]
    return tuple(parts[:3]), tuple(parts[3:])


def load_expected():
    """Return (meta, arrays) of the committed expected outputs."""
    with open(os.path.join(HERE, "coulomb_expected.json")) as f:
        meta = json.load(f)
    with np.load(os.path.join(HERE, "coulomb_expected.npz")) as z:
        arrays = {k: z[k] for k in z.files}
    return meta, arrays


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC)
