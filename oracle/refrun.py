"""Run the reference library (oracle/_ref/ref_driver) on a scenario.

TEST INFRASTRUCTURE ONLY: tests/ use it to compare the B200 engine with the
reference itself on the same GPU, bench.py to time the reference's GPU path.
The driver binary is built from the reference's sources by `make -C oracle ref`
(needs the reference checkout; the built binary then travels with the repo).
"""
from __future__ import annotations

import json
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "_ref", "ref_driver")
ARRAY_NAMES = ["particleKeys", "perm", "cornerstone", "leafCounts", "nearFieldCounts", "sfcBoxIndex", "hasBoxSplit",
               "boxDepth", "parentIndex", "childIndex", "levelOffset", "particleBeginIndex", "particleCounts",
               "sfcParticleIndex"]
DTYPES = {0: np.uint64, 1: np.uint32, 2: np.uint64, 3: np.uint32, 4: np.uint32, 5: np.uint64, 6: np.uint8,
          7: np.uint8, 8: np.int32, 9: np.int32, 10: np.int32, 11: np.uint32, 12: np.uint32, 13: np.uint64}


def available() -> bool:
    return os.path.exists(DRIVER) and os.access(DRIVER, os.X_OK)


def write_scenario(path, kind, frames, max_depth=-1, bucket=64, update_iterations=-1, nf=False, hilbert=False,
                   views=(True, True, True), box=(0, 1, 0, 1, 0, 1), timing_reps=0):
    """frames: list of (x, y, z) arrays, all float32 or all float64."""
    real = 0 if frames[0][0].dtype == np.float32 else 1
    n = frames[0][0].size
    hdr = struct.pack("<4I Q i I i 2I 3I I 4x 6d", 0x43534F41, kind, real, len(frames), n, max_depth, bucket,
                      update_iterations, int(nf), int(hilbert), *[int(bool(v)) for v in views], timing_reps,
                      *[float(b) for b in box])
    assert len(hdr) == 112
    with open(path, "wb") as f:
        f.write(hdr)
        for xyz in frames:
            for a in xyz:
                f.write(np.ascontiguousarray(a).tobytes())


def digest(a) -> int:
    """Order-sensitive digest of an integer array, as ref_driver --digest writes
    it: sum over i of splitmix64(a[i] + i * 0x9E3779B97F4A7C15) mod 2^64, each
    element taken as its unsigned bit pattern widened to 64 bits."""
    a = np.ascontiguousarray(a)
    u = a.view({1: np.uint8, 4: np.uint32, 8: np.uint64}[a.dtype.itemsize]).astype(np.uint64)
    z = u + np.arange(u.size, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    z ^= z >> np.uint64(30)
    z *= np.uint64(0xBF58476D1CE4E5B9)
    z ^= z >> np.uint64(27)
    z *= np.uint64(0x94D049BB133111EB)
    z ^= z >> np.uint64(31)
    return int(z.sum(dtype=np.uint64))


def read_output(path, digests=False):
    """List of per-frame dicts: name -> array (digests: name -> (count, digest)),
    plus 'scalars'."""
    out, cur = [], {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        (ident,) = struct.unpack_from("<I", data, pos)
        pos += 4
        if ident == 0xFFFFFFFF:
            cur["scalars"] = struct.unpack_from("<6Q", data, pos)
            pos += 48
            out.append(cur)
            cur = {}
            continue
        count, eb = struct.unpack_from("<QQ", data, pos)
        pos += 16
        if digests:
            (d,) = struct.unpack_from("<Q", data, pos)
            pos += 8
            cur[ARRAY_NAMES[ident]] = (count, d)
            continue
        arr = np.frombuffer(data, dtype=DTYPES[ident], count=count, offset=pos).copy()
        pos += count * eb
        cur[ARRAY_NAMES[ident]] = arr
    return out


def run(kind, frames, timeout=1800, digests=False, **cfg):
    """Run the reference on build(frame 0) + update(frame k) with its resize loop.

    digests: return (count, digest) per array instead of the arrays."""
    with tempfile.TemporaryDirectory() as d:
        sc, res = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        write_scenario(sc, kind, frames, **cfg)
        cmd = [DRIVER, sc, res] + (["--digest"] if digests else [])
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_driver failed ({r.returncode}): {r.stderr.strip()}")
        return read_output(res, digests=digests)


def time_reference(kind, frames, reps=10, timeout=1800, **cfg):
    """Build and captured-update times (ms) of the reference on this GPU: the
    median of `reps` warm builds of one tree (and its cold first build), and of
    `reps` graph replays of update() on frame 1."""
    with tempfile.TemporaryDirectory() as d:
        sc = os.path.join(d, "in.bin")
        write_scenario(sc, kind, frames, timing_reps=reps, **cfg)
        r = subprocess.run([DRIVER, sc, os.path.join(d, "unused")], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_driver failed ({r.returncode}): {r.stderr.strip()}")
        return json.loads(r.stdout.strip().splitlines()[-1])


def time_cub_sort(keys, reps=10, timeout=600):
    """CUB's SortPairs (64-bit keys carrying 32-bit indices, bits [0, 64), the
    reference's particle sort) on `keys` (numpy uint64) on this GPU: median ms."""
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "keys.bin")
        with open(path, "wb") as f:
            f.write(np.uint64(keys.size).tobytes())
            f.write(np.ascontiguousarray(keys, dtype=np.uint64).tobytes())
        r = subprocess.run([DRIVER, "--cub-sort", path, str(reps)], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_driver failed ({r.returncode}): {r.stderr.strip()}")
        return json.loads(r.stdout.strip().splitlines()[-1])
