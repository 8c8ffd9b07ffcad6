"""Input generators shared by the CPU (oracle) and GPU (library) tests.

The small deterministic particle sets restate the reference test inputs
(tests/tree_test.cu of nrottstegge/Adaptive_Trees); the synthetic generators
produce seeded stand-ins for the benchmark configurations (uniform cube,
truncated Plummer sphere, anisotropic Gaussian mixture) at any size.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np

ESC64 = np.finfo(np.float64).max
ESC32 = np.finfo(np.float32).max
ROOT_END = 1 << 63


# --- reference test inputs -------------------------------------------------
def slot_coordinates(active_mask: int, compact: bool = False, slots: int = 8):
    """coordinatesForMask (tree_test.cu:244-262): slot s at (0.25|0.75)^3 by its bits."""
    xs, ys, zs = [], [], []
    for s in range(slots):
        active = bool(active_mask & (1 << s))
        if not active and compact:
            continue
        xs.append((0.75 if s & 1 else 0.25) if active else ESC64)
        ys.append((0.75 if s & 2 else 0.25) if active else ESC64)
        zs.append((0.75 if s & 4 else 0.25) if active else ESC64)
    return tuple(np.array(a, dtype=np.float64) for a in (xs, ys, zs))


def lattice_particles(box, count: int = 65):
    """particles() (tree_test.cu:545-559): a scrambled lattice inside `box`."""
    pts = []
    for i in range(count):
        fx = ((i * 173) % 1024) / 1024.0
        fy = ((i * 317) % 1024) / 1024.0
        fz = ((i * 563) % 1024) / 1024.0
        pts.append((box[0] + fx * (box[1] - box[0]), box[2] + fy * (box[3] - box[2]), box[4] + fz * (box[5] - box[4])))
    return pts


def to_xyz(points, dtype=np.float64):
    a = np.array(points, dtype=np.float64).reshape(-1, 3)
    return tuple(np.ascontiguousarray(a[:, i].astype(dtype)) for i in range(3))


def escaped_point():
    return (ESC64, ESC64, ESC64)


# --- independent physical bisection (tree_test.cu:561-640), exact rationals --
class Cell:
    __slots__ = ("lo", "hi", "begin", "end", "depth")

    def __init__(self, lo, hi, begin=0, end=ROOT_END, depth=0):
        self.lo, self.hi, self.begin, self.end, self.depth = lo, hi, begin, end, depth


def root_cell(box):
    return Cell([Fraction(box[0]), Fraction(box[2]), Fraction(box[4])],
                [Fraction(box[1]), Fraction(box[3]), Fraction(box[5])])


def _longest(c):
    a = 0
    for k in (1, 2):
        if c.hi[k] - c.lo[k] > c.hi[a] - c.lo[a]:
            a = k
    return a


def split_cell(c):
    a = _longest(c)
    mid = (c.lo[a] + c.hi[a]) / 2
    km = c.begin + (c.end - c.begin) // 2
    left = Cell(list(c.lo), list(c.hi), c.begin, km, c.depth + 1)
    right = Cell(list(c.lo), list(c.hi), km, c.end, c.depth + 1)
    left.hi[a] = mid
    right.lo[a] = mid
    return left, right


def contains(c, p):
    return all(c.lo[k] <= Fraction(p[k]) < c.hi[k] for k in range(3))


def physical_key(p, box):
    """Key from 63 physical bisections; escaped -> ~0."""
    if p[0] == ESC64 and p[1] == ESC64 and p[2] == ESC64:
        return (1 << 64) - 1
    c = root_cell(box)
    fp = [Fraction(v) for v in p]
    while c.depth < 63:
        a = _longest(c)
        l, r = split_cell(c)
        c = r if fp[a] >= r.lo[a] else l
    return c.begin


def expected_binary_leaves(box, points, bucket, max_depth):
    out = []

    def rec(c, pts):
        inside = [p for p in pts if contains(c, p)]
        if len(inside) <= bucket or c.depth >= max_depth:
            out.append((c, len(inside)))
            return
        for ch in split_cell(c):
            rec(ch, inside)

    rec(root_cell(box), [p for p in points if p[0] != ESC64])
    return out


# --- seeded synthetic inputs of the benchmark configurations ---------------
def uniform_cube(n: int, seed: int = 1, dtype=np.float64):
    """x, y, z i.i.d. U[0,1) (plain octree configuration)."""
    rng = np.random.default_rng(seed)
    a = rng.random((3, n))
    return tuple(np.ascontiguousarray(a[i].astype(dtype)) for i in range(3))


def plummer_sphere(n: int, seed: int = 2, scale: float = 0.05, centre=(0.5, 0.5, 0.5), rmax: float = 0.5,
                   dtype=np.float32):
    """Truncated Plummer sphere: r = a / sqrt(u^(-2/3) - 1), isotropic, r <= rmax."""
    rng = np.random.default_rng(seed)
    out = np.empty((0, 3))
    while out.shape[0] < n:
        m = int((n - out.shape[0]) * 1.1) + 16
        u = rng.random(m)
        u = np.clip(u, 1e-12, 1.0 - 1e-12)
        r = scale / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        r = r[r <= rmax]
        v = rng.normal(size=(r.size, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        out = np.concatenate([out, v * r[:, None] + np.asarray(centre)])
    out = np.clip(out[:n], 0.0, np.nextafter(1.0, 0.0))
    return tuple(np.ascontiguousarray(out[:, i].astype(dtype)) for i in range(3))


def gaussian_mixture(n: int, seed: int = 3, clusters: int = 8, dtype=np.float64):
    """Equal-weight mixture of anisotropic Gaussians (centres U[0.2,0.8]^3,
    per-axis sigma log-uniform in [0.005, 0.05]), clamped to [0, 1)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2, 0.8, size=(clusters, 3))
    sig = np.exp(rng.uniform(np.log(0.005), np.log(0.05), size=(clusters, 3)))
    lab = rng.integers(0, clusters, size=n)
    pts = centres[lab] + rng.normal(size=(n, 3)) * sig[lab]
    pts = np.clip(pts, 0.0, np.nextafter(1.0, 0.0))
    return tuple(np.ascontiguousarray(pts[:, i].astype(dtype)) for i in range(3))


def jitter(xyz, sigma: float, seed: int, dtype=None):
    """Add N(0, sigma) to every coordinate, clamp to [0, 1-ulp] in the coordinate's precision."""
    rng = np.random.default_rng(seed)
    out = []
    for a in xyz:
        dt = dtype or a.dtype
        b = (a.astype(np.float64) + rng.normal(0.0, sigma, size=a.size)).astype(dt)
        b = np.clip(b, dt.type(0), np.nextafter(dt.type(1), dt.type(0)))
        out.append(np.ascontiguousarray(b))
    return tuple(out)
