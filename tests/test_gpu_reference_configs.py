"""Parity with the reference library at the benchmarked configurations.

The reference is compiled from its own sources into oracle/_ref/ref_driver
(make -C oracle ref) and runs on the same GPU and the same inputs as the
engine; each array of every frame is compared bit for bit (through a 64-bit
digest of its contents where the arrays run to hundreds of MB), as the
reference's regression test compares every buffer (tests/tree_test.cu:195-206).

The inputs are the benchmark's own generators (bench.py), at full size:
  * octree fp64, 2^20 particles i.i.d. U[0,1)^3 from default_rng(1), Morton,
    LeafCount 64, one build (all arrays, views on);
  * octree fp32, 16,777,216 Plummer particles (a = 0.05, r <= 0.5, seed 1234),
    Hilbert, NFCount 512, build + 2 updates with N(0, 1e-3) jitter;
  * binary k-d fp64, 8,388,608 particles from 8 anisotropic Gaussians
    (seed 3), LeafCount 32, build + 2 updates with N(0, 5e-4) jitter.
Each update runs the callers' resize loop (doBuffersNeedResize ->
resizeBuffers -> update), and the number of resizes must agree too.
"""
import numpy as np
import pytest

import bench
from oracle import refrun
from tests import scenarios as S
from tests.gpu_util import gpu_get, to_dev, tree_config

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not refrun.available():
        pytest.skip("reference driver oracle/_ref/ref_driver not built")


def engine_frames(kind, frames, digests, **cfg):
    """build(frame 0), update(frame k) with the resize loop; per frame the
    arrays (or their (count, digest)), the info and the cumulative resizes."""
    import adaptive_trees_b200 as ab
    xs = [to_dev(a) for a in frames[0]]
    t = ab.Tree(kind, *xs, tree_config(**cfg))
    out, resizes = [], 0
    for f, xyz in enumerate(frames):
        if f == 0:
            t.build()
        else:
            for d, a in zip(xs, xyz):
                d.copy_(torch.from_numpy(np.ascontiguousarray(a)).to("cuda"))
            t.update()
            while t.doBuffersNeedResize():
                resizes += 1
                assert resizes < 64
                t.resizeBuffers()
                t.update()
        t.doBuffersNeedResize()
        row = {}
        for name in refrun.ARRAY_NAMES:
            if kind == 1 and name == "nearFieldCounts":
                continue
            a = gpu_get(t, name)
            row[name] = (a.size, refrun.digest(a)) if digests else a
        row["info"] = t.info()
        row["resizes"] = resizes
        out.append(row)
    t.close()
    torch.cuda.synchronize()
    return out


def check_config(kind, frames, digests, nf=False, views=(False, False, False), **cfg):
    ref = refrun.run(kind, frames, digests=digests, nf=nf, views=tuple(bool(v) for v in views), timeout=3600,
                     **cfg)
    ours = engine_frames(kind, frames, digests, nf=nf, views=views, **cfg)
    assert len(ref) == len(ours) == len(frames)
    for f, (r, o) in enumerate(zip(ref, ours)):
        bad = []
        for name in refrun.ARRAY_NAMES:
            if name == "nearFieldCounts" and (kind == 1 or not nf):
                continue  # the reference computes it for NFCount octrees only
            a, e = o[name], r[name]
            if digests:
                if a != e:
                    bad.append(f"{name}: (size, digest) {a} != reference {e}")
            else:
                if a.size != e.size:
                    bad.append(f"{name}: size {a.size} != reference {e.size}")
                else:
                    idx = np.nonzero(a != e)[0]
                    if idx.size:
                        bad.append(f"{name}: {idx.size} mismatches at {idx[:5]}")
        assert not bad, f"frame {f}: " + "; ".join(bad)
        sc, info = r["scalars"], o["info"]
        assert (info.num_particles, info.num_active_particles, info.num_nodes, info.max_achieved_depth) == \
            tuple(sc[:4]), f"frame {f}: scalars {info} vs reference {sc}"
        assert o["resizes"] == sc[4], f"frame {f}: {o['resizes']} resizes, reference {sc[4]}"
    return ours


def jittered(xyz, sigma, steps, seed):
    frames = [xyz]
    for s in range(steps):
        frames.append(S.jitter(frames[-1], sigma, seed=seed + s))
    return frames


def test_reference_octree_uniform_2p20_fp64_morton_leafcount64():
    """One build from the root, P/Perm/K/N and every view array bit-exact."""
    n = 1 << 20
    r = np.random.default_rng(1)
    xyz = tuple(r.random(n) for _ in range(3))  # as bench.py's 2^20 workload
    out = check_config(0, [xyz], digests=False, bucket=64, views=(1, 1, 1))
    assert out[0]["info"].num_leaves > 20_000


def test_reference_octree_plummer_16mi_fp32_hilbert_nfcount512():
    """The benchmarked tree: build + 2 jittered updates, every array bit-exact."""
    xyz = bench.plummer(bench.N_DEFAULT, seed=1234)
    frames = jittered(xyz, 1e-3, 2, 700)
    out = check_config(0, frames, digests=True, bucket=bench.BUCKET, nf=True, hilbert=True)
    assert out[0]["info"].num_leaves > 10_000_000


def test_reference_binary_mixture_8mi_fp64_leafcount32():
    xyz = bench.mixture(1 << 23, 3)
    frames = jittered(xyz, 5e-4, 2, 800)
    out = check_config(1, frames, digests=True, bucket=32)
    assert out[0]["info"].num_leaves > 250_000
