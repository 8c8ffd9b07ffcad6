"""Parity of the B200 engine with the reference library itself, on the same GPU.

The reference is compiled from its own sources into oracle/_ref/ref_driver
(make -C oracle ref).  Each scenario runs build(frame 0) and update(frame k)
with the resize loop in both implementations and compares every output array
bit for bit after each frame.  Sizes are scaled-down versions of the
benchmark configurations (uniform cube, Plummer sphere, Gaussian mixture) plus
non-unit boxes, which pin the float-to-grid quantisation.
"""
import numpy as np
import pytest

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


def run_engine(kind, frames, **cfg):
    import adaptive_trees_b200 as ab
    xs = [to_dev(a) for a in frames[0]]
    t = ab.Tree(kind, *xs, tree_config(**cfg))
    out = []
    for f, xyz in enumerate(frames):
        if f == 0:
            t.build()
        else:
            for d, a in zip(xs, xyz):
                d.copy_(torch.from_numpy(np.ascontiguousarray(a)).to("cuda"))
            t.update()
            k = 0
            while t.doBuffersNeedResize():
                k += 1
                assert k < 64
                t.resizeBuffers()
                t.update()
        t.doBuffersNeedResize()
        out.append({name: gpu_get(t, name) for name in refrun.ARRAY_NAMES if not (kind == 1 and
                                                                                     name == "nearFieldCounts")})
        out[-1]["info"] = t.info()
    return out


def check_frames(kind, frames, nf=False, **cfg):
    ref = refrun.run(kind, frames, nf=nf, views=(True, True, True), **cfg)
    ours = run_engine(kind, frames, nf=nf, views=(1, 1, 1), **cfg)
    assert len(ref) == len(ours)
    for f, (r, o) in enumerate(zip(ref, ours)):
        for name in refrun.ARRAY_NAMES:
            if name == "nearFieldCounts" and (kind == 1 or not nf):
                continue  # not computed by the reference outside NFCount octrees
            a, e = o[name], r[name]
            assert a.size == e.size, f"frame {f} {name}: size {a.size} != reference {e.size}"
            bad = np.nonzero(a != e)[0]
            assert bad.size == 0, f"frame {f} {name}: {bad.size} mismatches at {bad[:5]}: {a[bad[:5]]} vs {e[bad[:5]]}"
        sc = r["scalars"]
        info = o["info"]
        assert info.num_particles == sc[0] and info.num_active_particles == sc[1]
        assert info.num_nodes == sc[2] and info.max_achieved_depth == sc[3]


def jittered(xyz, sigma, steps, seed):
    frames = [xyz]
    for s in range(steps):
        frames.append(S.jitter(frames[-1], sigma, seed=seed + s))
    return frames


def test_reference_uniform_leafcount_fp64():
    frames = jittered(S.uniform_cube(1 << 17, seed=1), 1e-3, 2, 10)
    check_frames(0, frames, bucket=64)


def test_reference_plummer_nfcount_hilbert_fp32():
    frames = jittered(S.plummer_sphere(1 << 17, seed=2, dtype=np.float32), 1e-3, 2, 20)
    check_frames(0, frames, bucket=512, nf=True, hilbert=True)


def test_reference_mixture_binary_fp64():
    frames = jittered(S.gaussian_mixture(1 << 17, seed=3), 5e-4, 2, 30)
    check_frames(1, frames, bucket=32)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("hilbert", [False, True])
def test_reference_non_unit_box_quantisation(dtype, hilbert):
    box = (0.1, 2.3, -1.0, 1.0, 0.5, 0.75)
    rng = np.random.default_rng(17)
    lo, hi = np.array(box[0::2]), np.array(box[1::2])
    pts = lo + rng.random((50_000, 3)) * (hi - lo) * 0.999999
    xyz = tuple(np.ascontiguousarray(pts[:, i].astype(dtype)) for i in range(3))
    frames = jittered(xyz, 1e-4, 1, 40)
    frames = [tuple(np.clip(a, np.array(lo[i], dtype), np.array(hi[i] * 0.999999, dtype)) for i, a in enumerate(f))
              for f in frames]
    check_frames(0, frames, bucket=32, hilbert=hilbert, box=box)


def test_reference_binary_non_cubic_box_fp32():
    box = (0, 1, 0, 1.25, 0, 1.75)
    rng = np.random.default_rng(19)
    pts = rng.random((40_000, 3)) * np.array([1, 1.25, 1.75]) * 0.999
    xyz = tuple(np.ascontiguousarray(pts[:, i].astype(np.float32)) for i in range(3))
    check_frames(1, [xyz, S.jitter(xyz, 1e-3, seed=50)], bucket=16, box=box)
