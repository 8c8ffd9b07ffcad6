"""Per-particle data in key order (ao_tree_gather) and the leaf begin indices.

These are the first thing an FMM does with the tree: gather charges and
coordinates through perm_d, and take each leaf's particle range.
"""
import numpy as np
import pytest

from .gpu_util import gpu_get, to_np, tree_config
from .scenarios import gaussian_mixture, plummer_sphere


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [0, 1])
def test_leaf_begins_and_gather(kind):
    import torch

    import adaptive_trees_b200 as ab
    if kind == 0:
        xyz = plummer_sphere(30_000, 4, dtype=np.float32)
        cfg = tree_config(bucket=64, nf=True, hilbert=True)
    else:
        xyz = gaussian_mixture(30_000, 5, dtype=np.float64)
        cfg = tree_config(bucket=16)
    x = np.array(xyz[0])
    x[:100] = 2.0  # escaped particles keep their slots at the end of P
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (x, xyz[1], xyz[2])]
    t = ab.Tree(kind, *dev, cfg)
    t.build()
    t.doBuffersNeedResize()
    n_leaf = gpu_get(t, "leafCounts")
    begins = to_np(t.get("leafBegins_d"))
    assert begins.size == n_leaf.size + 1
    assert begins[0] == 0 and begins[-1] == t.numActiveParticles()
    assert np.array_equal(np.diff(begins.astype(np.int64)), n_leaf.astype(np.int64))

    perm = gpu_get(t, "perm").astype(np.int64)
    rng = np.random.default_rng(1)
    for host in (x, rng.random(x.size), rng.integers(0, 1 << 31, x.size).astype(np.int32),
                 rng.random((x.size, 2)), rng.random((x.size, 3)).astype(np.float32)):
        src = torch.from_numpy(np.ascontiguousarray(host)).cuda()
        out = t.gather(src).cpu().numpy()
        assert np.array_equal(out, host[perm]), host.dtype
    with pytest.raises(ValueError):
        t.gather(torch.zeros(5, device="cuda"))
