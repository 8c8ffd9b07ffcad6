"""The C++ drop-in surface, used from C++ the way the reference's callers use it.

* tests/cpp/golden_regression.cu is a C++ caller in the style of the
  reference's regression test (tests/tree_test.cu:155-209): it includes
  include/adaptive_octree/tree.hpp, links libadaptive_trees_b200.so, builds
  and updates an Octree<double> and a Tree<double, Octree> facade on the
  Coulomb snapshots and assigns every getter to thrust::host_vector.  It is
  compiled with nvcc here (CPU) and run against the golden vectors (GPU).
* oracle/_ref/tree_example_b200 is the reference's own tests/tree_example.cu
  compiled unchanged against include/ and linked with the library (make -C
  oracle ref, where the reference checkout is present).  Its printed leaf and
  view-node counts and depth must equal those of the same tree built through
  the C ABI.
"""
import hashlib
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import refrun
from tests.golden.make_golden import load_expected, load_snapshots

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
LIBDIR = os.path.join(ROOT, "adaptive_trees_b200", "lib")
EXAMPLE = os.path.join(ROOT, "oracle", "_ref", "tree_example_b200")


@pytest.fixture(scope="module")
def golden_caller(tmp_path_factory):
    if not os.path.exists(NVCC) and not shutil.which("nvcc"):
        pytest.skip("nvcc not available")
    if not os.path.exists(os.path.join(LIBDIR, "libadaptive_trees_b200.so")):
        pytest.skip("library not built")
    out = str(tmp_path_factory.mktemp("cpp") / "golden_regression")
    cmd = [NVCC if os.path.exists(NVCC) else "nvcc", "-std=c++20", "-O2", "-gencode",
           "arch=compute_100a,code=sm_100a", f"-I{os.path.join(ROOT, 'include')}",
           os.path.join(ROOT, "tests", "cpp", "golden_regression.cu"), "-o", out, f"-L{LIBDIR}",
           "-ladaptive_trees_b200", "-Xlinker", "-rpath", "-Xlinker", LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    return out


def test_golden_regression_caller_compiles(golden_caller):
    assert os.access(golden_caller, os.X_OK)


def _torch_gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
def test_golden_regression_caller_matches_reference_vectors(golden_caller, tmp_path):
    _torch_gpu()
    (x0, y0, z0), (x1, y1, z1) = load_snapshots()
    frames = tmp_path / "frames.bin"
    with open(frames, "wb") as f:
        f.write(np.uint64(x0.size).tobytes())
        for a in (x0, y0, z0, x1, y1, z1):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    out = tmp_path / "out.bin"
    r = subprocess.run([golden_caller, str(frames), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    got = refrun.read_output(str(out))[0]
    meta, arrays = load_expected()
    for ref_name, spec in meta["arrays"].items():
        name = ref_name[:-2]  # particleKeys_d -> particleKeys
        if name not in got:
            continue
        a = got[name]
        assert a.size == spec["len"], name
        if ref_name in arrays:
            bad = np.nonzero(a != arrays[ref_name])[0]
            assert bad.size == 0, f"{name}: mismatches at {bad[:5]}"
        assert hashlib.sha256(a.tobytes()).hexdigest() == spec["sha256"], name
    assert got["scalars"][3] == meta["maxAchievedDepth"]


@pytest.mark.gpu
def test_reference_example_runs_unchanged_against_this_library(tmp_path):
    torch = _torch_gpu()
    if not os.path.exists(EXAMPLE):
        pytest.skip("oracle/_ref/tree_example_b200 not built (needs the reference checkout)")
    import adaptive_trees_b200 as ab
    (x, y, z), _ = load_snapshots()
    esc = np.finfo(np.float64).max
    path = tmp_path / "particles.dat"
    with open(path, "w") as f:
        f.write("# charge x y z\n")
        for a, b, c in zip(x.tolist(), y.tolist(), z.tolist()):
            f.write("ESC\n" if (a == esc and b == esc and c == esc) else f"0 {a!r} {b!r} {c!r}\n")
    r = subprocess.run([EXAMPLE, str(path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    built = next(line for line in lines if line.startswith("Built "))
    updated = next(line for line in lines if line.startswith("Updated "))
    leaves, nodes = int(built.split()[1]), int(built.split()[4])
    depth = int(built.rsplit("depth ", 1)[1].rstrip(")"))
    # the same tree through the C ABI: Binary, double, LeafCount 64, all views,
    # the default unit box grown to hold every active particle (tree_example.cu:27-45)
    act = ~((x == esc) & (y == esc) & (z == esc))
    box = (min(0.0, x[act].min()), max(1.0, x[act].max()), min(0.0, y[act].min()), max(1.0, y[act].max()),
           min(0.0, z[act].min()), max(1.0, z[act].max()))
    cfg = ab.TreeConfig(maxParticlesPerLeaf=64, box=box, views=ab.ViewConfig(True, True, True))
    xs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (x, y, z)]
    t = ab.Tree(1, *xs, cfg)
    t.build()
    assert (leaves, nodes, depth) == (t.info().num_leaves, t.numNodes(), t.maxAchievedDepth())
    t.update()
    while t.doBuffersNeedResize():
        t.resizeBuffers()
        t.update()
    assert int(updated.split()[1]) == t.info().num_leaves
    assert int(updated.split()[4]) == t.numActiveParticles()
    t.close()
