"""Benchmark of the B200 adaptive-tree engine on the 16Mi-particle octree workload.

Workload (one GPU): octree, 16,777,216 fp32 particles in a Plummer sphere
(scale 0.05, centre (0.5,0.5,0.5), truncated at r = 0.5), Hilbert keys,
NFCount refinement with near-field limit 512.  A step is one build() of the
tree from the root over the resident coordinates; the same run also times
graph-replayed update() steps on jittered coordinates (N(0, 1e-3), clamped to
the box).  Multi-GPU runs are replicas (one independent tree per GPU, no
collective on the path); the value is the total particles of all ranks over
the slowest rank's time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  --impl reference times the CPU oracle port of
the reference algorithm on a bounded sample (the reference has no CPU
implementation of this path); the reference library's own GPU time on this
box is reported by the default run under "reference_gpu", CUB's pair sort on
the same keys under "roofline" (the build's dominant kernel, the sort pass;
"roofline_update" is update()'s, the full near-field refresh), and bit-exact
parity of the timed tree with the reference library under "parity".  A single-GPU default run then
adds the metric's other configurations under "configs": c1 (2^20 uniform fp64
LeafCount octree), c3 (8Mi binary k-d tree), c4 (512 batched octrees against
a per-tree loop) and c5 (serving, --c5-seconds of requests), each with its
own clock record (--no-extras skips them).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 1 << 24
BUCKET = 512
METRIC = "particles/s (octree build, 16Mi Plummer fp32, Hilbert, NFCount 512)"
WORKLOAD = "octree build + graph-replayed update, 16Mi Plummer fp32 (a=0.05, r<=0.5), Hilbert keys, NFCount 512"
# DRAM bytes (read + write) of one 16Mi-key onesweep pass, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on that pass: 204.9 MB + 162.7 MB.
ONESWEEP_TRAFFIC_BYTES = 367.6e6
# Algorithmic bytes of the near-field refresh per leaf: K[i] read (8), the
# begin index B[i] read (4), NF[i] written (4), and the group flag, one byte
# per sibling group (1/8).
NF_BYTES_PER_LEAF = 16.125
# DRAM bytes (read + write) per leaf of the full near-field refresh, measured
# by ncu on that launch at 8 Mi particles (6,678,211 leaves); the traffic
# reported for the 16 Mi launch is this times its leaves (scaled, not
# re-measured in the run).
NF_TRAFFIC_BYTES_PER_LEAF = (292337664 + 30597888) / 6678211
# The arrays compared with the reference library in the line's parity record.
PARITY_ARRAYS = ("particleKeys", "perm", "cornerstone", "leafCounts", "nearFieldCounts")


def plummer(n, seed, scale=0.05, rmax=0.5):
    rng = np.random.default_rng(seed)
    out = np.empty((n, 3), dtype=np.float64)
    filled = 0
    while filled < n:
        m = int((n - filled) * 1.05) + 1024
        u = np.clip(rng.random(m), 1e-12, 1 - 1e-12)
        r = scale / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        r = r[r <= rmax]
        v = rng.normal(size=(r.size, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        take = min(r.size, n - filled)
        out[filled:filled + take] = v[:take] * r[:take, None] + 0.5
        filled += take
    np.clip(out, 0.0, np.nextafter(1.0, 0.0), out=out)
    return tuple(np.ascontiguousarray(out[:, i].astype(np.float32)) for i in range(3))


def rank_env():
    """(world size, rank, local rank) of a torchrun launch; (1, 0, 0) alone."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(v, world, device):
    """The slowest rank's value; every rank must call it (one all-reduce)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(total_units, slowest_ms):
    """Whole-job throughput: the units of all ranks over the slowest rank's time."""
    return total_units / (slowest_ms * 1e-3)


def partition_by_particles(sizes, world):
    """Owner rank of each independent system: largest first onto the least loaded rank.

    Systems never exchange data, so a rank builds and updates its share alone."""
    loads = [0] * world
    owner = [0] * len(sizes)
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        owner[i] = r
        loads[r] += int(sizes[i])
    return owner


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def wait_first(self, timeout=3.0):
        """Waits until nvidia-smi has printed its first sample, so a short
        timed region is still covered."""
        t0 = time.perf_counter()
        while self.proc and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle_build(n_sample, seed=7):
    """Single-threaded CPU port (oracle) of the reference build on a subset; particles/s."""
    from oracle import oracle as O
    x, y, z = plummer(n_sample, seed)
    cfg = O.make_config(max_particles_per_leaf=BUCKET, split_criterion=1, sfc_kind=1)
    t = O.OracleTree(0, x, y, z, cfg)
    t0 = time.perf_counter()
    t.build()
    dt = time.perf_counter() - t0
    return n_sample / dt, dt


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sample = args.cpu_sample
    vals = []
    for i in range(args.warmup + args.steps):
        v, _ = cpu_oracle_build(sample, seed=7 + i)
        if i >= args.warmup:
            vals.append(v)
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "particles/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sample / v * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": sample, "sample_of_n": args.n},
            "cpu_baseline": {"value": v, "unit": "particles/s", "cores": 1, "kind": "port",
                             "sample": f"one build of {sample} Plummer particles per step (CPU oracle port)"},
            "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def graph_ms(fn, stream, reps, warm=2):
    """Median device time of `fn` replayed from a CUDA graph (no host launch cost inside)."""
    import torch
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        fn()
    out = []
    for i in range(reps + warm):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        g.replay()
        b.record(stream)
        b.synchronize()
        if i >= warm:
            out.append(a.elapsed_time(b))
    del g
    return statistics.median(out)


class SortRig:
    """ao_sort_pairs on device keys with caller-owned scratch."""

    def __init__(self, keys, stream):
        import torch
        from adaptive_trees_b200 import _capi as C
        self.C, self.lib = C, C.load()
        self.n = keys.numel()
        self.keys = keys
        self.out = torch.empty_like(keys)
        self.vals = torch.empty(self.n, dtype=torch.uint32, device=keys.device)
        self.nbytes = ctypes.c_size_t()
        C.check(self.lib.ao_sort_pairs(None, ctypes.byref(self.nbytes), None, None, None, None, self.n, 0, 64, None))
        self.scratch = torch.empty(self.nbytes.value, dtype=torch.uint8, device=keys.device)
        self.stream = stream

    def __call__(self, end_bit=64):
        self.C.check(self.lib.ao_sort_pairs(ctypes.c_void_p(self.scratch.data_ptr()), ctypes.byref(self.nbytes),
                                            ctypes.c_void_p(self.keys.data_ptr()),
                                            ctypes.c_void_p(self.out.data_ptr()), None,
                                            ctypes.c_void_p(self.vals.data_ptr()), self.n, 0, end_bit,
                                            ctypes.c_void_p(self.stream.cuda_stream)))


def kernels_only(args):
    """Key generation and the 64-bit pair sort of the workload's keys, `reps` times each."""
    import torch
    import adaptive_trees_b200 as ab
    torch.cuda.set_device(0)
    s = torch.cuda.Stream()
    xs = [torch.from_numpy(a).cuda() for a in plummer(args.n, seed=1234)]
    with torch.cuda.stream(s):
        keys = ab.compute_sfc_keys(0, *xs, sfc_kind=ab.SfcKind.Hilbert, stream=s)
        rig = SortRig(keys, s)
        for _ in range(args.reps):
            ab.compute_sfc_keys(0, *xs, sfc_kind=ab.SfcKind.Hilbert, stream=s)
            rig(64)
    s.synchronize()
    print(json.dumps({"mode": "kernels", "n": args.n, "reps": args.reps}))
    return 0


def build_only(args):
    """One build and one update of the workload's tree at size --n (the
    default sort configuration, no tuning runs, so a profile sees only them)."""
    import torch
    import adaptive_trees_b200 as ab
    torch.cuda.set_device(0)
    ab.set_sort_autotune(False)
    s = torch.cuda.Stream()
    xs = [torch.from_numpy(a).cuda() for a in plummer(args.n, seed=1234)]
    cfg = ab.TreeConfig(maxParticlesPerLeaf=BUCKET, splitCriterion=ab.SplitCriterion.NFCount,
                        sfcKind=ab.SfcKind.Hilbert)
    with torch.cuda.stream(s):
        t = ab.Tree(0, *xs, cfg, stream=s)
        t.build()
        for x in xs:
            x.add_(1e-3 * torch.randn_like(x)).clamp_(0.0, 0.99999994)
        t.update()
        t.doBuffersNeedResize()
    s.synchronize()
    print(json.dumps({"mode": "build", "n": args.n, "leaves": t.info().num_leaves}))
    return 0


# The two other single-tree configurations (measured on request; the default
# line is C2).  kind 0 octree / 1 binary; updates with N(0, jitter) per step.
SINGLE_CONFIGS = {
    "c1": {"metric": "particles/s (octree build, 2^20 uniform fp64, Morton, LeafCount 64)",
           "workload": "octree, 1,048,576 fp64 particles i.i.d. U[0,1)^3 (default_rng(1)), Morton, LeafCount 64; "
                       "one build from the root",
           "kind": 0, "n": 1 << 20, "bucket": 64, "updates": 0, "jitter": 0.0},
    "c3": {"metric": "particles/s (binary k-d build, 8Mi Gaussian mixture fp64, LeafCount 32)",
           "workload": "binary k-d tree, 8,388,608 fp64 particles from 8 anisotropic Gaussians (centres "
                       "U[0.2,0.8]^3, sigma log-uniform [0.005,0.05], seed 3), LeafCount 32; build + 10 "
                       "graph-replayed updates with N(0, 5e-4) jitter",
           "kind": 1, "n": 1 << 23, "bucket": 32, "updates": 10, "jitter": 5e-4},
}


def mixture(n, seed, clusters=8):
    """Equal-weight mixture of anisotropic Gaussians, clamped to [0, 1)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2, 0.8, size=(clusters, 3))
    sigmas = np.exp(rng.uniform(np.log(0.005), np.log(0.05), size=(clusters, 3)))
    which = rng.integers(0, clusters, size=n)
    pts = centres[which] + sigmas[which] * rng.normal(size=(n, 3))
    np.clip(pts, 0.0, np.nextafter(1.0, 0.0), out=pts)
    return tuple(np.ascontiguousarray(pts[:, i]) for i in range(3))


def single_config_bench(args):
    """C1 / C3 as their own line."""
    line = single_config_record(args.config, args.steps, args.warmup, args.cpu_sample, not args.no_cpu_baseline,
                                not args.no_reference_gpu)
    print(json.dumps(line), flush=True)
    return 0


def single_config_record(config, steps, warmup, cpu_sample, cpu_baseline=True, reference_gpu=True):
    """C1 / C3: one tree of the configuration, next to the reference library on the same GPU."""
    import torch

    import adaptive_trees_b200 as ab
    from types import SimpleNamespace
    args = SimpleNamespace(config=config, steps=steps, warmup=warmup, cpu_sample=cpu_sample,
                           no_cpu_baseline=not cpu_baseline, no_reference_gpu=not reference_gpu)
    spec = SINGLE_CONFIGS[args.config]
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    s = torch.cuda.Stream(device=dev)
    n = spec["n"]
    if spec["kind"] == 0:
        r = np.random.default_rng(1)
        hx = tuple(r.random(n) for _ in range(3))
    else:
        hx = mixture(n, 3)
    pinned = [torch.from_numpy(a).pin_memory() for a in hx]
    xs = [p.to(dev) for p in pinned]
    torch.cuda.synchronize()
    cfg = ab.TreeConfig(maxParticlesPerLeaf=spec["bucket"])
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn):
        a, b = ev(), ev()
        a.record(s)
        fn()
        b.record(s)
        b.synchronize()
        return a.elapsed_time(b)

    with torch.cuda.stream(s):
        tree = ab.Tree(spec["kind"], *xs, cfg, stream=s)
        for _ in range(args.warmup):
            tree.build()
        launches0 = tree.info().kernel_launches
        with ClockSampler(0) as clocks:
            # at least half a second of builds, so the clock record covers them
            clocks.wait_first()
            build_ms, t0 = [], time.perf_counter()
            while len(build_ms) < args.steps or time.perf_counter() - t0 < 0.5:
                build_ms.append(timed(tree.build))
        launches = (tree.info().kernel_launches - launches0) // max(1, len(build_ms))
        info = tree.info()
        leaves = info.num_leaves
        by_levels, passes = tree.buildPath()
        # end to end: pinned host coordinates in, build, the counters out
        host_counters = torch.zeros(3, dtype=torch.int32).pin_memory()
        cnt = tree.counters()

        def e2e_step():
            for d, p in zip(xs, pinned):
                d.copy_(p, non_blocking=True)
            tree.build()
            for k, (ptr, ts) in enumerate(zip(cnt, ("<i4", "<i4", "<u4"))):
                host_counters[k:k + 1].copy_(ab.device_tensor(ptr, 1, ts).view(torch.int32), non_blocking=True)
        e2e_ms = statistics.median([timed(e2e_step) for _ in range(args.steps)])
        update_ms, resizes = [], 0
        frame1 = None
        if spec["updates"]:
            gen = torch.Generator(device=dev)
            gen.manual_seed(31)
            upper = float(np.nextafter(1.0, 0.0))

            def jitter():
                for t in xs:
                    t.add_(torch.randn(t.shape, generator=gen, device=dev, dtype=t.dtype) * spec["jitter"])
                    t.clamp_(0.0, upper)

            def capture():
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=s):
                    tree.update()
                return g
            tree.build()
            graph = capture()
            for i in range(spec["updates"]):
                jitter()
                s.synchronize()
                if frame1 is None:
                    frame1 = tuple(t.cpu().numpy() for t in xs)
                update_ms.append(timed(graph.replay))
                if tree.doBuffersNeedResize():
                    resizes += 1
                    del graph
                    tree.resizeBuffers()
                    tree.update()
                    graph = capture()
            del graph
    line = {"metric": spec["metric"], "value": n / (statistics.median(build_ms) * 1e-3), "unit": "particles/s",
            "n_gpus": 1, "steps": len(build_ms), "warmup": args.warmup, "ms_per_step": statistics.median(build_ms),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": spec["workload"], "n": n, "coords": "float64", "leaves": int(leaves),
                       "parallelism": "replicas1", "sort": ab.sort_tuning(n),
                       "build_path": {"by_levels": bool(by_levels), "reference_rounds": int(passes)}},
            "clocks": clocks.summary(), "gpu_launches": int(launches),
            "e2e": {"value": n / (e2e_ms * 1e-3), "unit": "particles/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": 3 * 8 * n, "d2h_bytes_per_step": 12}}
    if update_ms:
        um = statistics.median(update_ms)
        line["update"] = {"value": n / (um * 1e-3), "unit": "particles/s", "ms_per_step": um,
                          "graph_replayed": True, "resizes": resizes, "steps": len(update_ms)}
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        m = min(n, args.cpu_sample)
        t = O.OracleTree(spec["kind"], *(a[:m] for a in hx), O.make_config(max_particles_per_leaf=spec["bucket"]))
        t0 = time.perf_counter()
        t.build()
        line["cpu_baseline"] = {"value": m / (time.perf_counter() - t0), "unit": "particles/s", "cores": 1,
                                "kind": "port", "sample": f"one build of the first {m} particles (CPU oracle port)"}
    if not args.no_reference_gpu:
        try:
            from oracle import refrun
            if refrun.available():
                frames = [hx, frame1 if frame1 is not None else hx]
                r = refrun.time_reference(spec["kind"], frames, reps=3, bucket=spec["bucket"],
                                          views=(False, False, False))
                line["reference_gpu"] = {"build_ms": r["build_ms"], "update_ms": r["update_ms"],
                                         "build_value": n / (r["build_ms"] * 1e-3), "unit": "particles/s",
                                         "what": "reference library compiled for sm_100a, same inputs and GPU"}
        except Exception as e:  # informational
            line["reference_gpu"] = {"error": str(e)[:200]}
    tree.close()
    return line


C4_SYSTEMS = 512
C4_METRIC = "particles/s (batched octree build, 512 systems, fp32, Morton, LeafCount 64)"
C4_WORKLOAD = ("512 independent octrees, sizes floor(10^U(3,6)) (seed 4), fp32 uniform or Plummer (coin flip per "
               "system), Morton keys, LeafCount 64; one batched build and 10 graph-replayed batched updates "
               "(N(0,1e-3) jitter) against a loop of plain per-tree build()/update() on the same inputs")


def c4_systems():
    rng = np.random.default_rng(4)
    sizes = np.floor(10.0 ** rng.uniform(3.0, 6.0, C4_SYSTEMS)).astype(np.int64)
    plum = rng.random(C4_SYSTEMS) < 0.5
    return sizes, plum


def batched_bench(args):
    """C4 as its own line (every rank; rank 0 prints)."""
    line, same = batched_record(args.steps, args.warmup)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0 if same else 1


def batched_record(steps, warmup, distributed=True):
    """C4: Batch (one set of launches for all systems) against a loop of plain trees.

    Returns (line or None on ranks other than 0, identical outputs)."""
    import torch
    import torch.distributed as dist

    import adaptive_trees_b200 as ab
    from types import SimpleNamespace
    args = SimpleNamespace(steps=steps, warmup=warmup)
    world, rank, local = rank_env() if distributed else (1, 0, 0)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    s = torch.cuda.Stream(device=dev)
    sizes_all, plum_all = c4_systems()
    # systems never exchange data: each rank takes a particle-balanced share
    owner = partition_by_particles(sizes_all, world)
    mine = [k for k in range(C4_SYSTEMS) if owner[k] == rank]
    sizes, plum = sizes_all[mine], plum_all[mine]
    total_all = int(sizes_all.sum())
    total = int(sizes.sum())
    offs = np.concatenate([[0], np.cumsum(sizes)])
    host = [np.empty(total, np.float32) for _ in range(3)]
    for j, k in enumerate(mine):
        n = int(sizes[j])
        if plum[k]:
            xyz = plummer(n, 100 + k)
        else:
            r = np.random.default_rng(100 + k)
            xyz = tuple(r.random(n, dtype=np.float32) for _ in range(3))
        for a in range(3):
            host[a][offs[j]:offs[j + 1]] = xyz[a]
    allc = [torch.from_numpy(h).to(dev) for h in host]
    views = [[c[offs[j]:offs[j + 1]] for c in allc] for j in range(len(mine))]
    cfg = ab.TreeConfig(maxParticlesPerLeaf=64)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn):
        a, b = ev(), ev()
        a.record(s)
        fn()
        b.record(s)
        b.synchronize()
        return a.elapsed_time(b)

    names = ("particleKeys_d", "perm_d", "cornerstone_d", "leafCounts_d")

    def identical(batch, trees):
        batch.doBuffersNeedResize()
        for k, t in enumerate(trees):
            t.doBuffersNeedResize()
            for nm in names:
                a, b = batch.get(k, nm), t.get(nm)
                if a.numel() != b.numel() or not torch.equal(a.view(torch.uint8), b.view(torch.uint8)):
                    return False
        return True

    with torch.cuda.stream(s):
        batch = ab.Batch([v[0] for v in views], [v[1] for v in views], [v[2] for v in views], cfg, stream=s)
        trees = [ab.Tree(0, *v, cfg, stream=s) for v in views]
        launches = lambda: trees[0].info().kernel_launches  # noqa: E731  (process-wide counter)
        for _ in range(args.warmup):
            batch.build()
            for t in trees:
                t.build()
        l0 = launches()
        clocks = ClockSampler(local)
        clocks.__enter__()
        b_build = [timed(batch.build) for _ in range(args.steps)]
        batch_launches = launches() - l0

        def plain_build():
            for t in trees:
                t.build()
        p_build = [timed(plain_build) for _ in range(args.steps)]
        same = identical(batch, trees)

        gen = torch.Generator(device=dev)
        gen.manual_seed(77)

        def jitter():
            for c in allc:
                c.add_(torch.randn(c.shape, generator=gen, device=dev, dtype=c.dtype) * 1e-3).clamp_(0.0, 0.99999994)

        def capture():
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                batch.update()
            return g

        graph = capture()
        b_upd, p_upd, resizes = [], [], 0

        def plain_update():
            for t in trees:
                t.update()
        for _ in range(10):
            jitter()
            s.synchronize()
            b_upd.append(timed(graph.replay))
            p_upd.append(timed(plain_update))
            flags = [t.doBuffersNeedResize() for t in trees]
            if batch.doBuffersNeedResize() or any(flags):
                resizes += 1
                for t, f in zip(trees, flags):
                    if f:
                        t.resizeBuffers()
                        t.update()
                batch.resizeBuffers()
                batch.update(frozen=[not f for f in flags])
                del graph
                graph = capture()
            same = same and identical(batch, trees)
        clocks.__exit__(None, None, None)
        del graph
        batch.close()
        for t in trees:
            t.close()
    bb = max_over_ranks(statistics.median(b_build), world, dev)
    pb = max_over_ranks(statistics.median(p_build), world, dev)
    bu = max_over_ranks(statistics.median(b_upd), world, dev)
    pu = max_over_ranks(statistics.median(p_upd), world, dev)
    same = max_over_ranks(0.0 if same else 1.0, world, dev) == 0.0
    sort_choice = ab.sort_tuning(total, segmented=True)
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return None, same
    line = {"metric": C4_METRIC, "value": job_rate(total_all, bb), "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": bb, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": C4_WORKLOAD, "systems": C4_SYSTEMS, "particles": total_all,
                       "largest": int(sizes_all.max()), "smallest": int(sizes_all.min()),
                       "parallelism": f"systems partitioned over {world} rank(s), no collective on the path",
                       "sort": sort_choice},
            "batched": {"build_ms": bb, "update_ms": bu, "build_value": job_rate(total_all, bb),
                        "update_value": job_rate(total_all, bu), "update_graph_replayed": True,
                        "build_launches": batch_launches // max(1, args.steps)},
            "plain_loop": {"build_ms": pb, "update_ms": pu, "build_value": job_rate(total_all, pb),
                           "update_value": job_rate(total_all, pu)},
            "speedup": {"build": pb / bb, "update": pu / bu}, "identical_outputs": bool(same), "resizes": resizes,
            "clocks": clocks.summary()}
    return line, same


C5_METRIC = "particles/s served (Poisson 2000 req/s, 30% builds / 70% updates, 120 GB budget)"


def serving_bench(args):
    """C5 as its own line."""
    line = serving_record(args.duration, args.warm_seconds, args.slots, args.live_trees)
    print(json.dumps(line), flush=True)
    return 0 if not line["requests"]["failed"] else 1


def serving_record(duration, warm_seconds, slots, live_trees):
    """C5: a Server fed by an open-loop Poisson client; latency from submit to result."""
    import torch

    import adaptive_trees_b200 as ab
    from types import SimpleNamespace
    args = SimpleNamespace(duration=duration, warm_seconds=warm_seconds, slots=slots, live_trees=live_trees)
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rate, budget, max_n = 2000.0, 120 << 30, 4_000_000
    rng = np.random.default_rng(5)
    # coordinate pools: per distribution one base set and four jittered copies
    pools = {}
    for dist in ("uniform", "plummer"):
        if dist == "plummer":
            base = plummer(max_n, 55)
        else:
            r = np.random.default_rng(56)
            base = tuple(r.random(max_n, dtype=np.float32) for _ in range(3))
        versions = [tuple(torch.from_numpy(a).to(dev) for a in base)]
        g = torch.Generator(device=dev)
        g.manual_seed(57)
        for _ in range(4):
            versions.append(tuple((t + torch.randn(t.shape, generator=g, device=dev) * 1e-3).clamp_(0.0, 0.99999994)
                                  for t in versions[0]))
        pools[dist] = versions
    torch.cuda.synchronize()

    def make_requests(seconds, first_id):
        """Arrival times and requests of an open-loop client over `seconds`."""
        reqs, live, t, tid = [], [], 0.0, first_id
        while True:
            t += rng.exponential(1.0 / rate)
            if t >= seconds:
                break
            if not live or rng.random() < 0.3:
                n = int(10 ** rng.uniform(4.0, np.log10(max_n)))
                dist = "plummer" if rng.random() < 0.5 else "uniform"
                nf = rng.random() < 0.5
                cfg = ab.TreeConfig(maxParticlesPerLeaf=512 if nf else 64,
                                    splitCriterion=ab.SplitCriterion.NFCount if nf else ab.SplitCriterion.LeafCount,
                                    sfcKind=ab.SfcKind.Hilbert if rng.random() < 0.5 else ab.SfcKind.Morton)
                off = int(rng.integers(0, max_n - n + 1))
                if len(live) >= args.live_trees:
                    reqs.append((t, ("release", live.pop(0))))
                live.append((tid, dist, n, off, [0]))
                reqs.append((t, ("build", live[-1], cfg)))
                tid += 1
            else:
                tr = live[int(rng.integers(0, len(live)))]
                tr[4][0] = tr[4][0] % 4 + 1
                reqs.append((t, ("update", tr, tr[4][0])))
        return reqs, live, tid

    def submit(server, req):
        kind = req[0]
        if kind == "release":
            return server.release(req[1][0])
        tid, dist, n, off, _ = req[1]
        v = 0 if kind == "build" else req[2]
        xyz = [a[off:off + n] for a in pools[dist][v]]
        if kind == "build":
            return server.build(tid, *xyz, config=req[2])
        return server.update(tid, *xyz)

    def play(server, reqs):
        t0 = time.perf_counter()
        tickets, late = [], []
        for at, req in reqs:
            while True:
                dt = at - (time.perf_counter() - t0)
                if dt <= 0:
                    break
                time.sleep(min(dt, 0.002) if dt > 0.0005 else 0)
            late.append(-dt)
            tickets.append(submit(server, req))
        server.drain()
        return tickets, late

    server = ab.Server(slots=args.slots, memory_budget_bytes=budget)
    warm, live, next_id = make_requests(args.warm_seconds, 0)
    play(server, warm)[0]
    for tr in live:
        server.release(tr[0])
    server.drain()
    server.reset_stats()
    reqs, live, _ = make_requests(args.duration, next_id)
    with ClockSampler(0) as clocks:
        tickets, late = play(server, reqs)
    st = server.stats()
    results = [server.wait(k) for k in tickets]
    failed = [r["message"] for r in results if r["status"] != 0]
    # latency by second of arrival: a steady tail or bursts
    per_second = []
    for sec in range(int(np.ceil(args.duration))):
        lat = [r["latency_ms"] for (at, _), r in zip(reqs, results) if sec <= at < sec + 1 and r["status"] == 0]
        if lat:
            per_second.append([round(float(np.percentile(lat, 50)), 2), round(float(np.percentile(lat, 99)), 2)])
    offered = sum(r[1][1][2] for r in reqs if r[1][0] != "release")
    server.close()
    line = {"metric": C5_METRIC, "value": st["particles_per_s"], "unit": "particles/s", "n_gpus": 1,
            "steps": len(reqs), "warmup": len(warm), "ms_per_step": st["mean_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "C5 serving: open-loop Poisson client, 2000 req/s, 30% builds of new trees / "
                                   "70% updates of live trees, sizes floor(10^U(4, log10 4e6)), fp32 uniform or "
                                   "Plummer, Morton or Hilbert, LeafCount 64 or NFCount 512; 120 GB budget",
                       "duration_s": args.duration, "slots": args.slots, "live_trees": args.live_trees,
                       "parallelism": "replicas1"},
            "latency": {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                        "max_ms": st["max_ms"]},
            "requests": {"completed": st["completed"], "failed": st["failed"], "first_failures": failed[:3]},
            "latency_by_second_p50_p99": per_second,
            "client_late_ms": {"p50": float(np.percentile(late, 50)) * 1e3, "max": float(max(late)) * 1e3},
            "host_cpus": os.cpu_count(),
            "offered_particles_per_s": offered / args.duration, "span_s": st["span_s"],
            "peak_bytes": st["peak_bytes"], "clocks": clocks.summary()}
    if args.duration < 60:
        line["config"]["window_note"] = (f"{args.duration:g} s of requests, shorter than the configured 60 s, "
                                         "to keep the default benchmark run within minutes")
    return line


def reference_parity(tree, xs, frames, stream):
    """Bit-exact check of the timed tree against the reference library.

    The timed tree is built again from frame 0 (the benchmark's coordinates)
    and updated on frame 1 with the callers' resize loop; the reference
    library (oracle/_ref/ref_driver, compiled from the reference's sources)
    runs build + update on the same frames.  Every array of PARITY_ARRAYS is
    compared through its 64-bit content digest after each frame, with the
    tree's scalars and the resize count."""
    import torch

    from oracle import refrun
    ours, resizes = [], 0
    for f, fr in enumerate(frames):
        for d, a in zip(xs, fr):
            d.copy_(torch.from_numpy(a), non_blocking=False)
        if f == 0:
            tree.build()
        else:
            tree.update()
            while tree.doBuffersNeedResize():
                resizes += 1
                tree.resizeBuffers()
                tree.update()
        tree.doBuffersNeedResize()
        stream.synchronize()
        row = {}
        for name in PARITY_ARRAYS:
            t = tree.get(name + "_d")
            wide = {torch.uint64: torch.int64, torch.uint32: torch.int32}.get(t.dtype)
            a = t.view(wide).cpu().numpy() if wide is not None else t.cpu().numpy()
            row[name] = (int(a.size), refrun.digest(a))
        info = tree.info()
        row["scalars"] = (info.num_particles, info.num_active_particles, info.num_nodes, info.max_achieved_depth,
                          resizes)
        ours.append(row)
    ref = refrun.run(0, frames, digests=True, bucket=BUCKET, nf=True, hilbert=True, views=(False, False, False),
                     timeout=1800)
    mismatches = []
    for f, (o, r) in enumerate(zip(ours, ref)):
        for name in PARITY_ARRAYS:
            if o[name] != tuple(r[name]):
                mismatches.append(f"frame {f} {name}")
        if tuple(o["scalars"]) != tuple(r["scalars"][:5]):
            mismatches.append(f"frame {f} scalars {o['scalars']} vs {tuple(r['scalars'][:5])}")
    return {"ref_lib_bit_exact": not mismatches and len(ref) == len(ours), "frames": ["build", "update"],
            "buffers": list(PARITY_ARRAYS), "mismatches": mismatches[:8],
            "how": "64-bit content digests of the timed tree's arrays vs the reference library compiled for "
                   "sm_100a (oracle/_ref/ref_driver), same coordinates, build then update(N(0,1e-3) jitter)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--cpu-sample", type=int, default=1 << 20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--mode", default="bench", choices=["bench", "kernels", "build"],
                    help="kernels: only key generation + the 64-bit pair sort of the workload's keys; "
                         "build: one build + one update of the workload's tree (small commands for ncu)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: the 16Mi NFCount octree (headline); c1: 2^20 uniform fp64 LeafCount octree; "
                         "c3: 8Mi fp64 binary k-d tree; c4: 512 batched octrees vs a per-tree loop; "
                         "c5: serving under a Poisson request stream")
    ap.add_argument("--duration", type=float, default=10.0, help="c5: seconds of requests")
    ap.add_argument("--warm-seconds", type=float, default=2.0, help="c5: seconds of untimed requests first")
    ap.add_argument("--slots", type=int, default=32, help="c5: server worker threads")
    ap.add_argument("--live-trees", type=int, default=256, help="c5: resident trees the client keeps")
    ap.add_argument("--no-extras", action="store_true",
                    help="default run: skip the c1/c3/c4/c5 records that follow the headline")
    ap.add_argument("--c5-seconds", type=float, default=20.0, help="default run: seconds of the c5 record")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.mode == "kernels":
        return kernels_only(args)
    if args.mode == "build":
        return build_only(args)
    if args.config in SINGLE_CONFIGS:
        return single_config_bench(args)
    if args.config == "c4":
        return batched_bench(args)
    if args.config == "c5":
        return serving_bench(args)

    import torch
    import torch.distributed as dist

    import adaptive_trees_b200 as ab
    from adaptive_trees_b200 import _capi as C

    world, rank, local = rank_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    s = torch.cuda.Stream(device=dev)
    n = args.n
    hx = plummer(n, seed=1234 + rank)
    pinned = [torch.from_numpy(a).pin_memory() for a in hx]
    xs = [p.to(dev) for p in pinned]
    torch.cuda.synchronize()
    cfg = ab.TreeConfig(maxParticlesPerLeaf=BUCKET, splitCriterion=ab.SplitCriterion.NFCount,
                        sfcKind=ab.SfcKind.Hilbert)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    with torch.cuda.stream(s):
        tree = ab.Tree(0, *xs, cfg, stream=s)
        # ---------------- warm-up builds
        for _ in range(args.warmup):
            tree.build()
        s.synchronize()
        launches0 = tree.info().kernel_launches
        # ---------------- timed builds (inputs 192 MiB > L2: no flush needed)
        barrier()
        build_ms = []
        # clocks are sampled across the timed builds, updates and end-to-end steps
        clocks = ClockSampler(local)
        clocks.__enter__()
        for _ in range(args.steps):
            a, b = ev(), ev()
            a.record(s)
            tree.build()
            b.record(s)
            b.synchronize()
            build_ms.append(a.elapsed_time(b))
        barrier()
        launches = tree.info().kernel_launches - launches0
        info = tree.info()
        leaves = info.num_leaves

        # ---------------- graph-replayed updates
        gen = torch.Generator(device=dev)
        gen.manual_seed(99 + rank)
        upper = float(np.nextafter(np.float32(1.0), np.float32(0.0)))

        def jitter():
            for t in xs:
                t.add_(torch.randn(t.shape, generator=gen, device=dev, dtype=t.dtype) * 1e-3).clamp_(0.0, upper)

        def capture():
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                tree.update()
            return g

        jitter()
        tree.update()
        while tree.doBuffersNeedResize():
            tree.resizeBuffers()
            tree.update()
        graph = capture()
        update_ms, resizes = [], 0
        for i in range(args.warmup + args.steps):
            jitter()
            s.synchronize()
            a, b = ev(), ev()
            a.record(s)
            graph.replay()
            b.record(s)
            b.synchronize()
            if i >= args.warmup:
                update_ms.append(a.elapsed_time(b))
            if tree.doBuffersNeedResize():
                resizes += 1
                del graph
                tree.resizeBuffers()
                tree.update()
                graph = capture()
        del graph

        # ---------------- end to end: host coordinates -> build -> counters to host
        cnt_ptr = tree.counters()
        host_counters = torch.zeros(3, dtype=torch.int32).pin_memory()
        e2e_ms = []
        for i in range(args.warmup + args.steps):
            a, b = ev(), ev()
            a.record(s)
            for d, p in zip(xs, pinned):
                d.copy_(p, non_blocking=True)
            tree.build()
            nl = ab.device_tensor(cnt_ptr[0], 1, "<i4")
            nn = ab.device_tensor(cnt_ptr[1], 1, "<i4")
            na = ab.device_tensor(cnt_ptr[2], 1, "<u4").view(torch.int32)
            host_counters[0:1].copy_(nl, non_blocking=True)
            host_counters[1:2].copy_(nn, non_blocking=True)
            host_counters[2:3].copy_(na, non_blocking=True)
            b.record(s)
            b.synchronize()
            if i >= args.warmup:
                e2e_ms.append(a.elapsed_time(b))
        assert int(host_counters[0]) == leaves

        clocks.__exit__(None, None, None)

        # ---------------- stage times and the near-field kernel, timed with
        # the tree's own CUDA events on its stream (direct calls, not graphs)
        tree.setProfiling(True)
        build_stages, update_stages = [], []
        for i in range(args.warmup + args.steps):
            tree.build()
            bst = tree.stageTimes()
            jitter()
            tree.update()
            ust = tree.stageTimes()
            if tree.doBuffersNeedResize():
                tree.resizeBuffers()
                tree.update()
            if i >= args.warmup:
                build_stages.append(bst)
                update_stages.append(ust)
        tree.setProfiling(False)
        nf_leaves = tree.info().num_leaves
        sort_choice = ab.sort_tuning(n)

        # ---------------- roofline: onesweep pass timed live via ao_sort_pairs,
        # replayed from CUDA graphs so no host launch time is inside the events
        # the keys as the build's sort receives them: unsorted, from the coordinates
        keys_in = ab.compute_sfc_keys(0, *xs, sfc_kind=ab.SfcKind.Hilbert, stream=s)
        s.synchronize()
        rig = SortRig(keys_in, s)
        t64 = graph_ms(lambda: rig(64), s, 7)
        t8 = graph_ms(lambda: rig(8), s, 7)
        pass_ms = (t64 - t8) / 7.0
        keygen_ms = graph_ms(lambda: ab.compute_sfc_keys(0, *xs, sfc_kind=ab.SfcKind.Hilbert, stream=s), s, 7)
    barrier()

    step_ms = max_over_ranks(statistics.median(build_ms), world, dev)
    upd_ms = max_over_ranks(statistics.median(update_ms), world, dev)
    e2e = max_over_ranks(statistics.median(e2e_ms), world, dev)
    total = n * world
    hbm, peak_kind = peaks()
    pass_bytes = 24.0 * n
    achieved = pass_bytes / (pass_ms * 1e-3) / 1e9
    # the dominant kernel of the timed step: one build runs 8 onesweep passes,
    # 38 % of its device time, more than any other kernel
    roof_sort = {"bound": "hbm", "kernel": "onesweepKernel (one 8-bit pass of the 64-bit key + 32-bit value sort)",
                 "why": "the build's dominant kernel: 8 launches per build, 1.33 of 3.61 ms serialised device time",
                 "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                 "traffic": ONESWEEP_TRAFFIC_BYTES, "traffic_kind": "ncu capture of one 16Mi pass, not re-measured",
                 "algorithmic_bytes_per_launch": pass_bytes,
                 "launch_ms": pass_ms, "sort_64bit_ms": t64,
                 "keygen": {"ms": keygen_ms, "achieved_gbs": (20.0 * n) / (keygen_ms * 1e-3) / 1e9}}
    if rank == 0 and not args.no_reference_gpu:
        try:
            from oracle import refrun
            if refrun.available():
                kh = keys_in.view(torch.int64).cpu().numpy().view(np.uint64)
                cub = refrun.time_cub_sort(kh, reps=10)
                roof_sort["cub_sort_64bit_ms"] = cub["cub_sort_ms"]
                roof_sort["cub_what"] = ("cub::DeviceRadixSort::SortPairs (CCCL 3.3, the reference's call, "
                                         "octree.cu:301-304) on the same unsorted keys, same GPU")
        except Exception as e:  # informational
            roof_sort["cub_error"] = str(e)[:200]

    def med(rows, key):
        return statistics.median(r[key] for r in rows)

    # the dominant kernel of update(): the near-field refresh.  Its full
    # launch covers every leaf, so its algorithmic bytes are known exactly.
    nf_ms = max_over_ranks(med(update_stages, "near_field_first_ms"), world, dev)
    nf_bytes = NF_BYTES_PER_LEAF * nf_leaves
    nf_achieved = nf_bytes / (nf_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": "octNearFieldKernel<Hilbert, All> (the full near-field refresh of update())",
            "achieved": nf_achieved, "peak": hbm, "unit": "GB/s", "frac": nf_achieved / hbm, "peak_kind": peak_kind,
            "traffic": (NF_TRAFFIC_BYTES_PER_LEAF * nf_leaves) if NF_TRAFFIC_BYTES_PER_LEAF else None,
            "algorithmic_bytes_per_launch": nf_bytes, "launch_ms": nf_ms, "leaves": nf_leaves,
            "note": "search-bound: 27 neighbour-cell populations per parent cell come from hash tables or "
                    "searches of the sorted keys; HBM is the roof, not the limit"}
    stages = {
        "build": {k: med(build_stages, k) for k in ("keys_and_sort_ms", "passes_ms", "finish_ms", "total_ms",
                                                     "near_field_ms")},
        "update": {k: med(update_stages, k) for k in ("keys_and_sort_ms", "refresh_ms", "passes_ms", "finish_ms",
                                                      "total_ms", "near_field_ms", "near_field_first_ms")},
        "build_near_field_launches": build_stages[-1]["near_field_launches"],
        "update_near_field_launches": update_stages[-1]["near_field_launches"],
        "how": "CUDA events on the tree's stream around each stage (ao_tree_set_profiling), direct calls"}
    # the whole build on the byte model of the path: per particle the
    # coordinates read (3 x 4 B), key + index written (12 B), the upfront
    # histogram read (8 B), 24 B per radix pass (8 passes), one streaming read
    # of the sorted keys (8 B); per leaf K and N written (12 B)
    model_bytes = n * (3 * 4 + 12 + 8 + 24 * 8 + 8) + 12 * leaves
    model_gbs = model_bytes / (step_ms * 1e-3) / 1e9
    roof_build = {"bound": "hbm", "what": "whole build() on the byte model N(3 s_r + 12 + 8 + 24 R + 8) + 12 L "
                                          "(s_r = 4, R = 8)", "bytes": model_bytes, "ms": step_ms,
                  "achieved": model_gbs, "peak": hbm, "unit": "GB/s", "frac": model_gbs / hbm, "peak_kind": peak_kind}
    line = {"metric": METRIC, "value": total / (step_ms * 1e-3), "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_per_gpu": n, "coords": "float32", "leaves": leaves,
                       "l2": "inputs 192 MiB > 126 MB L2; no flush", "views": "off",
                       "parallelism": f"replicas{world}", "sort": sort_choice},
            "clocks": clocks.summary(), "gpu_launches": int(launches),
            "update": {"value": total / (upd_ms * 1e-3), "unit": "particles/s", "ms_per_step": upd_ms,
                       "graph_replayed": True, "resizes": resizes},
            "e2e": {"value": total / (e2e * 1e-3), "unit": "particles/s", "ms_per_step": e2e,
                    "h2d_bytes_per_step": 3 * 4 * n, "d2h_bytes_per_step": 12},
            "roofline": roof_sort, "roofline_update": roof, "roofline_build": roof_build, "stages": stages}
    if hasattr(tree, "buildPath"):
        lv, rounds = tree.buildPath()
        line["config"]["build_path"] = {"by_levels": lv, "reference_rounds": rounds}
    if rank == 0 and not args.no_cpu_baseline:
        v, dt = cpu_oracle_build(args.cpu_sample)
        line["cpu_baseline"] = {"value": v, "unit": "particles/s", "cores": 1, "kind": "port",
                                "sample": f"one build of {args.cpu_sample} Plummer particles (CPU oracle port)"}
    if rank == 0 and not args.no_reference_gpu:
        try:
            from oracle import refrun
            if refrun.available():
                rng = np.random.default_rng(5)
                frame1 = tuple(np.clip(a + rng.normal(0, 1e-3, a.size).astype(np.float32), 0, upper).astype(
                    np.float32) for a in hx)
                with torch.cuda.stream(s):
                    line["parity"] = reference_parity(tree, xs, [hx, frame1], s)
                r = refrun.time_reference(0, [hx, frame1], reps=10, bucket=BUCKET, nf=True, hilbert=True,
                                          views=(False, False, False))
                line["reference_gpu"] = {"build_ms": r["build_ms"], "update_ms": r["update_ms"],
                                         "build_min_ms": r["build_min_ms"], "build_max_ms": r["build_max_ms"],
                                         "cold_build_ms": r["cold_build_ms"], "reps": r["reps"],
                                         "build_value": n / (r["build_ms"] * 1e-3),
                                         "update_value": n / (r["update_ms"] * 1e-3), "unit": "particles/s",
                                         "what": "reference library compiled for sm_100a, same inputs and GPU; "
                                                 "build_ms: median of warm builds of one tree (its buffers "
                                                 "already grown), cold_build_ms: the first build of a fresh tree"}
        except Exception as e:  # the reference run is informational
            line.setdefault("parity", {"ref_lib_bit_exact": None, "error": str(e)[:200]})
            line["reference_gpu"] = {"error": str(e)[:200]}
    if world > 1:
        dist.destroy_process_group()
    if rank == 0 and world == 1 and not args.no_extras:
        # the other configurations of the metric, each with its own clocks
        tree.close()
        del rig, keys_in
        ab.release_cached_memory()
        torch.cuda.empty_cache()
        extras = {}
        for name, fn in (("c1", lambda: single_config_record("c1", args.steps, args.warmup, 1 << 18, True,
                                                             not args.no_reference_gpu)),
                         ("c3", lambda: single_config_record("c3", args.steps, args.warmup, 1 << 16, True,
                                                             not args.no_reference_gpu)),
                         ("c4", lambda: batched_record(args.steps, args.warmup, distributed=False)[0]),
                         ("c5", lambda: serving_record(args.c5_seconds, 2.0, 32, 256))):
            try:
                extras[name] = fn()
            except Exception as e:  # a failed leg is reported, the headline stands
                extras[name] = {"error": str(e)[:300]}
            ab.release_cached_memory()
            torch.cuda.empty_cache()
        line["configs"] = extras
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
