// ref_driver.cu -- runs the REFERENCE library (nrottstegge/Adaptive_Trees,
// compiled from its own sources by oracle/Makefile into oracle/_ref/) on a
// scenario file and dumps every output array.
//
// TEST INFRASTRUCTURE ONLY: used by tests/ to pin parity of the B200 engine
// against the reference itself, and by bench.py to time the reference's GPU
// path on the same box.  Written against the reference's public API
// (adaptive_octree::Tree<Real, Kind>, tree.hpp:11-134).
//
// Input file (little-endian):
//   u32 magic 'AOSC', u32 kind, u32 real, u32 frames, u64 n,
//   i32 maxDepth, u32 bucket, i32 updateIterations, u32 nf, u32 hilbert,
//   u32 views[3], u32 timingReps, f64 box[6],
//   then `frames` x (x[n], y[n], z[n]) in Real.
// Output file: per frame, for each of 14 arrays: u32 id, u64 count,
//   u64 elemBytes, bytes; then u32 0xFFFFFFFF, u64 scalars[6]
//   (numParticles, numActive, numNodes, maxAchievedDepth, resizes, 0).
//   With a third argument `--digest` each array's bytes are replaced by one
//   u64 digest (arrayDigest below), so large trees are compared without
//   writing them out.
// With timingReps > 0 it instead prints one JSON line of timings:
//   cold_build_ms (the first build of a fresh tree, with its allocations),
//   build_ms (median of `reps` later builds of the same tree, its buffers
//   already grown), update_ms (median of captured-graph replays of update()
//   over frame 1).
// `ref_driver --cub-sort keys.bin reps` instead times cub::DeviceRadixSort::
// SortPairs on the keys of keys.bin, the sort the reference's build calls.
#include <cuda_runtime.h>
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <type_traits>
#include <vector>

#include "adaptive_octree/tree.hpp"

namespace
{
struct Header
{
    std::uint32_t magic, kind, real, frames;
    std::uint64_t n;
    std::int32_t maxDepth;
    std::uint32_t bucket;
    std::int32_t updateIterations;
    std::uint32_t nf, hilbert, views[3], timingReps;
    double box[6];
};

void check(cudaError_t e, const char *w)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(w) + ": " + cudaGetErrorString(e));
}

bool g_digest = false;

// Order-sensitive digest of an integer array: the sum over i of
// splitmix64(a[i] + i * 0x9E3779B97F4A7C15) modulo 2^64, each element taken as
// its unsigned bit pattern widened to 64 bits.  oracle/refrun.py computes the
// same function with numpy.
template <class T>
std::uint64_t arrayDigest(const T *a, std::size_t n)
{
    using U = std::conditional_t<sizeof(T) == 1, std::uint8_t,
                                 std::conditional_t<sizeof(T) == 4, std::uint32_t, std::uint64_t>>;
    std::uint64_t sum = 0;
    for (std::size_t i = 0; i < n; ++i)
    {
        U u;
        std::memcpy(&u, a + i, sizeof(U));
        std::uint64_t z = std::uint64_t(u) + std::uint64_t(i) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        sum += z ^ (z >> 31);
    }
    return sum;
}

template <class T>
void dump(std::ofstream &out, std::uint32_t id, const thrust::device_vector<T> &v)
{
    static_assert(sizeof(T) == 1 || sizeof(T) == 4 || sizeof(T) == 8, "array element width");
    thrust::host_vector<T> h = v;
    const std::uint64_t count = h.size(), eb = sizeof(T);
    out.write(reinterpret_cast<const char *>(&id), 4);
    out.write(reinterpret_cast<const char *>(&count), 8);
    out.write(reinterpret_cast<const char *>(&eb), 8);
    if (g_digest)
    {
        const std::uint64_t d = arrayDigest(h.data(), h.size());
        out.write(reinterpret_cast<const char *>(&d), 8);
    }
    else if (count)
    {
        out.write(reinterpret_cast<const char *>(h.data()), std::streamsize(count * eb));
    }
}

template <class Real, adaptive_octree::TreeType Kind>
int run(const Header &h, const std::vector<char> &payload, const char *outPath)
{
    using Tree = adaptive_octree::Tree<Real, Kind>;
    const size_t n = h.n;
    const Real *frames = reinterpret_cast<const Real *>(payload.data());
    thrust::device_vector<Real> x(n), y(n), z(n);
    auto load = [&](unsigned f) {
        const Real *base = frames + size_t(f) * 3 * n;
        if (n)
        {
            check(cudaMemcpy(thrust::raw_pointer_cast(x.data()), base, n * sizeof(Real), cudaMemcpyHostToDevice), "x");
            check(cudaMemcpy(thrust::raw_pointer_cast(y.data()), base + n, n * sizeof(Real), cudaMemcpyHostToDevice),
                  "y");
            check(cudaMemcpy(thrust::raw_pointer_cast(z.data()), base + 2 * n, n * sizeof(Real),
                             cudaMemcpyHostToDevice),
                  "z");
        }
    };
    typename Tree::Config c;
    c.maxDepth = h.maxDepth;
    c.maxParticlesPerLeaf = h.bucket;
    c.updateIterations = h.updateIterations;
    c.box = {Real(h.box[0]), Real(h.box[1]), Real(h.box[2]), Real(h.box[3]), Real(h.box[4]), Real(h.box[5])};
    c.splitCriterion = h.nf ? adaptive_octree::SplitCriterion::NFCount : adaptive_octree::SplitCriterion::LeafCount;
    c.sfcKind = h.hilbert ? adaptive_octree::SfcKind::Hilbert : adaptive_octree::SfcKind::Morton;
    c.views = {h.views[0] != 0, h.views[1] != 0, h.views[2] != 0};
    cudaStream_t stream;
    check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
    c.stream = stream;
    const Real *xp = thrust::raw_pointer_cast(x.data()), *yp = thrust::raw_pointer_cast(y.data()),
               *zp = thrust::raw_pointer_cast(z.data());

    if (h.timingReps > 0)
    {
        cudaEvent_t a, b;
        check(cudaEventCreate(&a), "ev");
        check(cudaEventCreate(&b), "ev");
        std::vector<double> builds, updates;
        load(0);
        check(cudaDeviceSynchronize(), "sync");
        auto timedBuild = [&](Tree &tree) {
            check(cudaStreamSynchronize(stream), "sync");
            check(cudaEventRecord(a, stream), "rec");
            tree.build();
            check(cudaEventRecord(b, stream), "rec");
            check(cudaEventSynchronize(b), "sync");
            float ms = 0;
            check(cudaEventElapsedTime(&ms, a, b), "elapsed");
            return double(ms);
        };
        {
            Tree warm(xp, yp, zp, n, c);  // loads the process's kernels
            warm.build();
        }
        Tree tree(xp, yp, zp, n, c);
        const double coldMs = timedBuild(tree);  // a fresh tree: its buffers grow during the build
        timedBuild(tree);
        for (unsigned r = 0; r < h.timingReps; ++r) builds.push_back(timedBuild(tree));
        if (h.frames > 1) load(1);
        check(cudaDeviceSynchronize(), "sync");
        cudaGraph_t graph;
        cudaGraphExec_t exec;
        check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeGlobal), "capture");
        tree.update();
        check(cudaStreamEndCapture(stream, &graph), "capture");
        check(cudaGraphInstantiate(&exec, graph, 0), "instantiate");
        for (unsigned r = 0; r < h.timingReps + 3; ++r)
        {
            check(cudaEventRecord(a, stream), "rec");
            check(cudaGraphLaunch(exec, stream), "launch");
            check(cudaEventRecord(b, stream), "rec");
            check(cudaEventSynchronize(b), "sync");
            float ms = 0;
            check(cudaEventElapsedTime(&ms, a, b), "elapsed");
            if (r >= 3) updates.push_back(ms);
            if (tree.doBuffersNeedResize())
            {
                cudaGraphExecDestroy(exec);
                cudaGraphDestroy(graph);
                tree.resizeBuffers();
                check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeGlobal), "capture");
                tree.update();
                check(cudaStreamEndCapture(stream, &graph), "capture");
                check(cudaGraphInstantiate(&exec, graph, 0), "instantiate");
            }
        }
        std::sort(builds.begin(), builds.end());
        std::sort(updates.begin(), updates.end());
        std::printf("{\"build_ms\": %.6f, \"update_ms\": %.6f, \"build_min_ms\": %.6f, \"update_min_ms\": %.6f, "
                    "\"build_max_ms\": %.6f, \"update_max_ms\": %.6f, \"cold_build_ms\": %.6f, \"reps\": %u}\n",
                    builds[builds.size() / 2], updates[updates.size() / 2], builds.front(), updates.front(),
                    builds.back(), updates.back(), coldMs, h.timingReps);
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        return 0;
    }

    std::ofstream out(outPath, std::ios::binary);
    Tree tree(xp, yp, zp, n, c);
    std::uint64_t resizes = 0;
    for (unsigned f = 0; f < h.frames; ++f)
    {
        load(f);
        check(cudaDeviceSynchronize(), "sync");
        if (f == 0)
        {
            tree.build();
        }
        else
        {
            tree.update();
            while (tree.doBuffersNeedResize())
            {
                ++resizes;
                tree.resizeBuffers();
                tree.update();
            }
        }
        (void)tree.doBuffersNeedResize();
        check(cudaDeviceSynchronize(), "sync");
        dump(out, 0, tree.particleKeys_d());
        dump(out, 1, tree.perm_d());
        dump(out, 2, tree.cornerstone_d());
        dump(out, 3, tree.leafCounts_d());
        if constexpr (Kind == adaptive_octree::TreeType::Octree) dump(out, 4, tree.nearFieldCounts_d());
        dump(out, 5, tree.sfcBoxIndex_d());
        dump(out, 6, tree.hasBoxSplit_d());
        dump(out, 7, tree.boxDepth_d());
        dump(out, 8, tree.parentIndex_d());
        dump(out, 9, tree.childIndex_d());
        dump(out, 10, tree.levelOffset_d());
        dump(out, 11, tree.particleBeginIndex_d());
        dump(out, 12, tree.particleCounts_d());
        dump(out, 13, tree.sfcParticleIndex_d());
        const std::uint32_t end = 0xFFFFFFFFu;
        const std::uint64_t sc[6] = {tree.numParticles(), tree.numActiveParticles(), tree.numNodes(),
                                     tree.maxAchievedDepth(), resizes, 0};
        out.write(reinterpret_cast<const char *>(&end), 4);
        out.write(reinterpret_cast<const char *>(sc), sizeof(sc));
    }
    return 0;
}
}  // namespace

// CUB's pair sort, as the reference calls it (octree.cu:301-304: 64-bit keys
// carrying 32-bit indices over bits [0, 64)), timed on the keys of `path`
// (u64 count, then the keys): prints {"cub_sort_ms": median, ...}.
int cubSort(const char *path, int reps)
{
    std::ifstream in(path, std::ios::binary);
    std::uint64_t n = 0;
    in.read(reinterpret_cast<char *>(&n), 8);
    std::vector<unsigned long long> keys(n);
    in.read(reinterpret_cast<char *>(keys.data()), std::streamsize(n * 8));
    if (!in) throw std::runtime_error("short key file");
    std::vector<unsigned> iota(n);
    for (std::uint64_t i = 0; i < n; ++i) iota[i] = unsigned(i);
    thrust::device_vector<unsigned long long> kin(keys.begin(), keys.end()), kout(n);
    thrust::device_vector<unsigned> vin(iota.begin(), iota.end()), vout(n);
    size_t tempBytes = 0;
    check(cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, thrust::raw_pointer_cast(kin.data()),
                                          thrust::raw_pointer_cast(kout.data()), thrust::raw_pointer_cast(vin.data()),
                                          thrust::raw_pointer_cast(vout.data()), n, 0, 64),
          "sort size");
    thrust::device_vector<unsigned char> temp(tempBytes);
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "ev");
    check(cudaEventCreate(&b), "ev");
    std::vector<double> ms;
    for (int r = 0; r < reps + 3; ++r)
    {
        check(cudaEventRecord(a), "rec");
        check(cub::DeviceRadixSort::SortPairs(thrust::raw_pointer_cast(temp.data()), tempBytes,
                                              thrust::raw_pointer_cast(kin.data()), thrust::raw_pointer_cast(kout.data()),
                                              thrust::raw_pointer_cast(vin.data()), thrust::raw_pointer_cast(vout.data()),
                                              n, 0, 64),
              "sort");
        check(cudaEventRecord(b), "rec");
        check(cudaEventSynchronize(b), "sync");
        float t = 0;
        check(cudaEventElapsedTime(&t, a, b), "elapsed");
        if (r >= 3) ms.push_back(t);
    }
    std::sort(ms.begin(), ms.end());
    std::printf("{\"cub_sort_ms\": %.6f, \"cub_sort_min_ms\": %.6f, \"n\": %llu, \"reps\": %d}\n", ms[ms.size() / 2],
                ms.front(), (unsigned long long)n, reps);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc == 4 && std::strcmp(argv[1], "--cub-sort") == 0)
    {
        try
        {
            return cubSort(argv[2], std::atoi(argv[3]));
        }
        catch (const std::exception &e)
        {
            std::fprintf(stderr, "ref_driver: %s\n", e.what());
            return 1;
        }
    }
    if (argc < 3 || (argc > 3 && std::strcmp(argv[3], "--digest") != 0))
    {
        std::fprintf(stderr, "usage: ref_driver scenario.bin out.bin [--digest]\n");
        return 2;
    }
    g_digest = argc > 3;
    try
    {
        std::ifstream in(argv[1], std::ios::binary);
        Header h{};
        in.read(reinterpret_cast<char *>(&h), sizeof(h));
        if (!in || h.magic != 0x43534f41u) throw std::runtime_error("bad scenario header");
        const size_t bytes = size_t(h.frames) * 3 * h.n * (h.real ? 8 : 4);
        std::vector<char> payload(bytes);
        in.read(payload.data(), std::streamsize(bytes));
        if (!in) throw std::runtime_error("short scenario file");
        using adaptive_octree::TreeType;
        if (h.kind == 0 && h.real == 0) return run<float, TreeType::Octree>(h, payload, argv[2]);
        if (h.kind == 0 && h.real == 1) return run<double, TreeType::Octree>(h, payload, argv[2]);
        if (h.kind == 1 && h.real == 0) return run<float, TreeType::Binary>(h, payload, argv[2]);
        return run<double, TreeType::Binary>(h, payload, argv[2]);
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "ref_driver: %s\n", e.what());
        return 1;
    }
}
