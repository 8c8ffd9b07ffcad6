// golden_regression.cu -- a C++ caller of the drop-in headers, written the way
// the reference's own regression test uses the reference library
// (tests/tree_test.cu:155-209 of nrottstegge/Adaptive_Trees): thrust device
// vectors of coordinates, adaptive_octree::Octree<double> with designated
// initialisers, build(), thrust::copy of the next frame, update() with the
// resize loop, and getters assigned to thrust::host_vector.
//
//   golden_regression <frames.bin> <out.bin>
//
// frames.bin: u64 n, then x0, y0, z0, x1, y1, z1 (n doubles each).
// out.bin: the arrays in the layout oracle/ref_driver.cu writes (per array
// u32 id, u64 count, u64 element bytes, the bytes; then u32 0xFFFFFFFF and
// six u64 scalars), so the test reads it with oracle/refrun.py.
//
// Besides writing the arrays it checks, and fails with exit code 1 if not:
//   * the Tree<double, TreeType::Octree> facade gives the same arrays as the
//     backend (tree_test.cu:1113-1131);
//   * a getter converts to thrust::device_vector and std::vector with the
//     same contents as thrust::host_vector;
//   * the device pointers of the particle arrays stay put across update()
//     (tree_test.cu:481-501), and the public macros compile.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>

#include "adaptive_octree/tree.hpp"

namespace
{
int g_failures = 0;

void expect(bool ok, const std::string &what)
{
    if (!ok)
    {
        std::fprintf(stderr, "golden_regression: FAILED %s\n", what.c_str());
        ++g_failures;
    }
}

template <class T>
void write(std::ofstream &out, std::uint32_t id, const thrust::host_vector<T> &h)
{
    const std::uint64_t count = h.size(), eb = sizeof(T);
    out.write(reinterpret_cast<const char *>(&id), 4);
    out.write(reinterpret_cast<const char *>(&count), 8);
    out.write(reinterpret_cast<const char *>(&eb), 8);
    if (count) out.write(reinterpret_cast<const char *>(h.data()), std::streamsize(count * eb));
}

template <class T>
void requireSame(const thrust::host_vector<T> &a, const thrust::host_vector<T> &b, const char *name)
{
    bool same = a.size() == b.size();
    for (std::size_t i = 0; same && i < a.size(); ++i) same = a[i] == b[i];
    expect(same, std::string("facade and backend differ in ") + name);
}
}  // namespace

int main(int argc, char **argv)
{
    if (argc != 3)
    {
        std::fprintf(stderr, "usage: golden_regression frames.bin out.bin\n");
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    std::uint64_t n = 0;
    in.read(reinterpret_cast<char *>(&n), 8);
    std::vector<double> f(6 * n);
    in.read(reinterpret_cast<char *>(f.data()), std::streamsize(f.size() * sizeof(double)));
    if (!in) throw std::runtime_error("short frames file");
    const double *x0 = f.data(), *y0 = x0 + n, *z0 = y0 + n, *x1 = z0 + n, *y1 = x1 + n, *z1 = y1 + n;

    ADAPTIVE_OCTREE_NVTX_RANGE_PUSH("golden regression");
    thrust::device_vector<double> x_d(x0, x0 + n), y_d(y0, y0 + n), z_d(z0, z0 + n);
    checkGpuErrors(cudaDeviceSynchronize());

    using Backend = adaptive_octree::Octree<double>;
    Backend tree(thrust::raw_pointer_cast(x_d.data()), thrust::raw_pointer_cast(y_d.data()),
                 thrust::raw_pointer_cast(z_d.data()), n,
                 {.maxParticlesPerLeaf = 64 * 64 * 27,
                  .splitCriterion = Backend::SplitCriterion::NFCount,
                  .views = {.treeStructure = true, .particleCountsPerBox = true, .particleMapping = true},
                  .interactive = false});
    using Facade = adaptive_octree::Tree<double, adaptive_octree::TreeType::Octree>;
    Facade::Config fc;
    fc.maxParticlesPerLeaf = 64 * 64 * 27;
    fc.splitCriterion = Facade::SplitCriterion::NFCount;
    fc.views = {.treeStructure = true, .particleCountsPerBox = true, .particleMapping = true};
    Facade facade(thrust::raw_pointer_cast(x_d.data()), thrust::raw_pointer_cast(y_d.data()),
                  thrust::raw_pointer_cast(z_d.data()), n, fc);

    tree.build();
    facade.build();
    const auto keysPointer = thrust::raw_pointer_cast(tree.particleKeys_d().data());
    const auto permutationPointer = thrust::raw_pointer_cast(tree.perm_d().data());

    thrust::copy(x1, x1 + n, x_d.begin());
    thrust::copy(y1, y1 + n, y_d.begin());
    thrust::copy(z1, z1 + n, z_d.begin());
    ADAPTIVE_OCTREE_CHECK_CUDA(cudaDeviceSynchronize());

    std::uint64_t resizes = 0;
    tree.update();
    while (tree.doBuffersNeedResize())
    {
        expect(++resizes < 64, "resize loop ends");
        if (resizes >= 64) break;
        tree.resizeBuffers();
        tree.update();
    }
    facade.update();
    while (facade.doBuffersNeedResize())
    {
        facade.resizeBuffers();
        facade.update();
    }
    expect(thrust::raw_pointer_cast(tree.particleKeys_d().data()) == keysPointer, "key pointer stable");
    expect(thrust::raw_pointer_cast(tree.perm_d().data()) == permutationPointer, "permutation pointer stable");

    const thrust::host_vector<adaptive_octree::KeyType> keys = tree.particleKeys_d();
    const thrust::host_vector<adaptive_octree::PermIndex> perm = tree.perm_d();
    const thrust::host_vector<adaptive_octree::KeyType> cornerstone = tree.cornerstone_d();
    const thrust::host_vector<unsigned> leafCounts = tree.leafCounts_d();
    const thrust::host_vector<unsigned> nearField = tree.nearFieldCounts_d();
    const thrust::host_vector<adaptive_octree::KeyType> boxKeys = tree.sfcBoxIndex_d();
    const thrust::host_vector<std::uint8_t> split = tree.hasBoxSplit_d();
    const thrust::host_vector<std::uint8_t> depth = tree.boxDepth_d();
    const thrust::host_vector<adaptive_octree::NodeIndex> parents = tree.parentIndex_d();
    const thrust::host_vector<adaptive_octree::NodeIndex> children = tree.childIndex_d();
    const thrust::host_vector<adaptive_octree::NodeIndex> levels = tree.levelOffset_d();
    const thrust::host_vector<unsigned> begins = tree.particleBeginIndex_d();
    const thrust::host_vector<unsigned> counts = tree.particleCounts_d();
    const thrust::host_vector<adaptive_octree::KeyType> mapping = tree.sfcParticleIndex_d();

    requireSame<adaptive_octree::KeyType>(facade.particleKeys_d(), keys, "particleKeys_d");
    requireSame<adaptive_octree::PermIndex>(facade.perm_d(), perm, "perm_d");
    requireSame<adaptive_octree::KeyType>(facade.cornerstone_d(), cornerstone, "cornerstone_d");
    requireSame<unsigned>(facade.leafCounts_d(), leafCounts, "leafCounts_d");
    requireSame<unsigned>(facade.nearFieldCounts_d(), nearField, "nearFieldCounts_d");
    requireSame<adaptive_octree::KeyType>(facade.sfcBoxIndex_d(), boxKeys, "sfcBoxIndex_d");
    requireSame<adaptive_octree::NodeIndex>(facade.parentIndex_d(), parents, "parentIndex_d");
    requireSame<unsigned>(facade.particleCounts_d(), counts, "particleCounts_d");
    requireSame<adaptive_octree::KeyType>(facade.sfcParticleIndex_d(), mapping, "sfcParticleIndex_d");
    expect(facade.maxAchievedDepth() == tree.maxAchievedDepth(), "facade depth");

    // the other conversions of a getter
    const thrust::device_vector<adaptive_octree::PermIndex> permCopy = tree.perm_d();
    const thrust::host_vector<adaptive_octree::PermIndex> permBack = permCopy;
    requireSame(permBack, perm, "perm_d through thrust::device_vector");
    const std::vector<unsigned> countsStd = tree.leafCounts_d();
    expect(countsStd.size() == leafCounts.size() &&
               std::equal(countsStd.begin(), countsStd.end(), leafCounts.begin()),
           "leafCounts_d through std::vector");
    expect(tree.leafCounts_d().size() + 1 == tree.cornerstone_d().size(), "leaf count size");
    expect(!tree.particleKeys_d().empty() && tree.particleKeys_d().capacity() >= tree.particleKeys_d().size(),
           "getter size and capacity");
    ADAPTIVE_OCTREE_NVTX_RANGE_POP();

    std::ofstream out(argv[2], std::ios::binary);
    write(out, 0, keys);
    write(out, 1, perm);
    write(out, 2, cornerstone);
    write(out, 3, leafCounts);
    write(out, 4, nearField);
    write(out, 5, boxKeys);
    write(out, 6, split);
    write(out, 7, depth);
    write(out, 8, parents);
    write(out, 9, children);
    write(out, 10, levels);
    write(out, 11, begins);
    write(out, 12, counts);
    write(out, 13, mapping);
    const std::uint32_t end = 0xFFFFFFFFu;
    const std::uint64_t sc[6] = {tree.numParticles(), tree.numActiveParticles(), tree.numNodes(),
                                 tree.maxAchievedDepth(), resizes, 0};
    out.write(reinterpret_cast<const char *>(&end), 4);
    out.write(reinterpret_cast<const char *>(sc), sizeof(sc));
    out.close();
    std::printf("golden_regression: %zu leaves, %zu view nodes, depth %u, %d failures\n", leafCounts.size(),
                tree.numNodes(), tree.maxAchievedDepth(), g_failures);
    return g_failures ? 1 : 0;
}
