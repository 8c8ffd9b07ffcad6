// kdtree3d.hpp -- adaptive binary k-d tree (KDTree3D<Real>) of the B200 engine.
//
// Same interface as nrottstegge/Adaptive_Trees include/adaptive_octree/
// kdtree3d.hpp:18-126 (longest-side bisection, LeafCount refinement).
#pragma once

#include <cstddef>
#include <cstdint>
#include <iosfwd>
#include <memory>

#include "adaptive_octree/config.hpp"

namespace aot { class TreeEngine; }

namespace adaptive_octree
{
template <class Real>
class AO_CXX_API KDTree3D
{
public:
    using KeyType = adaptive_octree::KeyType;
    using NodeIndex = adaptive_octree::NodeIndex;
    using ViewConfig = adaptive_octree::ViewConfig;
    using Config = KDTree3DConfig<Real>;

    KDTree3D(const Real *x_d, const Real *y_d, const Real *z_d, std::size_t numParticles, Config config = {});
    ~KDTree3D();
    KDTree3D(KDTree3D &&) noexcept;
    KDTree3D &operator=(KDTree3D &&) noexcept;
    KDTree3D(const KDTree3D &) = delete;
    KDTree3D &operator=(const KDTree3D &) = delete;

    void print(std::ostream &out) const;
    void build();
    void update();
    void computeViews(ViewConfig views);
    void computeViews();
    [[nodiscard]] bool doBuffersNeedResize() const;
    void resizeBuffers();

    [[nodiscard]] const NodeIndex *numLeaves_d() const;
    [[nodiscard]] const NodeIndex *numNodes_d() const;
    [[nodiscard]] const unsigned *numActiveParticles_d() const;

    [[nodiscard]] const DeviceVector<KeyType> &particleKeys_d() const;
    [[nodiscard]] const DeviceVector<PermIndex> &perm_d() const;
    // Leaf i covers [K[i], K[i+1]); root boundaries are {0, maxKey}.
    [[nodiscard]] const DeviceVector<KeyType> &cornerstone_d() const;
    [[nodiscard]] const DeviceVector<unsigned> &leafCounts_d() const;
    [[nodiscard]] const DeviceVector<KeyType> &sfcBoxIndex_d() const;
    [[nodiscard]] const DeviceVector<std::uint8_t> &hasBoxSplit_d() const;
    [[nodiscard]] const DeviceVector<std::uint8_t> &boxDepth_d() const;
    [[nodiscard]] const DeviceVector<NodeIndex> &parentIndex_d() const;
    [[nodiscard]] const DeviceVector<NodeIndex> &childIndex_d() const;
    [[nodiscard]] const DeviceVector<NodeIndex> &levelOffset_d() const;
    [[nodiscard]] unsigned maxAchievedDepth() const;
    [[nodiscard]] const DeviceVector<unsigned> &particleBeginIndex_d() const;
    [[nodiscard]] const DeviceVector<unsigned> &particleCounts_d() const;
    [[nodiscard]] const DeviceVector<KeyType> &sfcParticleIndex_d() const;

    [[nodiscard]] std::size_t numParticles() const;
    [[nodiscard]] std::size_t numActiveParticles() const;
    [[nodiscard]] std::size_t numNodes() const;

    aot::TreeEngine &engine() const { return *engine_; }

private:
    std::unique_ptr<aot::TreeEngine> engine_;
    // what the getters return: refreshed from the engine at each getter call
    // (one tree object is used from one host thread, as in the reference)
    mutable GetterViews views_;
};
}  // namespace adaptive_octree
