// octree.hpp -- adaptive octree (Octree<Real>) of the B200 engine.
//
// Same interface as nrottstegge/Adaptive_Trees include/adaptive_octree/
// octree.hpp:24-135: borrowed device coordinates, build()/update()/
// computeViews(), doBuffersNeedResize()/resizeBuffers(), device counters and
// the P/Perm/K/N/NF and view getters.  Getters return const DeviceVector<T>&
// (see config.hpp) over engine-owned device arrays.
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
class AO_CXX_API Octree
{
public:
    using KeyType = adaptive_octree::KeyType;
    using NodeIndex = adaptive_octree::NodeIndex;
    using SplitCriterion = adaptive_octree::SplitCriterion;
    using SfcKind = adaptive_octree::SfcKind;
    using ViewConfig = adaptive_octree::ViewConfig;
    using Config = OctreeConfig<Real>;

    // Escaped slots hold escapedParticleCoordinate<Real> in all three
    // coordinates.  The coordinates are borrowed, not copied.
    Octree(const Real *x_d, const Real *y_d, const Real *z_d, std::size_t numParticles, Config config = {});
    ~Octree();
    Octree(Octree &&) noexcept;
    Octree &operator=(Octree &&) noexcept;
    Octree(const Octree &) = delete;
    Octree &operator=(const Octree &) = delete;

    void print(std::ostream &out) const;
    void build();
    void update();
    void computeViews(ViewConfig views);
    void computeViews();

    // Call outside capture, after update or graph replay.  Refreshes the
    // host-visible sizes from the device state.
    [[nodiscard]] bool doBuffersNeedResize() const;
    // Grow topology/view storage by 25%, clear the flag, then recapture.
    void resizeBuffers();

    [[nodiscard]] const NodeIndex *numLeaves_d() const;
    [[nodiscard]] const NodeIndex *numNodes_d() const;
    [[nodiscard]] const unsigned *numActiveParticles_d() const;

    [[nodiscard]] const DeviceVector<KeyType> &particleKeys_d() const;
    [[nodiscard]] const DeviceVector<PermIndex> &perm_d() const;
    [[nodiscard]] const DeviceVector<KeyType> &cornerstone_d() const;
    [[nodiscard]] const DeviceVector<unsigned> &leafCounts_d() const;
    [[nodiscard]] const DeviceVector<unsigned> &nearFieldCounts_d() const;
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
    [[nodiscard]] SplitCriterion splitCriterion() const;
    [[nodiscard]] SfcKind sfcKind() const;

    aot::TreeEngine &engine() const { return *engine_; }

private:
    std::unique_ptr<aot::TreeEngine> engine_;
    // what the getters return: refreshed from the engine at each getter call
    // (one tree object is used from one host thread, as in the reference)
    mutable GetterViews views_;
};
}  // namespace adaptive_octree
