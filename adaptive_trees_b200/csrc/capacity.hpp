// capacity.hpp -- the reference's octree buffer-capacity bookkeeping, replayed on the host.
//
// The reference keeps the cornerstone K_d and the build's tmpTree in thrust
// vectors and swaps them every build round (octree.cu:159-180); their
// capacities after the build, with 25% headroom (resizeWithHeadroom,
// helpers.cuh:122-141), decide leafCapacity, and prepareGraphBuffers
// (octree.cu:182-241) and every state readback (octree.cu:498-537) move their
// sizes again.  doBuffersNeedResize() answers from leafCapacity, so the model
// must follow the reference step by step.  One instance per tree; the forest
// engine keeps one per system.
#pragma once

#include <algorithm>
#include <cstddef>
#include <utility>

namespace aot
{
struct OctreeCapacity
{
    // K_d.resize(2) in the constructor (octree.cu:149); tmpTree starts empty
    size_t kSize = 2, kCap = 2, tSize = 0, tCap = 0;

    // vector growth on resize (append) and reserve
    static void resize(size_t &size, size_t &cap, size_t n)
    {
        if (n > cap) cap = std::max(size + std::max(size, n - size), 2 * cap);
        size = n;
    }
    static void reserve(size_t &cap, size_t n) { cap = std::max(cap, n); }

    // rebalanceBuild starts from the root
    void buildStart() { kSize = 2; }

    // Replays the build rounds that changed the tree (`proposals[r]` = leaves
    // after round r: tmpTree resized with headroom, then swapped with K_d) and
    // returns the leafCapacity of the finished tree of `leaves` leaves.
    size_t finishBuild(const long long *proposals, size_t rounds, size_t leaves)
    {
        for (size_t r = 0; r < rounds; ++r)
        {
            const size_t req = size_t(proposals[r]) + 1;
            if (req > tCap) tCap = req + req / 4;
            tSize = req;
            std::swap(kSize, tSize);
            std::swap(kCap, tCap);
        }
        kSize = leaves + 1;
        return std::max({kCap - 1, tSize == 0 ? size_t(0) : tCap - 1, leaves + (leaves + 3) / 4});
    }

    // prepareGraphBuffers(capacity): both vectors reserved and resized to
    // capacity + 1, then back to the live tree's size.
    void prepare(size_t capacity)
    {
        const size_t leaves = kSize - 1;
        reserve(kCap, capacity + 1);
        resize(kSize, kCap, capacity + 1);
        reserve(tCap, capacity + 1);
        resize(tSize, tCap, capacity + 1);
        kSize = tSize = leaves + 1;
    }

    // a state readback sizes both vectors to the current tree
    void stateRead(size_t leaves) { kSize = tSize = leaves + 1; }
};
}  // namespace aot
