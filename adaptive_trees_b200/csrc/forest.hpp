// forest.hpp -- host side of the forest engine: many independent octrees
// ("systems", each with its own particles) built and updated together.
//
// Each system behaves as one Tree<Real, Octree> with LeafCount refinement and
// the shared config: the same keys, permutation, cornerstone, counts,
// leafCapacity and needsResize answers as a tree built on the system alone.
// The work of all systems runs in the same launches (segmented sort, one
// decision/scan/scatter per round or pass over all systems' leaves), so a
// forest of many small systems is not bound by per-launch latency the way a
// loop over single trees is.  update() issues only kernel launches and
// memsets and can be captured into a CUDA graph.
#pragma once

#include <memory>
#include <vector>

#include "engine.hpp"

namespace aot
{
class ForestEngine
{
public:
    // x[s], y[s], z[s]: borrowed device coordinates of system s (n[s] each).
    ForestEngine(const void *const *x, const void *const *y, const void *const *z, const size_t *n, int numSystems,
                 const EngineConfig &cfg);
    ~ForestEngine();
    ForestEngine(const ForestEngine &) = delete;
    ForestEngine &operator=(const ForestEngine &) = delete;

    void build();
    // frozen: host array of numSystems bytes; systems marked non-zero keep
    // their tree (their keys are still re-sorted).  nullptr: update all.
    void update(const unsigned char *frozen);
    // Opt-in: update passes until a pass changes no system (or every change
    // is rejected for capacity), at most maxPasses; the state is read between
    // groups of cfg.iterations passes.  changedPasses (optional, one host
    // wait) receives the passes that changed some system.
    void updateUntilConverged(const unsigned char *frozen, unsigned maxPasses, unsigned *changedPasses);
    bool needsResize();                  // any system (reads the device state)
    void resizeBuffers();                // grows the systems that need it
    void setCoordinates(int s, const void *x, const void *y, const void *z);
    // 0 (default): build() builds every system's converged tree by levels in
    // one persistent launch, falling back to the rounds where they would not
    // converge within maxDepth; 1: always the rounds.  Both give the same trees.
    void setBuildMode(int mode);
    bool lastBuildByLevels() const;

    enum Buffer { ParticleKeys = 0, Perm = 1, Cornerstone = 2, LeafCounts = 3 };
    // device view of a system's buffer as of the last state readback
    void buffer(int s, int which, const void **ptr, size_t *len) const;
    struct SystemInfo
    {
        size_t particles, active, leaves, leafCapacity;
        bool needsResize;
    };
    SystemInfo info(int s) const;
    int numSystems() const;
    size_t numParticles() const;

private:
    struct Impl;
    std::unique_ptr<Impl> m_;
    void sortParticles(bool withSample);
    bool sortPersistent(int config);
    void launchKeygen(bool hist);
    bool levelBuild();
    void sortKeys(int config);
    void pass(bool build, const unsigned char *frozenDevice);
    void beginUpdate(const unsigned char *frozen);
    void endUpdate();
    void readState(bool model);
    void ensurePhysical(size_t entries);
};
}  // namespace aot
