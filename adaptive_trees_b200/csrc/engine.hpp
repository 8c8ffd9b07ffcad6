// engine.hpp -- host-side engine shared by Octree<Real>, KDTree3D<Real> and the C ABI.
//
// One TreeEngine holds one tree: borrowed device coordinates, the sorted keys
// P and permutation Perm, the A/B leaf buffers, the device-resident state,
// the capacity bookkeeping of the reference and the view arrays.  All work is
// issued on the caller's stream; update() and computeViews() issue only
// kernel launches and memsets and can be captured into a CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "adaptive_octree/config.hpp"
#include "capacity.hpp"

namespace aot
{
struct DeviceState;

// Keys per tile of the onesweep radix sort (threads x items per thread).
constexpr size_t kSortTileItems = 2560;

// A CUDA runtime failure inside the engine.
struct CudaError : std::runtime_error
{
    cudaError_t code;
    CudaError(cudaError_t c, const char *what)
        : std::runtime_error(std::string(what) + ": " + cudaGetErrorString(c)), code(c) {}
};

inline void check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw CudaError(e, what);
}
#define AOT_CHECK(x) ::aot::check((x), #x)
#define AOT_LAUNCH_CHECK() ::aot::check(cudaGetLastError(), "kernel launch")

struct EngineConfig
{
    int kind = 0;   // 0 octree, 1 binary
    int real = 1;   // 0 float, 1 double
    unsigned bucket = 64;
    unsigned maxDepth = 21;
    unsigned iterations = 2;
    bool nf = false;
    bool hilbert = false;
    double box[6] = {0, 1, 0, 1, 0, 1};
    adaptive_octree::ViewConfig views{};
    cudaStream_t stream = nullptr;
    // a build may time the sort configurations for the sort tuner (off for
    // latency-bound callers: they use the tuned choice or the default)
    bool tuneSort = true;
};

// Process-wide cache of device and pinned host blocks.
//
// cudaMalloc, cudaFree and cudaMallocHost synchronise the whole device, so a
// process that creates and destroys trees while other trees' work is queued
// (a serving loop) would stall all of it at every allocation.  Freed blocks
// are therefore kept per device and size class (quarter-octave steps) and
// handed to the next request of that class; the driver is only asked on a
// miss.  A block may be given back only when no queued work can still touch
// it: engines synchronise their stream before they release their buffers.
namespace blockcache
{
void *take(size_t bytes, size_t *classBytes);  // device block of >= bytes
void give(void *p, size_t classBytes);
void *takeHost(size_t bytes, size_t *classBytes);  // pinned host block
void giveHost(void *p, size_t classBytes);
size_t cachedBytes();  // device bytes held for reuse
void trim();           // returns every cached block to the driver
// Non-blocking streams and timing-free events of the current device, kept
// for reuse as the blocks are: creating and destroying them for every tree
// takes driver locks that the threads of a server would contend on.  A
// stream is given back once the work its owner queued is done.
cudaStream_t takeStream();
void giveStream(cudaStream_t s, int device);
cudaEvent_t takeEvent();
void giveEvent(cudaEvent_t e, int device);
}  // namespace blockcache

// Host wait for the work queued on `s` so far.  By default the thread spins
// (cudaStreamSynchronize), the lowest latency for one tree.  A thread that
// called sleepingWaits(true) -- one of many host threads waiting at once, as
// in a serving loop -- polls briefly, yielding its core, then sleeps on a
// blocking-sync event, so waiting threads do not starve the working ones.
void waitStream(cudaStream_t s);
void sleepingWaits(bool on);  // for the calling thread

// Device allocation that only grows, backed by the block cache.  The owner
// must have no queued work on the block when it is destroyed.
struct DevMem
{
    void *p = nullptr;
    size_t bytes = 0;
    DevMem() = default;
    DevMem(const DevMem &) = delete;
    DevMem &operator=(const DevMem &) = delete;
    ~DevMem();
    // discard contents; a replaced block waits for `owner` (the stream the
    // owner queues its work on), or for the whole device without one
    void reserve(size_t b, cudaStream_t owner = nullptr);
    void grow(size_t b, size_t keep, cudaStream_t s);  // keep the first `keep` bytes
    void release();                                    // back to the cache (no queued work may use it)
    template <class T> T *as() const { return static_cast<T *>(p); }
};

class TreeEngine
{
public:
    TreeEngine(const void *x, const void *y, const void *z, size_t n, const EngineConfig &cfg);
    ~TreeEngine();
    TreeEngine(const TreeEngine &) = delete;
    TreeEngine &operator=(const TreeEngine &) = delete;

    void build();
    void update();
    // Opt-in: update passes until one changes nothing (or would exceed the
    // leaf capacity), at most maxPasses; returns the passes that changed the
    // tree when `changedPasses` is set (a host wait at the end).
    void updateUntilConverged(unsigned maxPasses, unsigned *changedPasses);
    void computeViews(const adaptive_octree::ViewConfig &v);
    bool doBuffersNeedResize();
    void resizeBuffers();
    void setCoordinates(const void *x, const void *y, const void *z);

    // getters (logical sizes from the last host readback)
    enum Buffer
    {
        ParticleKeys = 0, Perm, Cornerstone, LeafCounts, NearFieldCounts, SfcBoxIndex, HasBoxSplit, BoxDepth,
        ParentIndex, ChildIndex, LevelOffset, ParticleBeginIndex, ParticleCounts, SfcParticleIndex, LeafBegins,
        NumBuffers
    };
    void buffer(int which, const void **ptr, size_t *len, size_t *cap, size_t *elemBytes) const;
    const int *numLeavesDevice() const;
    const int *numNodesDevice() const;
    const unsigned *numActiveParticlesDevice() const;
    size_t numParticles() const { return n_; }
    size_t numActiveParticles() const { return hostActive_; }
    size_t numNodes() const { return hostNodes_; }
    size_t numLeaves() const { return hostLeaves_; }
    unsigned maxAchievedDepth() const;
    size_t leafCapacity() const { return leafCapacity_; }
    const EngineConfig &config() const { return cfg_; }
    // diagnostics: committed build rounds, physical leaf capacity
    int buildRounds() const { return buildRounds_; }
    // How an octree build() reaches its tree: 0 (default) builds the
    // converged tree level by level where that gives the rounds' result and
    // falls back to the rounds otherwise; 1 always runs the rounds.
    void setBuildMode(int mode);
    // true when the last build() used the level-by-level builder
    bool lastBuildByLevels() const { return lastBuildByLevels_; }
    size_t physicalCapacity() const { return physCap_; }
    // kernel launches issued by the engine in this process
    static unsigned long long kernelLaunches();
    // device memory held by this tree's buffers
    size_t deviceBytes() const;
    // stable sort of (key, value) pairs by bits [beginBit, endBit)
    // (cub::DeviceRadixSort::SortPairs semantics; scratch == nullptr queries
    // the scratch size; valsIn == nullptr sorts the indices 0..n-1)
    static void sortPairs(void *scratch, size_t *scratchBytes, const unsigned long long *keysIn,
                          unsigned long long *keysOut, const unsigned *valsIn, unsigned *valsOut, size_t n,
                          int beginBit, int endBit, cudaStream_t s);
    // true when a pair sort of n items that ran in `scratch` on `s` had a
    // bounded look-back wait give up (waits for `s`)
    static bool sortPairsFailed(const void *scratch, size_t n, cudaStream_t s);
    // loads every kernel the pair sort can launch on the current device
    static void sortPairsPreload();
    // self-test of the bounded device waits (selftest.cu): runs a look-back
    // (0: radix sort pass, 1: decide+scan) whose predecessor tile never
    // publishes, with `spinLimit` polls allowed; returns the kernel's error
    // word (kErrLookback when the wait ran out and the kernel returned)
    static int boundedWaitProbe(int which, unsigned spinLimit);
    // the same with sort configuration `config` (its own scratch size)
    static void sortPairsWith(int config, void *scratch, size_t *scratchBytes, const unsigned long long *keysIn,
                              unsigned long long *keysOut, const unsigned *valsIn, unsigned *valsOut, size_t n,
                              int beginBit, int endBit, cudaStream_t s);
    // dst[i] = src[perm[i]] for the numParticles() elements of elemBytes
    // each: per-particle data in key order (device pointers, the tree's stream)
    void gather(const void *src, void *dst, size_t elemBytes) const;
    // Stage timing of build() and update() (the CUDA-event counterpart of the
    // reference's NVTX ranges behind ADAPTIVE_OCTREE_PROFILING,
    // config.hpp:20-28): when on, they record events at their stage
    // boundaries and around every near-field launch, and push NVTX ranges;
    // calls made while the stream is being captured record nothing.
    struct StageTimes
    {
        double keysAndSortMs = 0, refreshMs = 0, passesMs = 0, finishMs = 0, totalMs = 0;
        double nearFieldMs = 0;       // all near-field launches of the call
        double nearFieldFirstMs = 0;  // the first one (update(): the full refresh of every leaf)
        int nearFieldLaunches = 0;
        int call = 0;  // 1 build, 2 update
        bool valid = false;
    };
    void setProfiling(bool on);
    StageTimes stageTimes();  // of the last profiled build() or update(); waits for it
    // one-shot key generation without a sort (computeSfcKeys semantics)
    static void computeKeys(int kind, int real, const void *x, const void *y, const void *z, size_t n,
                            const double *box, bool hilbert, unsigned maxDepth, unsigned long long *keys,
                            unsigned *perm, cudaStream_t s);

private:
    struct Impl;
    std::unique_ptr<Impl> m_;
    EngineConfig cfg_;
    size_t n_ = 0;
    const void *x_ = nullptr, *y_ = nullptr, *z_ = nullptr;
    size_t leafCapacity_ = 0, physCap_ = 0;
    size_t hostLeaves_ = 1, hostActive_ = 0, hostNodes_ = 0;
    int hostActiveBuffer_ = 0;
    bool built_ = false;
    int buildRounds_ = 0;
    int buildMode_ = 0;
    bool lastBuildByLevels_ = false;
    // thrust capacity model of K_d / tmpTree (octree.cu:453-457)
    OctreeCapacity capModel_;  // reference K_d / tmpTree capacities (octree)
    adaptive_octree::ViewConfig prepared_{};
    // stage events of build()/update(): start, sorted, refreshed (update),
    // passes done, end; near-field launches are bracketed by their own pairs
    enum Mark { MarkStart = 0, MarkSorted, MarkRefreshed, MarkPassed, MarkEnd, NumMarks };
    bool profiling_ = false, marking_ = false, marksRecorded_ = false;
    int markCall_ = 0, nfMarks_ = 0;
    int sortConfig_ = -1;  // sort configuration of the last sort (kept under stream capture)
    void mark(Mark m, int call = 0);
    void markNearField(bool begin);

    void sortParticles();
    // the converged octree by levels (levelbuild.cuh); false when the rounds
    // must run instead (the tree would not converge within maxDepth rounds,
    // or LeafCount thresholds wrap in 32 bits); fills the build's round
    // proposals
    bool octreeLevelBuild(std::vector<long long> &proposals);
    bool binaryLevelBuild();
    void sortKeys(int config);
    void octreeBuild();
    void binaryBuild();
    void octreePass(bool buildMode, long long limit);
    void binaryPass(bool buildMode, long long limit);
    void refreshAll();
    void refreshCounts(bool all, unsigned blocks);
    void prepareGraphBuffers(size_t capacity);
    void ensurePhysical(size_t capacity);
    void buildViews(const adaptive_octree::ViewConfig &v);
    void prepareViews(size_t capacity, const adaptive_octree::ViewConfig &v);
    void syncViewSizes();
    void readState();
    void applyState();
    void materializeCounts();
};

// The radix sort tuner: which compiled sort configuration (digit width, keys
// per thread) a sort of n keys uses on the current device, for contiguous
// (tree, pair) or segmented (forest) sorts.  Sizes are grouped by bit length.
// The first tree or forest build of a size class times every configuration
// on its own keys and keeps the fastest; later sorts of that class reuse it.
struct SortTuning
{
    int config;          // index into the compiled configurations
    int digitBits;
    int itemsPerThread;  // tile = 256 threads x itemsPerThread keys
    bool tuned;          // chosen by timing (else the default or a forced one)
};
int sortConfigCount();
SortTuning sortConfigInfo(int config);
SortTuning sortTuning(bool segmented, size_t n);
bool sortNeedsTuning(bool segmented, size_t n);
// time(c) sorts with configuration c and returns its duration in ms; each
// configuration is timed twice and the second time counts.
int sortTune(bool segmented, size_t n, float (*time)(int, void *), void *ctx);
void sortSetAutotune(bool on);
void sortForceConfig(int config);  // -1 lifts the force
void sortForgetTuning();

// TreeEngine::sortPairs with its scratch in a fixed device array of
// sort_noalloc.cu (no allocation; at most sortPairsNoAllocMaxItems() items;
// concurrent calls on one device race).
void sortPairsNoAlloc(const unsigned long long *keysIn, unsigned long long *keysOut, const unsigned *valsIn,
                      unsigned *valsOut, size_t n, int beginBit, int endBit, cudaStream_t s);
size_t sortPairsNoAllocMaxItems();
// true when the last sortPairsNoAlloc of n items on this device had a bounded
// look-back wait give up (waits for `s`)
bool sortPairsNoAllocFailed(size_t n, cudaStream_t s);

}  // namespace aot
