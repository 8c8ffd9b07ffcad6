// engine.cu -- host orchestration of the B200 adaptive-tree engine.
//
// Follows the reference's control flow for build/update/views
// (octree.cu:427-551, kdtree3d.cu:227-297, tree_view.cu:814-1134) with
// B200-specific choices:
//   * keygen + onesweep sort replace computeSfcKeys + CUB SortPairs;
//   * the octree build runs its split/merge rounds on the device without a
//     host round-trip per round: rounds are issued in batches, every kernel
//     stops as soon as the device state says the tree converged, and the host
//     reads the state once per batch; the reference's vector capacity growth,
//     which decides leafCapacity, is replayed on the host from the per-round
//     proposals recorded on the device;
//   * the binary build emulates the reference's reject/grow/retry capacity
//     loop on the device (25% steps) instead of a host sync per pass.
#include "engine.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <tuple>
#include <mutex>
#include <stdexcept>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "engine_util.cuh"
#include "keygen.cuh"
#include "binlevel.cuh"
#include "levelbuild.cuh"
#include "rebalance.cuh"
#include "tree_view.cuh"

namespace aot
{
static_assert(sort::kTile == int(kSortTileItems), "kSortTileItems must match the onesweep tile");
// --------------------------------------------------------------------------
// block cache
// --------------------------------------------------------------------------
namespace blockcache
{
namespace
{
// Misses are served by a stream-ordered pool of this library (cudaMallocAsync
// does not synchronise the device as cudaMalloc does); blocks never go back
// to the pool except through trim().
struct DevicePool
{
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
};
struct Cache
{
    std::mutex mu;
    std::map<std::pair<int, size_t>, std::vector<void *>> dev;  // (device, class) -> blocks
    std::map<size_t, std::vector<void *>> host;
    std::map<int, DevicePool> pools;
    size_t devBytes = 0;
};
Cache &cache()
{
    static Cache *c = new Cache();  // never destroyed: blocks may be given back during process exit
    return *c;
}
// size class: b rounded up to 2^k or 1.5 * 2^k (at most 50% above b), >= 256 bytes
size_t sizeClass(size_t b)
{
    if (b <= 256) return 256;
    const size_t top = size_t(1) << (63 - __builtin_clzll(b));
    if (b == top) return b;
    return b <= top + top / 2 ? top + top / 2 : 2 * top;
}
int currentDevice()
{
    int d = 0;
    AOT_CHECK(cudaGetDevice(&d));
    return d;
}
// with k.mu held
DevicePool &poolOf(Cache &k, int d)
{
    DevicePool &p = k.pools[d];
    if (!p.pool)
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = d;
        AOT_CHECK(cudaMemPoolCreate(&p.pool, &props));
        unsigned long long keep = ~0ull;  // keep what it maps until trim()
        AOT_CHECK(cudaMemPoolSetAttribute(p.pool, cudaMemPoolAttrReleaseThreshold, &keep));
        AOT_CHECK(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking));
    }
    return p;
}
}  // namespace

void *take(size_t bytes, size_t *classBytes)
{
    const size_t c = sizeClass(bytes);
    const int d = currentDevice();
    Cache &k = cache();
    cudaStream_t s = nullptr;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(k.mu);
        auto it = k.dev.find({d, c});
        if (it != k.dev.end() && !it->second.empty())
        {
            void *p = it->second.back();
            it->second.pop_back();
            k.devBytes -= c;
            *classBytes = c;
            return p;
        }
        DevicePool &dp = poolOf(k, d);
        s = dp.stream;
        pool = dp.pool;
    }
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, c, pool, s);
    if (e == cudaErrorMemoryAllocation)
    {
        // give the cached blocks back and retry once
        (void)cudaGetLastError();
        trim();
        e = cudaMallocFromPoolAsync(&p, c, pool, s);
    }
    AOT_CHECK(e);
    waitStream(s);  // usable from any stream from here on
    *classBytes = c;
    return p;
}

void give(void *p, size_t classBytes)
{
    if (!p) return;
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return;
    Cache &k = cache();
    std::lock_guard<std::mutex> lock(k.mu);
    k.dev[{d, classBytes}].push_back(p);
    k.devBytes += classBytes;
}

void *takeHost(size_t bytes, size_t *classBytes)
{
    const size_t c = sizeClass(bytes);
    Cache &k = cache();
    {
        std::lock_guard<std::mutex> lock(k.mu);
        auto it = k.host.find(c);
        if (it != k.host.end() && !it->second.empty())
        {
            void *p = it->second.back();
            it->second.pop_back();
            *classBytes = c;
            return p;
        }
    }
    void *p = nullptr;
    AOT_CHECK(cudaMallocHost(&p, c));
    *classBytes = c;
    return p;
}

void giveHost(void *p, size_t classBytes)
{
    if (!p) return;
    Cache &k = cache();
    std::lock_guard<std::mutex> lock(k.mu);
    k.host[classBytes].push_back(p);
}

size_t cachedBytes()
{
    Cache &k = cache();
    std::lock_guard<std::mutex> lock(k.mu);
    return k.devBytes;
}

void trim()
{
    Cache &k = cache();
    std::lock_guard<std::mutex> lock(k.mu);
    int cur = 0;
    (void)cudaGetDevice(&cur);
    for (auto &kv : k.dev)
    {
        const int d = kv.first.first;
        auto pit = k.pools.find(d);
        if (pit == k.pools.end()) continue;
        (void)cudaSetDevice(d);
        for (void *p : kv.second) (void)cudaFreeAsync(p, pit->second.stream);
        kv.second.clear();
    }
    for (auto &kv : k.pools)
    {
        (void)cudaSetDevice(kv.first);
        (void)cudaStreamSynchronize(kv.second.stream);
        (void)cudaMemPoolTrimTo(kv.second.pool, 0);
    }
    (void)cudaSetDevice(cur);
    k.dev.clear();
    k.devBytes = 0;
}

namespace
{
struct Handles
{
    std::mutex mu;
    std::map<int, std::vector<cudaStream_t>> streams;
    std::map<int, std::vector<cudaEvent_t>> events;
};
Handles &handles()
{
    static Handles *h = new Handles;  // lives as long as the process (streams outlive static teardown)
    return *h;
}
}  // namespace

cudaStream_t takeStream()
{
    int d = 0;
    AOT_CHECK(cudaGetDevice(&d));
    Handles &h = handles();
    {
        std::lock_guard<std::mutex> lock(h.mu);
        auto &v = h.streams[d];
        if (!v.empty())
        {
            const cudaStream_t s = v.back();
            v.pop_back();
            return s;
        }
    }
    cudaStream_t s = nullptr;
    AOT_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}

void giveStream(cudaStream_t s, int device)
{
    if (!s) return;
    Handles &h = handles();
    std::lock_guard<std::mutex> lock(h.mu);
    h.streams[device].push_back(s);
}

cudaEvent_t takeEvent()
{
    int d = 0;
    AOT_CHECK(cudaGetDevice(&d));
    Handles &h = handles();
    {
        std::lock_guard<std::mutex> lock(h.mu);
        auto &v = h.events[d];
        if (!v.empty())
        {
            const cudaEvent_t e = v.back();
            v.pop_back();
            return e;
        }
    }
    cudaEvent_t e = nullptr;
    AOT_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return e;
}

void giveEvent(cudaEvent_t e, int device)
{
    if (!e) return;
    Handles &h = handles();
    std::lock_guard<std::mutex> lock(h.mu);
    h.events[device].push_back(e);
}
}  // namespace blockcache

namespace
{
thread_local bool t_sleepingWaits = false;
}

void sleepingWaits(bool on) { t_sleepingWaits = on; }

void waitStream(cudaStream_t s)
{
    if (!t_sleepingWaits)
    {
        AOT_CHECK(cudaStreamSynchronize(s));
        return;
    }
    // one blocking-sync event per host thread and device
    thread_local std::map<int, cudaEvent_t> events;
    int d = 0;
    AOT_CHECK(cudaGetDevice(&d));
    cudaEvent_t &ev = events[d];
    if (!ev) AOT_CHECK(cudaEventCreateWithFlags(&ev, cudaEventBlockingSync | cudaEventDisableTiming));
    AOT_CHECK(cudaEventRecord(ev, s));
    // short waits (a tree's own round trips) are polled, yielding the core
    // between polls; long ones sleep in the blocking synchronisation
    const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(1000);
    for (;;)
    {
        const cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return;
        if (e != cudaErrorNotReady) AOT_CHECK(e);
        if (std::chrono::steady_clock::now() >= until) break;
        std::this_thread::yield();
    }
    AOT_CHECK(cudaEventSynchronize(ev));
}

// --------------------------------------------------------------------------
// DevMem
// --------------------------------------------------------------------------
DevMem::~DevMem() { release(); }
void DevMem::release()
{
    if (p) blockcache::give(p, bytes);
    p = nullptr;
    bytes = 0;
}
void DevMem::reserve(size_t b, cudaStream_t owner)
{
    if (b <= bytes) return;
    if (p)
    {
        // work queued on the old block must end before another buffer can be
        // handed the block
        if (owner) waitStream(owner);
        else AOT_CHECK(cudaDeviceSynchronize());
        blockcache::give(p, bytes);
    }
    p = nullptr;
    bytes = 0;
    p = blockcache::take(b, &bytes);
}
void DevMem::grow(size_t b, size_t keep, cudaStream_t s)
{
    if (b <= bytes) return;
    size_t nb = 0;
    void *q = blockcache::take(b, &nb);
    keep = std::min(keep, bytes);
    if (keep && p) AOT_CHECK(cudaMemcpyAsync(q, p, keep, cudaMemcpyDeviceToDevice, s));
    if (p)
    {
        // the owner queues its work on this block on s only
        waitStream(s);
        blockcache::give(p, bytes);
    }
    p = q;
    bytes = nb;
}

namespace
{
// Kernel launches issued by this process (all trees); reported by
// ao_tree_get_info so a benchmark can state how many engine kernels ran.
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void noteLaunch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int smCount()
{
    static int sms = 0;
    if (!sms)
    {
        int dev = 0;
        AOT_CHECK(cudaGetDevice(&dev));
        AOT_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (sms <= 0) sms = 148;
    }
    return sms;
}

const HilbertTables &hilbertTables()
{
    static const HilbertTables t = makeHilbertTables();
    return t;
}

namespace
{
// makeBinaryGeometry (binary_node.cuh:17-40): the longest side is halved at
// every depth, first axis wins ties.
BinaryGeometry makeGeometry(const double *b, unsigned maxDepth, int real)
{
    if (maxDepth > kBinDepth) throw std::invalid_argument("Binary maxDepth exceeds key precision");
    double bx[6];
    for (int k = 0; k < 6; ++k) bx[k] = real == 0 ? double(float(b[k])) : b[k];
    long double len[3] = {(long double)bx[1] - bx[0], (long double)bx[3] - bx[2], (long double)bx[5] - bx[4]};
    for (auto s : len)
        if (!(s > 0) || !std::isfinite(s)) throw std::invalid_argument("Tree box must have finite positive sides");
    BinaryGeometry g{};
    g.mortonOrder = 1;
    for (unsigned d = 0; d < kBinDepth; ++d)
    {
        unsigned a = 0;
        if (len[1] > len[a]) a = 1;
        if (len[2] > len[a]) a = 2;
        g.axis[d] = (unsigned char)a;
        if (a != d % 3) g.mortonOrder = 0;
        len[a] *= 0.5L;
    }
    g.xmin = bx[0];
    g.xmax = bx[1];
    g.ymin = bx[2];
    g.ymax = bx[3];
    g.zmin = bx[4];
    g.zmax = bx[5];
    return g;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <class Real, Curve C>
void launchKeygenT(const Real *x, const Real *y, const Real *z, size_t n, const KeygenParams<Real> &prm, u64 *keys,
                   u32 *hist, int passes, cudaStream_t s)
{
    const bool vec = aligned16(x) && aligned16(y) && aligned16(z);
    constexpr int V = sizeof(Real) == 4 ? 4 : 2;
    const size_t groups = vec ? n / V : n;
    const unsigned blocks = std::max(1u, std::min<unsigned>(ceilDiv(std::max<size_t>(groups, 1), kKeygenThreads),
                                                             unsigned(smCount()) * 8u));
    if (vec) keygenKernel<Real, C, V><<<blocks, kKeygenThreads, 0, s>>>(x, y, z, n, prm, keys, hist, passes), noteLaunch();
    else keygenKernel<Real, C, 1><<<blocks, kKeygenThreads, 0, s>>>(x, y, z, n, prm, keys, hist, passes), noteLaunch();
    AOT_LAUNCH_CHECK();
}

template <class Real>
void launchKeygen(int kind, bool hilbert, const Real *x, const Real *y, const Real *z, size_t n,
                  const KeygenParams<Real> &prm, u64 *keys, u32 *hist, int passes, cudaStream_t s)
{
    if (kind == 1) launchKeygenT<Real, Curve::Binary>(x, y, z, n, prm, keys, hist, passes, s);
    else if (hilbert) launchKeygenT<Real, Curve::Hilbert>(x, y, z, n, prm, keys, hist, passes, s);
    else launchKeygenT<Real, Curve::Morton>(x, y, z, n, prm, keys, hist, passes, s);
}

__global__ void iotaKernel(u32 *perm, size_t n)
{
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        perm[i] = u32(i);
}

// Sort scratch layout: hist[kPassSlots][256] | bins[kPassSlots][256] |
// tileCounters[kPassSlots] (u32), then look-back status words (u64): passes x
// tiles x 256 of configuration `config`, or room for every configuration
// (config < 0: kPassSlots passes of the smallest tiles).
struct SortArena
{
    DevMem counters, status;
    void ensure(size_t n, int config, cudaStream_t owner)
    {
        counters.reserve((2 * sort::kPassSlots * sort::kRadix + sort::kPassSlots) * sizeof(u32), owner);
        const size_t words = config < 0
                                 ? size_t(sort::kPassSlots) * std::max<size_t>(1, (n + sort::kMinTile - 1) / sort::kMinTile)
                                 : size_t(sort::configPasses(config)) *
                                       std::max<size_t>(1, (n + sort::configTile(config) - 1) / sort::configTile(config));
        status.reserve(words * sort::kRadix * sizeof(u64), owner);
    }
    u32 *hist() const { return counters.as<u32>(); }
    u32 *bins() const { return counters.as<u32>() + sort::kPassSlots * sort::kRadix; }
    u32 *tileCounters() const { return counters.as<u32>() + 2 * sort::kPassSlots * sort::kRadix; }
};

size_t configTiles(int cfg, size_t n) { return std::max<size_t>(1, (n + sort::configTile(cfg) - 1) / sort::configTile(cfg)); }

// Onesweep passes of configuration `cfg` over (k[0], v[0]) -> ... for bits
// [beginBit, endBit); the counts must already be in hist.  valsAreIndices:
// the first pass generates the values.  Returns the index (0/1) of the
// buffers holding the result.
int runPasses(int cfg, cudaStream_t s, u64 *k[2], u32 *v[2], size_t n, int beginBit, int endBit, bool valsAreIndices,
              SortArena &a, int *error)
{
    sort::setPassSmemAll();
    const int bitsPer = sort::kSortConfigs[cfg].bits;
    const int passes = (endBit - beginBit + bitsPer - 1) / bitsPer;
    const size_t tiles = configTiles(cfg, n);
    sort::binsKernel<<<1, sort::kRadix, 0, s>>>(a.hist(), a.bins(), passes), noteLaunch();
    AOT_LAUNCH_CHECK();
    for (int p = 0; p < passes; ++p)
    {
        const int in = p & 1, out = in ^ 1;
        const int shift = beginBit + p * bitsPer;
        sort::launchPass(cfg, s, k[in], (p == 0 && valsAreIndices) ? nullptr : v[in], k[out], v[out], n, shift,
                         a.bins() + p * sort::kRadix, a.tileCounters() + p,
                         a.status.as<u64>() + size_t(p) * tiles * sort::kRadix, error, std::min(bitsPer, endBit - shift)),
            noteLaunch();
        AOT_LAUNCH_CHECK();
    }
    return passes & 1;
}

// Zeroes the counters and the status words configuration `cfg` reads.
void clearArena(int cfg, cudaStream_t s, SortArena &a, size_t n, int passes)
{
    AOT_CHECK(cudaMemsetAsync(a.counters.p, 0, a.counters.bytes, s));
    AOT_CHECK(cudaMemsetAsync(a.status.p, 0, size_t(passes) * configTiles(cfg, n) * sort::kRadix * sizeof(u64), s));
}

// Generic stable sort of (keys, identity indices) by bits [0, 8*passes),
// default configuration.
int sortWithIndices(cudaStream_t s, u64 *k[2], u32 *v[2], size_t n, int passes, SortArena &a, int *error)
{
    if (n == 0) return 0;
    const int cfg = sort::kDefaultSortConfig;
    a.ensure(n, cfg, s);
    clearArena(cfg, s, a, n, passes);
    const unsigned blocks = std::max(1u, std::min<unsigned>(ceilDiv(n, sort::kThreads), unsigned(smCount()) * 8u));
    sort::launchHistogram(cfg, s, blocks, k[0], n, 0, passes, a.hist(), 8 * passes), noteLaunch();
    AOT_LAUNCH_CHECK();
    return runPasses(cfg, s, k, v, n, 0, 8 * passes, true, a, error);
}

}  // namespace

unsigned gridFor(size_t n, unsigned threads) { return std::max(1u, ceilDiv(std::max<size_t>(n, 1), threads)); }

unsigned long long TreeEngine::kernelLaunches() { return g_launches.load(std::memory_order_relaxed); }

// --------------------------------------------------------------------------
// sort tuner
// --------------------------------------------------------------------------
namespace
{
struct TunerState
{
    std::mutex mu;
    std::map<std::tuple<int, int, int>, int> chosen;  // (device, segmented, size class) -> configuration
    std::map<std::tuple<int, int, int>, int> timing;  // classes being timed by some thread
    bool autotune = true;
    int forced = -1;
};
TunerState &tuner()
{
    static TunerState t;
    return t;
}
std::tuple<int, int, int> tuneKey(bool segmented, size_t n)
{
    int dev = 0;
    AOT_CHECK(cudaGetDevice(&dev));
    int cls = 0;
    while (cls < 63 && (size_t(1) << (cls + 1)) <= std::max<size_t>(n, 1)) ++cls;
    return {dev, segmented ? 1 : 0, cls};
}
}  // namespace

int sortConfigCount() { return sort::kNumSortConfigs; }

SortTuning sortConfigInfo(int config)
{
    if (config < 0 || config >= sort::kNumSortConfigs) throw std::invalid_argument("sort: unknown configuration");
    return {config, sort::kSortConfigs[config].bits, sort::kSortConfigs[config].items, false};
}

SortTuning sortTuning(bool segmented, size_t n)
{
    TunerState &t = tuner();
    const auto key = tuneKey(segmented, n);
    std::lock_guard<std::mutex> lock(t.mu);
    if (t.forced >= 0) return sortConfigInfo(t.forced);
    const auto it = t.chosen.find(key);
    if (it != t.chosen.end())
    {
        SortTuning r = sortConfigInfo(it->second);
        r.tuned = true;
        return r;
    }
    return sortConfigInfo(sort::kDefaultSortConfig);
}

bool sortNeedsTuning(bool segmented, size_t n)
{
    TunerState &t = tuner();
    const auto key = tuneKey(segmented, n);
    std::lock_guard<std::mutex> lock(t.mu);
    return t.autotune && t.forced < 0 && t.chosen.find(key) == t.chosen.end() && t.timing.find(key) == t.timing.end();
}

int sortTune(bool segmented, size_t n, float (*time)(int, void *), void *ctx)
{
    TunerState &t = tuner();
    const auto key = tuneKey(segmented, n);
    {
        std::lock_guard<std::mutex> lock(t.mu);
        t.timing[key] = 1;  // other threads sort this class with the default meanwhile
    }
    struct Done
    {
        TunerState &t;
        std::tuple<int, int, int> key;
        ~Done()
        {
            std::lock_guard<std::mutex> lock(t.mu);
            t.timing.erase(key);
        }
    } done{t, key};
    int best = sort::kDefaultSortConfig;
    float bestMs = 0.f;
    for (int c = 0; c < sort::kNumSortConfigs; ++c)
    {
        time(c, ctx);  // first launches of a configuration load and set up its kernels
        const float ms = time(c, ctx);
        if (c == 0 || ms < bestMs)
        {
            best = c;
            bestMs = ms;
        }
    }
    std::lock_guard<std::mutex> lock(t.mu);
    t.chosen[key] = best;
    return best;
}

void sortSetAutotune(bool on)
{
    std::lock_guard<std::mutex> lock(tuner().mu);
    tuner().autotune = on;
}

void sortForceConfig(int config)
{
    if (config >= sort::kNumSortConfigs) throw std::invalid_argument("sort: unknown configuration");
    std::lock_guard<std::mutex> lock(tuner().mu);
    tuner().forced = config < 0 ? -1 : config;
}

void sortForgetTuning()
{
    std::lock_guard<std::mutex> lock(tuner().mu);
    tuner().chosen.clear();
}

// --------------------------------------------------------------------------
// stand-alone stable pair sort (cub::DeviceRadixSort::SortPairs semantics)
// --------------------------------------------------------------------------
namespace
{
struct PairSortLayout
{
    // altKeys | altVals | counters | status, each part 256-byte aligned.  The
    // counters part starts with the error word (and 3 pad words), so its
    // offset depends on n only and ao_sort_pairs_check can find it whatever
    // configuration ran; then hist[passes][256], bins[passes][256] and the
    // passes' tile counters.
    size_t altKeys = 0, altVals = 0, counters = 0, status = 0, total = 0, tiles = 0;
    int passes = 0;
    static constexpr size_t kCounterHead = 4;  // error word + padding (u32 words)
    static size_t up(size_t b) { return (b + 255) & ~size_t(255); }
    static size_t countersOffset(size_t n) { return up(up(n * sizeof(u64)) + n * sizeof(u32)); }
    PairSortLayout(size_t n, int cfg)
    {
        tiles = configTiles(cfg, n);
        passes = sort::configPasses(cfg);
        altKeys = 0;
        altVals = up(altKeys + n * sizeof(u64));
        counters = countersOffset(n);
        status = up(counters + counterWords() * sizeof(u32));
        total = up(status + size_t(passes) * tiles * sort::kRadix * sizeof(u64));
    }
    size_t counterWords() const { return kCounterHead + 2 * size_t(passes) * sort::kRadix + passes; }
};
}  // namespace

// The scratch a caller sizes must fit whichever configuration the tuner
// later picks, so the size query answers the largest.
void TreeEngine::sortPairs(void *scratch, size_t *scratchBytes, const unsigned long long *keysIn,
                           unsigned long long *keysOut, const unsigned *valsIn, unsigned *valsOut, size_t n,
                           int beginBit, int endBit, cudaStream_t s)
{
    if (!scratchBytes) throw std::invalid_argument("ao_sort_pairs: scratch_bytes must not be null");
    if (!scratch)
    {
        size_t most = 0;
        for (int c = 0; c < sort::kNumSortConfigs; ++c)
        {
            size_t b = 0;
            sortPairsWith(c, nullptr, &b, keysIn, keysOut, valsIn, valsOut, n, beginBit, endBit, s);
            most = std::max(most, b);
        }
        *scratchBytes = most;
        return;
    }
    sortPairsWith(sortTuning(false, n).config, scratch, scratchBytes, keysIn, keysOut, valsIn, valsOut, n, beginBit,
                  endBit, s);
}

void TreeEngine::sortPairsWith(int cfg, void *scratch, size_t *scratchBytes, const unsigned long long *keysIn,
                               unsigned long long *keysOut, const unsigned *valsIn, unsigned *valsOut, size_t n,
                               int beginBit, int endBit, cudaStream_t s)
{
    if (!scratchBytes) throw std::invalid_argument("ao_sort_pairs: scratch_bytes must not be null");
    if (beginBit < 0 || endBit > 64 || beginBit > endBit)
        throw std::invalid_argument("ao_sort_pairs: need 0 <= begin_bit <= end_bit <= 64");
    if (n > size_t(std::numeric_limits<std::uint32_t>::max()))
        throw std::invalid_argument("ao_sort_pairs: more than 2^32 - 1 items");
    if (cfg < 0 || cfg >= sort::kNumSortConfigs) throw std::invalid_argument("ao_sort_pairs: unknown configuration");
    const PairSortLayout lay(n, cfg);
    if (!scratch)
    {
        *scratchBytes = lay.total;
        return;
    }
    if (*scratchBytes < lay.total) throw std::invalid_argument("ao_sort_pairs: scratch too small");
    if (n == 0) return;
    if (!keysIn || !keysOut || !valsOut) throw std::invalid_argument("ao_sort_pairs: null array");
    if (keysIn == keysOut) throw std::invalid_argument("ao_sort_pairs: keys_in and keys_out must differ");
    char *base = static_cast<char *>(scratch);
    u64 *altK = reinterpret_cast<u64 *>(base + lay.altKeys);
    u32 *altV = reinterpret_cast<u32 *>(base + lay.altVals);
    u32 *head = reinterpret_cast<u32 *>(base + lay.counters);
    int *error = reinterpret_cast<int *>(head);
    u32 *ctr = head + PairSortLayout::kCounterHead;  // hist
    u64 *status = reinterpret_cast<u64 *>(base + lay.status);
    const int slots = lay.passes;  // rows of hist and bins
    u32 *bins = ctr + size_t(slots) * sort::kRadix;
    u32 *tileCounters = ctr + 2 * size_t(slots) * sort::kRadix;
    const int bitsPer = sort::kSortConfigs[cfg].bits;
    const int passes = (endBit - beginBit + bitsPer - 1) / bitsPer;
    if (passes == 0)
    {
        AOT_CHECK(cudaMemsetAsync(error, 0, sizeof(int), s));  // ao_sort_pairs_check reads it
        AOT_CHECK(cudaMemcpyAsync(keysOut, keysIn, n * sizeof(u64), cudaMemcpyDeviceToDevice, s));
        if (valsIn) AOT_CHECK(cudaMemcpyAsync(valsOut, valsIn, n * sizeof(u32), cudaMemcpyDeviceToDevice, s));
        else iotaKernel<<<gridFor(n, 256), 256, 0, s>>>(valsOut, n), noteLaunch();
        AOT_LAUNCH_CHECK();
        return;
    }
    AOT_CHECK(cudaMemsetAsync(head, 0, lay.counterWords() * sizeof(u32), s));
    AOT_CHECK(cudaMemsetAsync(status, 0, size_t(passes) * lay.tiles * sort::kRadix * sizeof(u64), s));
    const unsigned blocks = std::max(1u, std::min<unsigned>(ceilDiv(n, sort::kThreads), unsigned(smCount()) * 8u));
    sort::launchHistogram(cfg, s, blocks, reinterpret_cast<const u64 *>(keysIn), n, beginBit, passes, ctr, endBit),
        noteLaunch();
    sort::binsKernel<<<1, sort::kRadix, 0, s>>>(ctr, bins, passes), noteLaunch();
    AOT_LAUNCH_CHECK();
    sort::setPassSmemAll();
    const u64 *kin = reinterpret_cast<const u64 *>(keysIn);
    const u32 *vin = valsIn;
    for (int p = 0; p < passes; ++p)
    {
        // the last pass writes keysOut; earlier passes alternate backwards from it
        const bool toOut = ((passes - 1 - p) & 1) == 0;
        u64 *kout = toOut ? reinterpret_cast<u64 *>(keysOut) : altK;
        u32 *vout = toOut ? valsOut : altV;
        const int shift = beginBit + p * bitsPer;
        const int bits = std::min(bitsPer, endBit - shift);
        sort::launchPass(cfg, s, kin, vin, kout, vout, n, shift, bins + p * sort::kRadix, tileCounters + p,
                         status + size_t(p) * lay.tiles * sort::kRadix, error, bits),
            noteLaunch();
        AOT_LAUNCH_CHECK();
        kin = kout;
        vin = vout;
    }
}

// Waits for `stream` and reads the error word of a pair sort of n items
// that ran in `scratch` (the bounded look-back of some pass gave up, so its
// output is not a sorted permutation).
bool TreeEngine::sortPairsFailed(const void *scratch, size_t n, cudaStream_t s)
{
    if (!scratch) throw std::invalid_argument("ao_sort_pairs_check: null scratch");
    int error = 0;
    AOT_CHECK(cudaMemcpyAsync(&error, static_cast<const char *>(scratch) + PairSortLayout::countersOffset(n),
                              sizeof(int), cudaMemcpyDeviceToHost, s));
    AOT_CHECK(cudaStreamSynchronize(s));
    return error != 0;
}

// Loads every kernel a pair sort with the default configuration can launch
// (lazy module loading would otherwise load one at its first launch).
void TreeEngine::sortPairsPreload()
{
    cudaFuncAttributes a;
    AOT_CHECK(cudaFuncGetAttributes(&a, iotaKernel));
    AOT_CHECK(cudaFuncGetAttributes(&a, sort::binsKernel));
    AOT_CHECK(cudaFuncGetAttributes(&a, sort::histogramKernel<8>));
    AOT_CHECK(cudaFuncGetAttributes(&a, sort::histogramKernel<7>));
#define AOT_CASE(i, B, I) AOT_CHECK(cudaFuncGetAttributes(&a, sort::onesweepKernel<B, I>));
    AOT_SORT_CONFIGS(AOT_CASE)
#undef AOT_CASE
    sort::setPassSmemAll();
}

// --------------------------------------------------------------------------
// Impl
// --------------------------------------------------------------------------
struct TreeEngine::Impl
{
    // particles
    DevMem P[2], Perm[2], sample;
    SortArena sortArena;
    // state
    DevMem stMem;
    DeviceState *st = nullptr;   // device (stMem)
    DeviceState *hst = nullptr;  // pinned mirror (block cache)
    size_t hstBytes = 0;
    cudaStream_t d2h = nullptr;
    cudaEvent_t ready = nullptr;
    // level build: the neighbour references of a level run on `side` beside
    // the expansion of the same level (neither needs the other)
    cudaStream_t side = nullptr;
    cudaEvent_t sideFork = nullptr, sideJoin = nullptr;
    int device = 0;  // the device of the pooled streams and events
    cudaEvent_t marks[8] = {};              // stage events (profiling)
    cudaEvent_t tuneStart = nullptr, tuneEnd = nullptr;  // sort tuner timing
    std::vector<cudaEvent_t> nfMarks;       // begin/end pairs around near-field launches
    DevMem history;
    // tree
    DevMem K[2], B[2], NF[2], N[2], G[2], offs, dirty, scan;
    DevMem nodeRows;  // node table of the near-field refresh (NFCount)
    // converged build by levels (levelbuild.cuh): unit arena and its control
    DevMem lvRows, lvVal, lvChild, lvLeaves, lvOffset, lvCtl, lvNbr, lvParent;
    size_t lvCap = 0;
    int lvLevels = int(kOctLevels);  // levels the last level build needed, with one to spare
    DevMem mergeSplits;              // merge-path cuts of the full begin refresh
    unsigned char *lvHost = nullptr; // pinned: the level build's one readback
    size_t lvHostBytes = 0;
    // binary tree by levels (binlevel.cuh)
    DevMem blRows, blMid, blChild, blLeaves, blOffset, blCtl;
    size_t blCap = 0;
    int blLevels = bl::kLevels;      // depths the last binary build needed, with one to spare
    bl::Control *blHost = nullptr;   // pinned readback
    size_t blHostBytes = 0;
    u32 nodeSlots = 0;
    bool nodeStale = true;         // the keys changed or the table moved: clear before use
    size_t scanTiles = 0;
    // views
    DevMem vBox, vSplit, vDepth, vParent, vChild, vLevelOffset, vPbegin, vPcount, vPmap, vMaxDepth;
    DevMem vLeafLevel, vLeafToNode, vLevels, vCandStart, vCandLevel, vLvKeys[2], vLvVals[2], vLayKeys[2], vLayVals[2];
    DevMem vIntStartSfc, vIntLevelSfc, vIntM, vIntStartLay, vIntLevelLay;
    SortArena viewSort;
    size_t viewLeafCap = 0, viewParticleCap = 0;
    bool viewScratch = false;
    adaptive_octree::ViewConfig viewPrepared{};
    size_t viewNodesLogical = 0, mappingLogical = 0;
    // keys
    KeygenParams<float> kpf{};
    KeygenParams<double> kpd{};

    ~Impl()
    {
        if (hst) blockcache::giveHost(hst, hstBytes);
        if (lvHost) blockcache::giveHost(lvHost, lvHostBytes);
        if (blHost) blockcache::giveHost(blHost, blHostBytes);
        blockcache::giveEvent(ready, device);
        for (cudaEvent_t e : marks)
            if (e) cudaEventDestroy(e);
        if (tuneStart) cudaEventDestroy(tuneStart);
        if (tuneEnd) cudaEventDestroy(tuneEnd);
        for (cudaEvent_t e : nfMarks) cudaEventDestroy(e);
        blockcache::giveStream(d2h, device);
        blockcache::giveEvent(sideFork, device);
        blockcache::giveEvent(sideJoin, device);
        blockcache::giveStream(side, device);
    }

    // device bytes held by this tree
    size_t bytes() const
    {
        const DevMem *all[] = {&P[0],        &P[1],        &Perm[0],        &Perm[1],      &sample,
                               &sortArena.counters, &sortArena.status, &stMem, &history, &K[0],
                               &K[1],        &B[0],        &B[1],           &NF[0],        &NF[1],
                               &N[0],        &N[1],        &G[0],           &G[1],         &offs,
                               &dirty,       &scan,        &vBox,           &vSplit,       &vDepth,
                               &vParent,     &vChild,      &vLevelOffset,   &vPbegin,      &vPcount,
                               &vPmap,       &vMaxDepth,   &vLeafLevel,     &vLeafToNode,  &vLevels,
                               &vCandStart,  &vCandLevel,  &vLvKeys[0],     &vLvKeys[1],   &vLvVals[0],
                               &vLvVals[1],  &vLayKeys[0], &vLayKeys[1],    &vLayVals[0],  &vLayVals[1],
                               &vIntStartSfc, &vIntLevelSfc, &vIntM,        &vIntStartLay, &vIntLevelLay,
                               &viewSort.counters, &viewSort.status, &nodeRows, &lvRows, &lvVal, &lvChild,
                               &lvLeaves, &lvOffset, &lvCtl, &lvNbr, &lvParent};
        size_t s = 0;
        for (const DevMem *d : all) s += d->bytes;
        return s;
    }

    rb::TreeBufs bufs() const
    {
        rb::TreeBufs t{};
        for (int k = 0; k < 2; ++k)
        {
            t.K[k] = K[k].as<u64>();
            t.B[k] = B[k].as<u32>();
            t.NF[k] = NF[k].as<u32>();
            t.G[k] = G[k].as<u8>();
            t.N[k] = N[k].as<u32>();
        }
        t.offs = offs.as<i64>();
        t.dirty = dirty.as<int>();
        t.scanStatus = scan.as<u64>();
        t.scanTile = reinterpret_cast<u32 *>(scan.as<u64>() + scanTiles);
        t.st = st;
        return t;
    }
    KeyIndex keyIndex(size_t n) const
    {
        KeyIndex k{};
        k.keys = P[0].as<u64>();
        k.sample = sample.as<u64>();
        k.n = n;
        k.ns = (n + kSampleStride - 1) >> kSampleShift;
        return k;
    }
    tv::ViewBufs viewBufs() const
    {
        tv::ViewBufs v{};
        v.box = vBox.as<u64>();
        v.split = vSplit.as<u8>();
        v.depth = vDepth.as<u8>();
        v.parent = vParent.as<int>();
        v.child = vChild.as<int>();
        v.levelOffset = vLevelOffset.as<int>();
        v.pbegin = vPbegin.as<u32>();
        v.pcount = vPcount.as<u32>();
        v.pmap = vPmap.as<u64>();
        v.maxDepth = vMaxDepth.as<u8>();
        v.leafLevel = vLeafLevel.as<u8>();
        v.leafToNode = vLeafToNode.as<int>();
        int *lv = vLevels.as<int>();
        v.leavesPerLevel = lv;
        v.internalPerLevel = lv + 66;
        v.nodesPerLevel = lv + 2 * 66;
        v.levelOffsetInternal = lv + 3 * 66;
        v.candStart = vCandStart.as<u64>();
        v.candLevel = vCandLevel.as<u8>();
        v.lvKeys = vLvKeys[0].as<u64>();
        v.lvKeysAlt = vLvKeys[1].as<u64>();
        v.lvVals = vLvVals[0].as<u32>();
        v.lvValsAlt = vLvVals[1].as<u32>();
        v.layKeys = vLayKeys[0].as<u64>();
        v.layKeysAlt = vLayKeys[1].as<u64>();
        v.layVals = vLayVals[0].as<u32>();
        v.layValsAlt = vLayVals[1].as<u32>();
        v.intStartSfc = vIntStartSfc.as<u64>();
        v.intLevelSfc = vIntLevelSfc.as<u8>();
        v.intMBySfc = vIntM.as<int>();
        v.intStartLay = vIntStartLay.as<u64>();
        v.intLevelLay = vIntLevelLay.as<u8>();
        return v;
    }
};

// --------------------------------------------------------------------------
// construction
// --------------------------------------------------------------------------
TreeEngine::TreeEngine(const void *x, const void *y, const void *z, size_t n, const EngineConfig &cfg)
    : m_(std::make_unique<Impl>()), cfg_(cfg), n_(n), x_(x), y_(y), z_(z)
{
    // Backend constructor checks (octree.cu:321-416, kdtree3d.cu:175-216).
    if (n > 0 && (!x || !y || !z))
        throw std::invalid_argument("adaptive_octree: coordinate device pointers must not be null");
    if (cfg.bucket == 0) throw std::invalid_argument("adaptive_octree: particle limit must be positive");
    if (cfg.iterations == 0) throw std::invalid_argument("adaptive_octree: updateIterations must be positive");
    if (cfg.kind == 1) m_->kpd.g = makeGeometry(cfg.box, cfg.maxDepth, cfg.real), m_->kpf.g = m_->kpd.g;
    if (n > size_t(std::numeric_limits<std::uint32_t>::max()))
        throw std::invalid_argument(
            "adaptive_octree: particle count exceeds 32-bit permutation index range");
    m_->kpf.q = makeQuantBox<float>(cfg.box);
    m_->kpd.q = makeQuantBox<double>(cfg.box);
    m_->kpf.h = hilbertTables();
    m_->kpd.h = hilbertTables();
    prepared_ = cfg.views;

    // stream-ordered set-up: nothing here synchronises the device
    m_->stMem.reserve(sizeof(DeviceState));
    m_->st = m_->stMem.as<DeviceState>();
    AOT_CHECK(cudaMemsetAsync(m_->st, 0, sizeof(DeviceState), cfg.stream));
    m_->hst = static_cast<DeviceState *>(blockcache::takeHost(sizeof(DeviceState), &m_->hstBytes));
    std::memset(m_->hst, 0, sizeof(DeviceState));
    AOT_CHECK(cudaGetDevice(&m_->device));
    m_->d2h = blockcache::takeStream();
    m_->ready = blockcache::takeEvent();
    if (n)
    {
        for (int k = 0; k < 2; ++k)
        {
            m_->P[k].reserve(n * sizeof(u64));
            m_->Perm[k].reserve(n * sizeof(u32));
        }
        m_->sample.reserve(((n + kSampleStride - 1) >> kSampleShift) * sizeof(u64));
        m_->sortArena.ensure(n, sort::kDefaultSortConfig, cfg.stream);
    }
    ensurePhysical(16);
    if (cfg.kind == 0)
    {
        const u64 root[2] = {0, kMaxKey};
        AOT_CHECK(cudaMemcpyAsync(m_->K[0].p, root, sizeof(root), cudaMemcpyHostToDevice, cfg.stream));
        waitStream(cfg.stream);
    }
}

size_t TreeEngine::deviceBytes() const { return m_->bytes(); }

namespace
{
// dst[i] = src[perm[i]], W-byte words
template <class W>
__global__ void gatherKernel(const W *__restrict__ src, W *__restrict__ dst, const u32 *__restrict__ perm, size_t n)
{
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        dst[i] = src[perm[i]];
}
__global__ void gatherBytesKernel(const unsigned char *__restrict__ src, unsigned char *__restrict__ dst,
                                  const u32 *__restrict__ perm, size_t n, size_t e)
{
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    {
        const unsigned char *s = src + size_t(perm[i]) * e;
        for (size_t b = 0; b < e; ++b) dst[i * e + b] = s[b];
    }
}
}  // namespace

void TreeEngine::gather(const void *src, void *dst, size_t elemBytes) const
{
    if (n_ == 0) return;
    if (!src || !dst) throw std::invalid_argument("adaptive_octree: gather needs device source and destination");
    if (elemBytes == 0) throw std::invalid_argument("adaptive_octree: gather element size must be positive");
    if (src == dst) throw std::invalid_argument("adaptive_octree: gather cannot work in place");
    cudaStream_t s = cfg_.stream;
    const u32 *perm = m_->Perm[0].as<u32>();
    const unsigned blocks = std::min<unsigned>(gridFor(n_, 256), unsigned(smCount()) * 16u);
    const uintptr_t align = reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst);
    if (elemBytes == 4 && align % 4 == 0)
        gatherKernel<u32><<<blocks, 256, 0, s>>>(static_cast<const u32 *>(src), static_cast<u32 *>(dst), perm, n_), noteLaunch();
    else if (elemBytes == 8 && align % 8 == 0)
        gatherKernel<u64><<<blocks, 256, 0, s>>>(static_cast<const u64 *>(src), static_cast<u64 *>(dst), perm, n_), noteLaunch();
    else if (elemBytes == 16 && align % 16 == 0)
        gatherKernel<uint4><<<blocks, 256, 0, s>>>(static_cast<const uint4 *>(src), static_cast<uint4 *>(dst), perm, n_), noteLaunch();
    else
        gatherBytesKernel<<<blocks, 256, 0, s>>>(static_cast<const unsigned char *>(src), static_cast<unsigned char *>(dst),
                                                 perm, n_, elemBytes), noteLaunch();
    AOT_LAUNCH_CHECK();
}

// The buffers go back to the block cache: no queued work may still use them.
TreeEngine::~TreeEngine()
{
    if (m_)
    {
        (void)cudaStreamSynchronize(cfg_.stream);
        if (m_->d2h) (void)cudaStreamSynchronize(m_->d2h);
        if (m_->side) (void)cudaStreamSynchronize(m_->side);
    }
}

void TreeEngine::setCoordinates(const void *x, const void *y, const void *z)
{
    if (n_ > 0 && (!x || !y || !z))
        throw std::invalid_argument("adaptive_octree: coordinate device pointers must not be null");
    x_ = x;
    y_ = y;
    z_ = z;
}

// Physical capacity of the leaf buffers (>= leafCapacity at all times).
void TreeEngine::ensurePhysical(size_t capacity)
{
    if (capacity <= physCap_ && m_->K[0].p) return;
    cudaStream_t s = cfg_.stream;
    const size_t c = std::max(capacity, physCap_);
    for (int k = 0; k < 2; ++k)
    {
        m_->K[k].grow((c + 1) * sizeof(u64), m_->K[k].bytes, s);
        m_->B[k].grow((c + 1) * sizeof(u32), m_->B[k].bytes, s);
        m_->N[k].grow((c + 1) * sizeof(u32), m_->N[k].bytes, s);
        if (cfg_.kind == 0 && cfg_.nf)
        {
            m_->NF[k].grow((c + 1) * sizeof(u32), m_->NF[k].bytes, s);
            m_->G[k].grow((c + 1) * sizeof(u8), m_->G[k].bytes, s);
        }
        else
        {
            // nearFieldCounts_d of a LeafCount tree (or a binary tree) is never
            // written: it reads as zeros, as the reference's value-initialised vector
            const size_t before = m_->NF[k].bytes;
            m_->NF[k].grow(sizeof(u32) * (c + 1), m_->NF[k].bytes, s);
            if (m_->NF[k].bytes != before) AOT_CHECK(cudaMemsetAsync(m_->NF[k].p, 0, m_->NF[k].bytes, s));
            m_->G[k].grow(16, m_->G[k].bytes, s);
        }
    }
    m_->offs.reserve((c + 1) * sizeof(i64), s);
    m_->dirty.reserve((c + 1) * sizeof(int), s);
    // the merge-path cuts of the full begin refresh (reserved here: an update
    // may run under stream capture, where nothing may be allocated)
    m_->mergeSplits.reserve(((c + 1 + n_) / rb::kMergeChunk + 3) * sizeof(u32), s);
    // candidate group leaders are first children of distinct internal nodes: <= (L - 1) / 7
    m_->scanTiles = (c + 1 + rb::kScanTile - 1) / rb::kScanTile;
    m_->scan.reserve((m_->scanTiles + 1) * sizeof(u64), s);
    if (cfg_.kind == 0 && cfg_.nf)
    {
        // every internal node of the tree (about a seventh of the leaves) and
        // cells that were internal nodes since the last sort, with room to
        // spare: linear probing stays short
        const size_t slots = std::min<size_t>(c / 4 + 1024, 0xffffffffu);
        if (slots > m_->nodeSlots)
        {
            m_->nodeRows.reserve(slots * rb::kGroupRow * sizeof(u32), s);
            m_->nodeSlots = u32(slots);
            m_->nodeStale = true;
        }
    }
    physCap_ = c;
}

// --------------------------------------------------------------------------
// keys + sort (octree.cu:285-307, kdtree3d.cu:161-172)
// --------------------------------------------------------------------------
void TreeEngine::sortParticles()
{
    m_->nodeStale = true;  // cell table entries hold indices into the sorted keys
    if (n_ == 0) return;
    cudaStream_t s = cfg_.stream;
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    AOT_CHECK(cudaStreamIsCapturing(s, &capture));
    if (capture == cudaStreamCaptureStatusNone && cfg_.tuneSort && sortNeedsTuning(false, n_))
    {
        // every configuration sorts identically, so the keys of the last
        // timed run are the sorted keys
        if (!m_->tuneStart) AOT_CHECK(cudaEventCreate(&m_->tuneStart));
        if (!m_->tuneEnd) AOT_CHECK(cudaEventCreate(&m_->tuneEnd));
        m_->sortArena.ensure(n_, -1, s);
        auto time = [](int c, void *ctx) -> float {
            TreeEngine &e = *static_cast<TreeEngine *>(ctx);
            AOT_CHECK(cudaEventRecord(e.m_->tuneStart, e.cfg_.stream));
            e.sortKeys(c);
            AOT_CHECK(cudaEventRecord(e.m_->tuneEnd, e.cfg_.stream));
            AOT_CHECK(cudaEventSynchronize(e.m_->tuneEnd));
            float ms = 0.f;
            AOT_CHECK(cudaEventElapsedTime(&ms, e.m_->tuneStart, e.m_->tuneEnd));
            return ms;
        };
        const int best = sortTune(false, n_, time, this);
        // keep only the chosen configuration's status words
        waitStream(s);
        m_->sortArena.status.release();
        m_->sortArena.ensure(n_, best, s);
    }
    else if (capture != cudaStreamCaptureStatusNone && sortConfig_ >= 0)
    {
        sortKeys(sortConfig_);  // under capture: the last sort's configuration and scratch
    }
    else
    {
        const int config = sortTuning(false, n_).config;
        m_->sortArena.ensure(n_, config, s);
        sortKeys(config);
    }
    const KeyIndex idx = m_->keyIndex(n_);
    rb::sampleKeysKernel<<<gridFor(idx.ns, 256), 256, 0, s>>>(m_->P[0].as<u64>(), n_, m_->sample.as<u64>(), idx.ns),
        noteLaunch();
    AOT_LAUNCH_CHECK();
}

// Keys of every particle, then the stable (key, slot) sort with sort
// configuration `config`; the result lands in P[0] / Perm[0].
void TreeEngine::sortKeys(int config)
{
    cudaStream_t s = cfg_.stream;
    SortArena &a = m_->sortArena;
    const int passes = sort::configPasses(config);
    if (passes & 1) throw std::logic_error("adaptive_octree: sort configurations must have an even pass count");
    clearArena(config, s, a, n_, passes);
    u64 *k[2] = {m_->P[0].as<u64>(), m_->P[1].as<u64>()};
    u32 *v[2] = {m_->Perm[0].as<u32>(), m_->Perm[1].as<u32>()};
    // 8-bit digits: the histogram comes with the keys; otherwise a pass of its own
    const bool fused = sort::kSortConfigs[config].bits == sort::kRadixBits;
    const int histPasses = fused ? sort::kMaxPasses : 0;
    if (cfg_.real == 0)
        launchKeygen<float>(cfg_.kind, cfg_.hilbert, static_cast<const float *>(x_), static_cast<const float *>(y_),
                            static_cast<const float *>(z_), n_, m_->kpf, k[0], a.hist(), histPasses, s);
    else
        launchKeygen<double>(cfg_.kind, cfg_.hilbert, static_cast<const double *>(x_), static_cast<const double *>(y_),
                             static_cast<const double *>(z_), n_, m_->kpd, k[0], a.hist(), histPasses, s);
    if (!fused)
    {
        const unsigned blocks = std::max(1u, std::min<unsigned>(ceilDiv(n_, sort::kThreads), unsigned(smCount()) * 8u));
        sort::launchHistogram(config, s, blocks, k[0], n_, 0, passes, a.hist(), 64), noteLaunch();
        AOT_LAUNCH_CHECK();
    }
    runPasses(config, s, k, v, n_, 0, 64, true, a, &m_->st->error);  // an even pass count ends in buffer 0
    sortConfig_ = config;
}

void TreeEngine::computeKeys(int kind, int real, const void *x, const void *y, const void *z, size_t n,
                             const double *box, bool hilbert, unsigned maxDepth, unsigned long long *keys,
                             unsigned *perm, cudaStream_t s)
{
    if (n == 0) return;
    if (n > size_t(std::numeric_limits<std::uint32_t>::max()))
        throw std::invalid_argument("adaptive_octree: particle count exceeds 32-bit permutation index range");
    KeygenParams<float> pf{};
    KeygenParams<double> pd{};
    if (kind == 1) pd.g = pf.g = makeGeometry(box, maxDepth, real);
    pf.q = makeQuantBox<float>(box);
    pd.q = makeQuantBox<double>(box);
    pf.h = pd.h = hilbertTables();
    if (real == 0)
        launchKeygen<float>(kind, hilbert, static_cast<const float *>(x), static_cast<const float *>(y),
                            static_cast<const float *>(z), n, pf, reinterpret_cast<u64 *>(keys), nullptr, 0, s);
    else
        launchKeygen<double>(kind, hilbert, static_cast<const double *>(x), static_cast<const double *>(y),
                             static_cast<const double *>(z), n, pd, reinterpret_cast<u64 *>(keys), nullptr, 0, s);
    if (perm)
    {
        iotaKernel<<<gridFor(n, 256), 256, 0, s>>>(perm, n), noteLaunch();
        AOT_LAUNCH_CHECK();
    }
}

// --------------------------------------------------------------------------
// rebalance passes
// --------------------------------------------------------------------------
namespace
{
__global__ void octInitRootKernel(rb::TreeBufs tb, const u64 *P, size_t n)
{
    DeviceState *st = tb.st;
    const unsigned active = n ? unsigned(lowerBoundDev(P, n, kMaxKey)) : 0u;
    tb.K[0][0] = 0;
    tb.K[0][1] = kMaxKey;
    tb.B[0][0] = 0;
    tb.B[0][1] = active;
    const u64 sq = u64(active) * active;
    tb.NF[0][0] = sq > 0xffffffffull / 27ull ? 0xffffffffu : u32(27ull * sq);  // octree.cu:23-38
    const int err = st->error;
    *st = DeviceState{};
    st->error = err;
    st->numLeaves = 1;
    st->newNumLeaves = 1;
    st->numActiveParticles = active;
}

// finishBuildStateKernel (octree.cu:40-47)
__global__ void octFinishBuildKernel(DeviceState *st)
{
    st->newNumLeaves = st->numLeaves;
    st->changed = st->converged = st->needsResize = 0;
    st->numNodes = 0;
    st->activeBuffer = 0;
    st->overflow = 0;
}

// initBinaryRootKernel (kdtree3d.cu:24-30)
__global__ void binInitRootKernel(rb::TreeBufs tb, long long logicalCap)
{
    DeviceState *st = tb.st;
    tb.K[0][0] = 0;
    tb.K[0][1] = kMaxKey;
    const int err = st->error;
    *st = DeviceState{};
    st->error = err;
    st->numLeaves = 1;
    st->newNumLeaves = 1;
    st->numNodes = 1;
    st->logicalCap = logicalCap;
}

__global__ void clearOverflowKernel(DeviceState *st) { st->overflow = 0; }
}  // namespace

void TreeEngine::octreePass(bool buildMode, long long limit)
{
    cudaStream_t s = cfg_.stream;
    const rb::TreeBufs tb = m_->bufs();
    const size_t cap = buildMode ? physCap_ : leafCapacity_;
    const size_t tiles = (cap + 1 + rb::kScanTile - 1) / rb::kScanTile;
    rb::beginPassKernel<<<1, 1, 0, s>>>(m_->st), noteLaunch();
    AOT_CHECK(cudaMemsetAsync(m_->scan.p, 0, (m_->scanTiles + 1) * sizeof(u64), s));
    const int mode = buildMode ? kModeOctreeBuild : kModeUpdate;
    long long *hist = buildMode ? m_->history.as<long long>() : nullptr;
    const unsigned scatterBlocks = std::min(gridFor(cap, rb::kScatterThreads), unsigned(smCount()) * 8u);
    const unsigned refreshBlocks = unsigned(smCount()) * 8u;
    if (cfg_.nf)
    {
        rb::octDecideScanKernel<true><<<unsigned(tiles), rb::kScanThreads, 0, s>>>(tb, cfg_.bucket), noteLaunch();
        rb::octScatterKernel<true><<<scatterBlocks, rb::kScatterThreads, 0, s>>>(tb, limit, mode, hist), noteLaunch();
    }
    else
    {
        rb::octDecideScanKernel<false><<<unsigned(tiles), rb::kScanThreads, 0, s>>>(tb, cfg_.bucket), noteLaunch();
        rb::octScatterKernel<false><<<scatterBlocks, rb::kScatterThreads, 0, s>>>(tb, limit, mode, hist), noteLaunch();
    }
    AOT_LAUNCH_CHECK();
    refreshCounts(false, refreshBlocks);
    AOT_LAUNCH_CHECK();
}

void TreeEngine::binaryPass(bool buildMode, long long limit)
{
    cudaStream_t s = cfg_.stream;
    const rb::TreeBufs tb = m_->bufs();
    const size_t cap = buildMode ? physCap_ : leafCapacity_;
    const size_t tiles = (cap + 1 + rb::kScanTile - 1) / rb::kScanTile;
    rb::beginPassKernel<<<1, 1, 0, s>>>(m_->st), noteLaunch();
    AOT_CHECK(cudaMemsetAsync(m_->scan.p, 0, (m_->scanTiles + 1) * sizeof(u64), s));
    const KeyIndex idx = m_->keyIndex(n_);
    rb::binDecideScanKernel<<<unsigned(tiles), rb::kScanThreads, 0, s>>>(tb, cfg_.bucket, cfg_.maxDepth), noteLaunch();
    rb::binScatterKernel<<<std::min(gridFor(cap, rb::kScatterThreads), unsigned(smCount()) * 8u), rb::kScatterThreads, 0, s>>>(
        tb, limit, buildMode ? kModeBinaryBuild : kModeUpdate), noteLaunch();
    rb::binRefreshKernel<false><<<unsigned(smCount()) * 8u, 256, 0, s>>>(tb, idx), noteLaunch();
    AOT_LAUNCH_CHECK();
}

// Full refresh of the per-leaf quantities of the active tree, after the
// reset of changed/converged/active count (resetRebalanceStateKernel +
// refreshGraphCountsGpu without dirty lists).
void TreeEngine::refreshAll()
{
    cudaStream_t s = cfg_.stream;
    const rb::TreeBufs tb = m_->bufs();
    const KeyIndex idx = m_->keyIndex(n_);
    rb::resetForUpdateKernel<<<1, 32, 0, s>>>(m_->st, m_->P[0].as<u64>(), n_), noteLaunch();
    const unsigned blocks = unsigned(smCount()) * 8u;
    if (cfg_.kind == 1)
    {
        rb::binRefreshKernel<true><<<blocks, 256, 0, s>>>(tb, idx), noteLaunch();
        AOT_LAUNCH_CHECK();
    }
    else
    {
        refreshCounts(true, blocks);
    }
}

// The digit -> block position table of the near-field kernel, once per device.
static void ensureDigitPos()
{
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    AOT_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64 || done[dev]) return;
    const HilbertTables h = makeHilbertTables();
    std::vector<unsigned long long> t(2 * 27 * 48);
    for (int hil = 0; hil < 2; ++hil)
        for (int q = 0; q < 27; ++q)
            for (int st = 0; st < 48; ++st)
            {
                unsigned long long packed = 0;
                for (int d = 0; d < 8; ++d)
                {
                    // block coordinate 2 * offset + child bit + 1 per axis, where Q touches P
                    const int o = hil ? h.decOct[st * 8 + d] : d;
                    const int dq[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
                    const int bit[3] = {o >> 2, (o >> 1) & 1, o & 1};
                    bool ok = true;
                    int p = 0;
                    for (int ax = 0; ax < 3; ++ax)
                    {
                        if ((dq[ax] < 0 && bit[ax] == 0) || (dq[ax] > 0 && bit[ax] == 1)) ok = false;
                        p = p * 4 + (2 * dq[ax] + bit[ax] + 1);
                    }
                    packed |= (unsigned long long)(ok ? p : 0xff) << (8 * d);
                }
                t[(hil * 27 + q) * 48 + st] = packed;
            }
    AOT_CHECK(cudaMemcpyToSymbol(rb::gDigitPos, t.data(), t.size() * sizeof(unsigned long long)));
    done[dev] = true;
}

// Per-leaf quantities of the active octree: begin indices, then (NFCount)
// near-field counts and group-merge flags.  all = every leaf, else the work
// lists of the last materialisation.
void TreeEngine::refreshCounts(bool all, unsigned blocks)
{
    cudaStream_t s = cfg_.stream;
    const rb::TreeBufs tb = m_->bufs();
    const KeyIndex idx = m_->keyIndex(n_);
    if (all)
    {
        // every leaf: a merge of the leaf keys with the particle keys
        const size_t chunks = (physCap_ + 1 + n_) / rb::kMergeChunk + 2;  // cuts: reserved by ensurePhysical
        const u64 *P = m_->P[0].as<u64>();
        rb::mergeSplitKernel<<<gridFor(chunks + 1, 256), 256, 0, s>>>(tb, P, m_->mergeSplits.as<u32>()), noteLaunch();
        rb::mergeBeginKernel<<<unsigned(std::min<size_t>(chunks, size_t(smCount()) * 8u)), 256, 0, s>>>(
            tb, P, m_->mergeSplits.as<u32>()),
            noteLaunch();
    }
    else
    {
        rb::octBeginKernel<false><<<blocks, rb::kRefreshThreads, 0, s>>>(tb, idx), noteLaunch();
    }
    if (cfg_.nf)
    {
        const HilbertTables &h = m_->kpd.h;
        const rb::NodeTable gt{m_->nodeRows.as<u32>(), m_->nodeSlots};
        ensureDigitPos();
        // a cleared table takes the nodes of every leaf, else those of the new leaves
        const bool fill = all || m_->nodeStale;
        if (m_->nodeStale)
        {
            AOT_CHECK(cudaMemsetAsync(gt.rows, 0, size_t(gt.slots) * rb::kGroupRow * sizeof(u32), s));
            m_->nodeStale = false;
        }
        if (fill) rb::nodeTableKernel<true><<<blocks, rb::kRefreshThreads, 0, s>>>(tb, gt), noteLaunch();
        else rb::nodeTableKernel<false><<<blocks, rb::kRefreshThreads, 0, s>>>(tb, gt), noteLaunch();
        markNearField(true);
        if (all && cfg_.hilbert)
            rb::octNearFieldKernel<true, true><<<blocks, rb::kRefreshThreads, 0, s>>>(tb, idx, cfg_.bucket, h, gt), noteLaunch();
        else if (all)
            rb::octNearFieldKernel<false, true><<<blocks, rb::kRefreshThreads, 0, s>>>(tb, idx, cfg_.bucket, h, gt), noteLaunch();
        else if (cfg_.hilbert)
            rb::octNearFieldKernel<true, false><<<blocks, rb::kRefreshThreads, 0, s>>>(tb, idx, cfg_.bucket, h, gt), noteLaunch();
        else
            rb::octNearFieldKernel<false, false><<<blocks, rb::kRefreshThreads, 0, s>>>(tb, idx, cfg_.bucket, h, gt), noteLaunch();
        markNearField(false);
    }
    AOT_LAUNCH_CHECK();
}

void TreeEngine::materializeCounts()
{
    rb::materializeCountsKernel<<<gridFor(std::max(leafCapacity_, physCap_), 256), 256, 0, cfg_.stream>>>(m_->bufs()), noteLaunch();
    AOT_LAUNCH_CHECK();
}

// --------------------------------------------------------------------------
// state readback (octree.cu:498-537, kdtree3d.cu:127-137)
// --------------------------------------------------------------------------
void TreeEngine::readState()
{
    AOT_CHECK(cudaEventRecord(m_->ready, cfg_.stream));
    AOT_CHECK(cudaStreamWaitEvent(m_->d2h, m_->ready, 0));
    AOT_CHECK(cudaMemcpyAsync(m_->hst, m_->st, sizeof(DeviceState), cudaMemcpyDeviceToHost, m_->d2h));
    waitStream(m_->d2h);
    applyState();
}

// The host's copies of the state from the mirror (filled by a readback, or
// by the host where it knows every value).
void TreeEngine::applyState()
{
    const DeviceState &h = *m_->hst;
    if (h.error) throw std::runtime_error("adaptive_octree: a device scan gave up waiting (bounded look-back)");
    hostActiveBuffer_ = h.activeBuffer;
    hostLeaves_ = size_t(std::max(h.numLeaves, 0));
    hostActive_ = h.numActiveParticles;
    hostNodes_ = size_t(std::max(h.numNodes, 0));
    if (cfg_.kind == 0) capModel_.stateRead(hostLeaves_);
    syncViewSizes();
}

bool TreeEngine::doBuffersNeedResize()
{
    if (!built_) return false;
    readState();
    return m_->hst->needsResize != 0;
}

// --------------------------------------------------------------------------
// capacity (octree.cu:182-241, kdtree3d.cu:96-116)
// --------------------------------------------------------------------------

void TreeEngine::prepareGraphBuffers(size_t capacity)
{
    if (cfg_.kind == 0)
    {
        const size_t maxLeaves = (size_t(std::numeric_limits<int>::max()) - 1) / 8 * 7 + 1;
        if (capacity > maxLeaves) throw std::length_error("adaptive_octree: buffer capacity exceeds node index range");
        leafCapacity_ = capacity;
        capModel_.prepare(capacity);
        ensurePhysical(capacity);
        prepareViews(capacity, prepared_);
        syncViewSizes();
    }
    else
    {
        const size_t maxLeaves = size_t(std::numeric_limits<int>::max()) / 2 + 1;
        if (capacity > maxLeaves) throw std::length_error("adaptive_octree: buffer capacity exceeds node index range");
        leafCapacity_ = capacity;
        ensurePhysical(capacity);
        if (built_ && prepared_.treeStructure | prepared_.particleCountsPerBox | prepared_.particleMapping)
            prepareViews(capacity, prepared_);
        syncViewSizes();
    }
}

void TreeEngine::resizeBuffers()
{
    if (!built_) throw std::logic_error("adaptive_octree: call build() before resizeBuffers()");
    readState();
    prepareGraphBuffers(leafCapacity_ + (leafCapacity_ + 3) / 4);
    AOT_CHECK(cudaMemsetAsync(&m_->st->needsResize, 0, sizeof(int), cfg_.stream));
    waitStream(cfg_.stream);
}

// --------------------------------------------------------------------------
// build / update
// --------------------------------------------------------------------------
void TreeEngine::build()
{
    if (cfg_.kind == 0) octreeBuild();
    else binaryBuild();
}

void TreeEngine::octreeBuild()
{
    cudaStream_t s = cfg_.stream;
    waitStream(s);
    mark(MarkStart, 1);
    capModel_.buildStart();
    sortParticles();
    mark(MarkSorted);
    // Room for the build; grown on overflow.
    const size_t estimate = std::max<size_t>(4096, cfg_.nf ? n_ + 4096 : n_ / 4 + 4096);
    ensurePhysical(std::max(physCap_, estimate));
    std::vector<long long> proposals;
    lastBuildByLevels_ = buildMode_ == 0 && octreeLevelBuild(proposals);
    size_t leaves = 0;
    if (lastBuildByLevels_)
    {
        leaves = hostLeaves_;
    }
    else
    {
        m_->history.reserve(std::max<size_t>(cfg_.maxDepth, 1) * sizeof(long long), cfg_.stream);
        rb::TreeBufs tb = m_->bufs();
        octInitRootKernel<<<1, 1, 0, s>>>(tb, m_->P[0].as<u64>(), n_), noteLaunch();
        AOT_LAUNCH_CHECK();
        // rebalanceBuild (octree.cu:159-180): at most maxDepth decision rounds
        int done = 0;
        const int maxRounds = int(cfg_.maxDepth);
        while (done < maxRounds)
        {
            const int batch = std::min(4, maxRounds - done);
            for (int r = 0; r < batch; ++r) octreePass(true, (long long)physCap_);
            AOT_CHECK(cudaMemcpyAsync(m_->hst, m_->st, sizeof(DeviceState), cudaMemcpyDeviceToHost, s));
            waitStream(s);
            const DeviceState h = *m_->hst;
            if (h.error) throw std::runtime_error("adaptive_octree: a device scan gave up waiting (bounded look-back)");
            done = h.rounds;
            if (h.converged) break;
            if (h.overflow)
            {
                const size_t need = size_t(h.proposal);
                ensurePhysical(std::max(need + need / 4, 2 * physCap_));
                clearOverflowKernel<<<1, 1, 0, s>>>(m_->st), noteLaunch();
                AOT_LAUNCH_CHECK();
            }
        }
        AOT_CHECK(cudaMemcpyAsync(m_->hst, m_->st, sizeof(DeviceState), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        const DeviceState h = *m_->hst;
        proposals.resize(size_t(h.iteration));
        if (h.iteration)
            AOT_CHECK(cudaMemcpy(proposals.data(), m_->history.p, proposals.size() * sizeof(long long),
                                 cudaMemcpyDeviceToHost));
        leaves = size_t(h.numLeaves);
        // The final tree must sit in buffer 0 (finishBuildStateKernel resets the
        // active buffer).
        if (h.activeBuffer == 1)
        {
            AOT_CHECK(cudaMemcpyAsync(m_->K[0].p, m_->K[1].p, (leaves + 1) * sizeof(u64), cudaMemcpyDeviceToDevice, s));
            AOT_CHECK(cudaMemcpyAsync(m_->B[0].p, m_->B[1].p, (leaves + 1) * sizeof(u32), cudaMemcpyDeviceToDevice, s));
            if (cfg_.nf)
            {
                AOT_CHECK(cudaMemcpyAsync(m_->NF[0].p, m_->NF[1].p, leaves * sizeof(u32), cudaMemcpyDeviceToDevice, s));
                AOT_CHECK(cudaMemcpyAsync(m_->G[0].p, m_->G[1].p, leaves * sizeof(u8), cudaMemcpyDeviceToDevice, s));
            }
        }
        octFinishBuildKernel<<<1, 1, 0, s>>>(m_->st), noteLaunch();
        AOT_LAUNCH_CHECK();
    }
    mark(MarkPassed);
    buildRounds_ = int(proposals.size());
    hostLeaves_ = leaves;
    // Replay the reference's K_d/tmpTree capacity history (octree.cu:159-180,
    // 453-457; resizeWithHeadroom, helpers.cuh:122-141).
    const size_t cap = capModel_.finishBuild(proposals.data(), proposals.size(), leaves);
    prepareGraphBuffers(cap);
    built_ = true;
    if (!lastBuildByLevels_) materializeCounts();  // the placement of a build by levels writes the counts
    buildViews(cfg_.views);
    mark(MarkEnd);
    // the state read at the end of a build (doBuffersNeedResize); a build by
    // levels without views already knows every value of the state
    const bool views = cfg_.views.treeStructure | cfg_.views.particleCountsPerBox | cfg_.views.particleMapping;
    if (lastBuildByLevels_ && !views) applyState();
    else (void)doBuffersNeedResize();
}

void TreeEngine::setBuildMode(int mode)
{
    if (mode != 0 && mode != 1) throw std::invalid_argument("adaptive_octree: build mode must be 0 (levels) or 1 (rounds)");
    buildMode_ = mode;
}

// The converged octree, level by level (levelbuild.cuh).  The tree is the
// one the reference's build rounds converge to; the round history (leaves
// after each round that changed the tree) comes from the per-region counts.
bool TreeEngine::octreeLevelBuild(std::vector<long long> &proposals)
{
    if (!cfg_.nf && u64(cfg_.bucket) * 512u > 0xffffffffull) return false;  // wrapping split thresholds
    cudaStream_t s = cfg_.stream;
    Impl &m = *m_;
    const bool nf = cfg_.nf;
    // NFCount trees (deep levels of many units) classify, count and place
    // with 8 CTAs per SM (an A/B at 16 Mi: 3.49 ms with 4, 3.40 ms with 8,
    // 3.42 ms with 16); LeafCount trees keep 4
    const unsigned blocks = unsigned(smCount()) * 4u;
    const unsigned wide = nf ? 2u : 1u;
    const KeyIndex idx = m.keyIndex(n_);
    const u64 *P = m.P[0].as<u64>();
    size_t cap = std::max<size_t>(m.lvCap, n_ / 4 + 4096);
    constexpr size_t kHeadBytes = (sizeof(lb::Control) + 255) & ~size_t(255);
    constexpr size_t kCtlBytes = kHeadBytes + (lb::kContribBins + lb::kArrivals) * sizeof(unsigned long long);
    if (!m.lvHost)
        m.lvHost = static_cast<unsigned char *>(blockcache::takeHost(kCtlBytes + 16, &m.lvHostBytes));
    unsigned char *host = m.lvHost;
    const lb::Control &hc = *reinterpret_cast<const lb::Control *>(host);
    for (;;)
    {
        if (cap >= (size_t(1) << 28)) return false;  // neighbour references hold unit * 8 + digit in 31 bits
        m.lvRows.reserve(cap * lb::kRow * sizeof(u32), s);
        if (nf)
        {
            m.lvVal.reserve(cap * 8 * sizeof(u32), s);
            m.lvNbr.reserve(cap * 27 * sizeof(u32), s);
            m.lvParent.reserve(cap * sizeof(u32), s);
        }
        m.lvChild.reserve(cap * 8 * sizeof(u32), s);
        m.lvLeaves.reserve(cap * sizeof(u32), s);
        m.lvOffset.reserve(cap * sizeof(u32), s);
        m.lvCtl.reserve(kCtlBytes, s);
        m.lvCap = cap;
        lb::Arena a{};
        a.rows = m.lvRows.as<u32>();
        a.val = nf ? m.lvVal.as<u32>() : nullptr;
        a.nbr = nf ? m.lvNbr.as<u32>() : nullptr;
        a.parent = nf ? m.lvParent.as<u32>() : nullptr;
        a.usys = nullptr;
        a.sysRoot = nullptr;
        a.child = m.lvChild.as<u32>();
        a.leaves = m.lvLeaves.as<u32>();
        a.offset = m.lvOffset.as<u32>();
        a.ctl = m.lvCtl.as<lb::Control>();
        a.contrib = reinterpret_cast<unsigned long long *>(m.lvCtl.as<unsigned char>() + kHeadBytes);
        a.landed = a.contrib + lb::kContribBins;
        a.cap = u32(cap);
        AOT_CHECK(cudaMemsetAsync(m.lvCtl.p, 0, kCtlBytes, s));
        if (nf) ensureDigitPos();
        lb::rootKernel<<<1, 32, 0, s>>>(a, m.bufs(), P, n_, cfg_.bucket, nf ? 1 : 0), noteLaunch();
        AOT_LAUNCH_CHECK();
        // Every kernel reads its level's size on the device, so the whole
        // build is queued without a host wait: the levels the last build
        // needed (all 21 the first time), their subtree counts and the
        // placement; one readback at the end checks that no deeper level
        // was left out.
        const int levels = std::max(1, std::min(int(kOctLevels), m.lvLevels));
        const bool useSide = nf;
        if (useSide && !m.side)
        {
            m.side = blockcache::takeStream();
            m.sideFork = blockcache::takeEvent();
            m.sideJoin = blockcache::takeEvent();
        }
        for (int l = 0; l < levels; ++l)
        {
            const bool fork = nf && l > 0 && useSide;
            if (fork)
            {
                // the neighbour references of level l need level l - 1 only
                AOT_CHECK(cudaEventRecord(m.sideFork, s));
                AOT_CHECK(cudaStreamWaitEvent(m.side, m.sideFork, 0));
                if (cfg_.hilbert) lb::nbrKernel<true><<<blocks * 2, lb::kThreads, 0, m.side>>>(a, l, m.kpd.h), noteLaunch();
                else lb::nbrKernel<false><<<blocks * 2, lb::kThreads, 0, m.side>>>(a, l, m.kpd.h), noteLaunch();
                AOT_CHECK(cudaEventRecord(m.sideJoin, m.side));
            }
            lb::expandKernel<<<blocks * 2, lb::kThreads, 0, s>>>(a, idx, l), noteLaunch();
            if (fork) AOT_CHECK(cudaStreamWaitEvent(s, m.sideJoin, 0));
            if (nf)
            {
                markNearField(true);
                if (cfg_.hilbert)
                {
                    if (l > 0 && !fork) lb::nbrKernel<true><<<blocks * 2, lb::kThreads, 0, s>>>(a, l, m.kpd.h), noteLaunch();
                    lb::nearFieldKernel<true><<<blocks / 4 * 5, lb::kThreads, 0, s>>>(a, idx, l, m.kpd.h), noteLaunch();
                }
                else
                {
                    if (l > 0 && !fork) lb::nbrKernel<false><<<blocks * 2, lb::kThreads, 0, s>>>(a, l, m.kpd.h), noteLaunch();
                    lb::nearFieldKernel<false><<<blocks / 4 * 5, lb::kThreads, 0, s>>>(a, idx, l, m.kpd.h), noteLaunch();
                }
                markNearField(false);
                if (cfg_.hilbert)
                    lb::classifyKernel<true, true><<<blocks * wide, lb::kThreads, 0, s>>>(a, l, cfg_.bucket, m.kpd.h), noteLaunch();
                else
                    lb::classifyKernel<true, false><<<blocks * wide, lb::kThreads, 0, s>>>(a, l, cfg_.bucket, m.kpd.h), noteLaunch();
            }
            else
            {
                lb::classifyKernel<false, false><<<blocks, lb::kThreads, 0, s>>>(a, l, cfg_.bucket, m.kpd.h), noteLaunch();
            }
            AOT_LAUNCH_CHECK();
        }
        for (int l = levels - 1; l >= 0; --l)
            lb::leafCountKernel<<<blocks * wide, lb::kThreads, 0, s>>>(a, l, levels), noteLaunch();
        AOT_LAUNCH_CHECK();
        auto place = [&]() {
            const rb::TreeBufs tb = m.bufs();
            for (int l = 0; l < levels; ++l)
            {
                if (nf)
                    lb::placeKernel<true><<<blocks * wide, lb::kThreads, 0, s>>>(a, tb.K[0], tb.B[0], tb.NF[0], tb.N[0], l, levels,
                                                                          u32(physCap_)),
                        noteLaunch();
                else
                    lb::placeKernel<false><<<blocks, lb::kThreads, 0, s>>>(a, tb.K[0], tb.B[0], nullptr, tb.N[0], l, levels,
                                                                           u32(physCap_)),
                        noteLaunch();
            }
            AOT_LAUNCH_CHECK();
        };
        place();
        // the round history is needed before finishKernel writes it; read
        // everything once
        // (with the device state: its active count, set by the root kernel)
        AOT_CHECK(cudaMemcpyAsync(host, m.lvCtl.p, kCtlBytes, cudaMemcpyDeviceToHost, s));
        AOT_CHECK(cudaMemcpyAsync(host + kCtlBytes, a.leaves, sizeof(u32), cudaMemcpyDeviceToHost, s));
        AOT_CHECK(cudaMemcpyAsync(m.hst, m.st, sizeof(DeviceState), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        u32 rootLeaves = 1;
        std::memcpy(&rootLeaves, host + kCtlBytes, sizeof(u32));
        if (hc.error) throw std::runtime_error("adaptive_octree: a device scan gave up waiting (bounded look-back)");
        if (hc.overflow)
        {
            cap *= 2;
            continue;
        }
        if (hc.late) return false;
        if (hc.levelCount[levels] != 0)
        {
            m.lvLevels = int(kOctLevels);  // deeper than the last build: all levels again
            continue;
        }
        int deepest = -1;  // deepest level holding units
        for (int l = 0; l < levels; ++l)
            if (hc.levelCount[l]) deepest = l;
        if (deepest < 0) rootLeaves = 1;
        // leaves after every round that changed the tree
        const auto *contrib = reinterpret_cast<const unsigned long long *>(host + kHeadBytes);
        const auto *landed = contrib + lb::kContribBins;
        int rounds = 0;
        for (int ai = 0; ai < lb::kArrivals; ++ai)
            for (int k = 1; k < lb::kJumps; ++k)
                for (int j = 1; j <= k; ++j)
                    if (contrib[(ai * lb::kJumps + k) * lb::kJumps + j]) rounds = std::max(rounds, ai + 1 + (k - j));
        if (rounds > int(cfg_.maxDepth)) return false;  // the rounds stop before converging
        proposals.assign(size_t(rounds), 0);
        for (int t = 1; t <= rounds; ++t)
        {
            unsigned long long leavesAt = landed[t];
            for (int ai = 0; ai + 1 <= t && ai < lb::kArrivals; ++ai)
                for (int k = 1; k < lb::kJumps; ++k)
                    for (int j = 1; j <= k; ++j)
                    {
                        const unsigned long long c = contrib[(ai * lb::kJumps + k) * lb::kJumps + j];
                        if (!c) continue;
                        const int e = k - (t - ai - 1) - j;
                        leavesAt += c << (3 * std::max(e, 0));
                    }
            proposals[size_t(t - 1)] = (long long)leavesAt;
        }
        if (rounds && proposals.back() != (long long)rootLeaves)
            throw std::logic_error("adaptive_octree: level build history does not end at the tree");
        if (hc.placeOverflow)
        {
            ensurePhysical(rootLeaves);
            AOT_CHECK(cudaMemsetAsync(&a.ctl->placeOverflow, 0, sizeof(int), s));
            place();
        }
        hostLeaves_ = rootLeaves;
        m.lvLevels = std::min(int(kOctLevels), deepest + 2);
        lb::finishKernel<<<1, 1, 0, s>>>(a, m.bufs(), rounds, levels, u32(physCap_)), noteLaunch();
        AOT_LAUNCH_CHECK();
        // the host mirror of what finishKernel writes (the readback above
        // brought the active count), so the build needs no second readback
        DeviceState &h = *m.hst;
        h.numLeaves = h.newNumLeaves = int(rootLeaves);
        h.proposal = (long long)rootLeaves;
        h.iteration = rounds;
        h.rounds = rounds + 1;
        h.changed = h.converged = h.needsResize = 0;
        h.numNodes = 0;
        h.activeBuffer = 0;
        h.overflow = 0;
        h.dirtyCount = 0;
        if (nf) AOT_CHECK(cudaMemsetAsync(m.G[0].p, 0, m.G[0].bytes, s));  // no group of the converged tree may merge
        return true;
    }
}

void TreeEngine::binaryBuild()
{
    cudaStream_t s = cfg_.stream;
    waitStream(s);
    built_ = false;
    hostLeaves_ = 1;
    prepareGraphBuffers(std::max<size_t>(2, leafCapacity_));
    sortParticles();
    const size_t estimate = std::max<size_t>(4096, 4 * (n_ / std::max(1u, cfg_.bucket)) + 4096);
    ensurePhysical(std::max({physCap_, estimate, leafCapacity_}));
    lastBuildByLevels_ = buildMode_ == 0 && binaryLevelBuild();
    if (lastBuildByLevels_)
    {
        built_ = true;
        if (prepared_.treeStructure | prepared_.particleCountsPerBox | prepared_.particleMapping)
            prepareViews(leafCapacity_, prepared_);
        buildViews(cfg_.views);  // the placement wrote the counts
        const bool views = cfg_.views.treeStructure | cfg_.views.particleCountsPerBox | cfg_.views.particleMapping;
        if (views) readState();
        else applyState();  // the finish kernel's state, known on the host
        return;
    }
    rb::TreeBufs tb = m_->bufs();
    binInitRootKernel<<<1, 1, 0, s>>>(tb, (long long)leafCapacity_), noteLaunch();
    AOT_LAUNCH_CHECK();
    refreshAll();
    // build loop (kdtree3d.cu:239-249): passes until converged
    long long passes = 0;
    for (;;)
    {
        const int batch = 8;
        for (int r = 0; r < batch; ++r) binaryPass(true, (long long)physCap_);
        passes += batch;
        AOT_CHECK(cudaMemcpyAsync(m_->hst, m_->st, sizeof(DeviceState), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        const DeviceState h = *m_->hst;
        if (h.error) throw std::runtime_error("adaptive_octree: a device scan gave up waiting (bounded look-back)");
        if (h.converged) break;
        if (h.overflow)
        {
            const size_t need = size_t(h.proposal);
            ensurePhysical(std::max(need + need / 4, 2 * physCap_));
            clearOverflowKernel<<<1, 1, 0, s>>>(m_->st), noteLaunch();
            AOT_LAUNCH_CHECK();
        }
        if (passes > 200000) throw std::runtime_error("adaptive_octree: binary build did not converge");
    }
    buildRounds_ = m_->hst->iteration;
    leafCapacity_ = size_t(m_->hst->logicalCap);
    ensurePhysical(leafCapacity_);
    built_ = true;
    if (prepared_.treeStructure | prepared_.particleCountsPerBox | prepared_.particleMapping)
        prepareViews(leafCapacity_, prepared_);
    materializeCounts();
    buildViews(cfg_.views);
    readState();
}

// The converged binary tree, level by level (binlevel.cuh): the tree the
// reference's build passes end with, its pass count and its leaf capacity.
// False where the passes must run: a depth limit beyond the 63 key bits.
bool TreeEngine::binaryLevelBuild()
{
    if (cfg_.maxDepth > 63) return false;
    cudaStream_t s = cfg_.stream;
    Impl &m = *m_;
    const unsigned blocks = unsigned(smCount()) * 4u;
    const KeyIndex idx = m.keyIndex(n_);
    const u64 *P = m.P[0].as<u64>();
    size_t cap = std::max<size_t>(m.blCap, 2 * (n_ / std::max(1u, cfg_.bucket)) + 4096);
    // pinned readback: the control block, then the root's subtree leaf count
    constexpr size_t kLeavesAt = (sizeof(bl::Control) + 15) & ~size_t(15);
    if (!m.blHost) m.blHost = static_cast<bl::Control *>(blockcache::takeHost(kLeavesAt + 16, &m.blHostBytes));
    const bl::Control &hc = *m.blHost;
    for (;;)
    {
        if (cap >= (size_t(1) << 31)) return false;
        m.blRows.reserve(cap * sizeof(uint4), s);
        m.blMid.reserve(cap * sizeof(u32), s);
        m.blChild.reserve(cap * 2 * sizeof(u32), s);
        m.blLeaves.reserve(cap * sizeof(u32), s);
        m.blOffset.reserve(cap * sizeof(u32), s);
        m.blCtl.reserve(sizeof(bl::Control), s);
        m.blCap = cap;
        bl::Arena a{};
        a.rows = m.blRows.as<uint4>();
        a.mid = m.blMid.as<u32>();
        a.child = m.blChild.as<u32>();
        a.leaves = m.blLeaves.as<u32>();
        a.offset = m.blOffset.as<u32>();
        a.ctl = m.blCtl.as<bl::Control>();
        a.cap = u32(cap);
        AOT_CHECK(cudaMemsetAsync(m.blCtl.p, 0, sizeof(bl::Control), s));
        bl::rootKernel<<<1, 32, 0, s>>>(a, m.bufs(), P, n_, cfg_.bucket, cfg_.maxDepth), noteLaunch();
        // as many depths as the last build needed (all 64 the first time);
        // the readback tells whether the tree went deeper
        const int levels = std::max(1, std::min(bl::kLevels, m.blLevels));
        for (int l = 0; l < levels; ++l)
            bl::levelKernel<<<blocks * 2, bl::kThreads, 0, s>>>(a, idx, l, cfg_.bucket, cfg_.maxDepth), noteLaunch();
        for (int l = levels - 1; l >= 0; --l)
            bl::leafCountKernel<<<blocks, bl::kThreads, 0, s>>>(a, l, levels), noteLaunch();
        auto place = [&]() {
            const rb::TreeBufs tb = m.bufs();
            for (int l = 0; l < levels; ++l)
                bl::placeKernel<<<blocks, bl::kThreads, 0, s>>>(a, tb.K[0], tb.B[0], tb.N[0], l, levels,
                                                               u32(physCap_)),
                    noteLaunch();
            AOT_LAUNCH_CHECK();
        };
        place();
        AOT_CHECK(cudaMemcpyAsync(m.blHost, m.blCtl.p, sizeof(bl::Control), cudaMemcpyDeviceToHost, s));
        unsigned char *leavesHost = reinterpret_cast<unsigned char *>(m.blHost) + kLeavesAt;
        AOT_CHECK(cudaMemcpyAsync(leavesHost, a.leaves, sizeof(u32), cudaMemcpyDeviceToHost, s));
        AOT_CHECK(cudaMemcpyAsync(m.hst, m.st, sizeof(DeviceState), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        u32 rootLeaves = 1;
        if (m.hst->error) throw std::runtime_error("adaptive_octree: a device scan gave up waiting (bounded look-back)");
        if (hc.overflow)
        {
            cap *= 2;
            continue;
        }
        if (hc.levelCount[levels] != 0)
        {
            m.blLevels = bl::kLevels;  // deeper than the last build: all depths again
            continue;
        }
        int deepest = -1;  // deepest depth holding units
        for (int l = 0; l < levels; ++l)
            if (hc.levelCount[l]) deepest = l;
        if (deepest >= 0) std::memcpy(&rootLeaves, leavesHost, sizeof(u32));
        if (hc.placeOverflow)
        {
            ensurePhysical(rootLeaves);
            AOT_CHECK(cudaMemsetAsync(&a.ctl->placeOverflow, 0, sizeof(int), s));
            place();
        }
        // one pass per depth of units; the capacity's 25 % steps end at the
        // first step at or above the final leaf count (the counts only grow)
        const int passes = deepest + 1;
        long long c = std::max<long long>((long long)leafCapacity_, 1);
        while ((long long)rootLeaves > c) c += (c + 3) / 4;
        m.blLevels = std::min(bl::kLevels, deepest + 2);
        bl::finishKernel<<<1, 1, 0, s>>>(a, m.bufs(), int(rootLeaves), passes, c), noteLaunch();
        AOT_LAUNCH_CHECK();
        // the host mirror of the finished state
        DeviceState &h = *m.hst;
        h.numLeaves = h.newNumLeaves = int(rootLeaves);
        h.numNodes = (int(rootLeaves) - 1) * 2 + 1;
        h.proposal = (long long)rootLeaves;
        h.iteration = passes;
        h.rounds = passes + 1;
        h.converged = 1;
        h.changed = h.needsResize = 0;
        h.activeBuffer = 0;
        h.overflow = 0;
        h.dirtyCount = 0;
        h.logicalCap = c;
        buildRounds_ = passes;
        hostLeaves_ = rootLeaves;
        leafCapacity_ = size_t(c);
        ensurePhysical(leafCapacity_);
        return true;
    }
}

void TreeEngine::update()
{
    if (!built_) throw std::logic_error("adaptive_octree: call build() before update()");
    mark(MarkStart, 2);
    sortParticles();
    mark(MarkSorted);
    refreshAll();
    mark(MarkRefreshed);
    for (unsigned i = 0; i < cfg_.iterations; ++i)
    {
        if (cfg_.kind == 0) octreePass(false, (long long)leafCapacity_);
        else binaryPass(false, (long long)leafCapacity_);
    }
    mark(MarkPassed);
    materializeCounts();
    buildViews(cfg_.views);
    mark(MarkEnd);
}

// --------------------------------------------------------------------------
// stage timing
// --------------------------------------------------------------------------
static const char *const kMarkNames[] = {"keys + sort", "refresh", "passes", "counts + views"};

void TreeEngine::setProfiling(bool on)
{
    if (on)
        for (cudaEvent_t &e : m_->marks)
            if (!e) AOT_CHECK(cudaEventCreate(&e));
    profiling_ = on;
    marksRecorded_ = false;
}

// Records stage mark m on the tree's stream and moves the NVTX range on
// (call: 1 build, 2 update, given with MarkStart).  Nothing is recorded while
// the stream is captured: the events would become graph nodes and time the
// capture, not the work.
void TreeEngine::mark(Mark m, int call)
{
    if (!profiling_) return;
    if (m == MarkStart)
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        AOT_CHECK(cudaStreamIsCapturing(cfg_.stream, &cs));
        marking_ = cs == cudaStreamCaptureStatusNone;
        marksRecorded_ = false;
        markCall_ = call;
        nfMarks_ = 0;
        if (!marking_) return;
        nvtxRangePushA(call == 1 ? "build" : "update");
        nvtxRangePushA(kMarkNames[0]);
    }
    if (!marking_) return;
    AOT_CHECK(cudaEventRecord(m_->marks[m], cfg_.stream));
    if (m == MarkSorted && markCall_ == 1)
        AOT_CHECK(cudaEventRecord(m_->marks[MarkRefreshed], cfg_.stream));  // a build has no full refresh
    if (m != MarkStart)
    {
        nvtxRangePop();
        if (m != MarkEnd) nvtxRangePushA(kMarkNames[m]);
    }
    if (m == MarkEnd)
    {
        nvtxRangePop();
        marking_ = false;
        marksRecorded_ = true;
    }
}

// Events around one near-field launch.
void TreeEngine::markNearField(bool begin)
{
    if (!marking_) return;
    std::vector<cudaEvent_t> &ev = m_->nfMarks;
    const size_t k = size_t(nfMarks_) * 2 + (begin ? 0 : 1);
    if (k >= ev.size())
    {
        cudaEvent_t e;
        AOT_CHECK(cudaEventCreate(&e));
        ev.push_back(e);
    }
    AOT_CHECK(cudaEventRecord(ev[k], cfg_.stream));
    if (begin) nvtxRangePushA("near field");
    else
    {
        nvtxRangePop();
        ++nfMarks_;
    }
}

TreeEngine::StageTimes TreeEngine::stageTimes()
{
    StageTimes t;
    if (!marksRecorded_) return t;
    AOT_CHECK(cudaEventSynchronize(m_->marks[MarkEnd]));
    auto ms = [&](cudaEvent_t a, cudaEvent_t b) {
        float v = 0;
        AOT_CHECK(cudaEventElapsedTime(&v, a, b));
        return double(v);
    };
    const cudaEvent_t *e = m_->marks;
    t.keysAndSortMs = ms(e[MarkStart], e[MarkSorted]);
    t.refreshMs = ms(e[MarkSorted], e[MarkRefreshed]);
    t.passesMs = ms(e[MarkRefreshed], e[MarkPassed]);
    t.finishMs = ms(e[MarkPassed], e[MarkEnd]);
    t.totalMs = ms(e[MarkStart], e[MarkEnd]);
    for (int k = 0; k < nfMarks_; ++k)
    {
        const double v = ms(m_->nfMarks[2 * k], m_->nfMarks[2 * k + 1]);
        t.nearFieldMs += v;
        if (k == 0) t.nearFieldFirstMs = v;
    }
    t.nearFieldLaunches = nfMarks_;
    t.call = markCall_;
    t.valid = true;
    return t;
}

// update() runs a fixed number of passes (octree.cu:471-481,
// kdtree3d.cu:259-270), so fast-moving particles can leave overfull or
// mergeable leaves behind.  This variant keeps passing until a pass finds
// nothing to change: passes are launched in groups of cfg.iterations and the
// device state is read between groups.  A pass launched after convergence
// returns at once in every kernel (halted state), so a group may overshoot at
// no cost.  The passes themselves are update()'s, so the result equals
// update() with iterations = maxPasses.
void TreeEngine::updateUntilConverged(unsigned maxPasses, unsigned *changedPasses)
{
    if (!built_) throw std::logic_error("adaptive_octree: call build() before update()");
    if (maxPasses == 0) throw std::invalid_argument("adaptive_octree: updateUntilConverged needs maxPasses >= 1");
    cudaStream_t s = cfg_.stream;
    mark(MarkStart, 2);
    sortParticles();
    mark(MarkSorted);
    refreshAll();
    mark(MarkRefreshed);
    const unsigned group = std::max(1u, cfg_.iterations);
    unsigned launched = 0;
    while (launched < maxPasses)
    {
        const unsigned k = std::min(group, maxPasses - launched);
        for (unsigned i = 0; i < k; ++i)
        {
            if (cfg_.kind == 0) octreePass(false, (long long)leafCapacity_);
            else binaryPass(false, (long long)leafCapacity_);
        }
        launched += k;
        if (launched == maxPasses) break;
        // the raw state only: host-side sizes and the capacity model follow
        // the reference's readbacks, which happen in doBuffersNeedResize()
        AOT_CHECK(cudaMemcpyAsync(m_->hst, m_->st, sizeof(DeviceState), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        if (m_->hst->error) throw std::runtime_error("adaptive_octree: a device scan gave up waiting (bounded look-back)");
        if (m_->hst->converged) break;
    }
    mark(MarkPassed);
    materializeCounts();
    buildViews(cfg_.views);
    mark(MarkEnd);
    if (changedPasses)
    {
        AOT_CHECK(cudaMemcpyAsync(m_->hst, m_->st, sizeof(DeviceState), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        if (m_->hst->error) throw std::runtime_error("adaptive_octree: a device scan gave up waiting (bounded look-back)");
        *changedPasses = unsigned(m_->hst->updatePasses);
    }
}

void TreeEngine::computeViews(const adaptive_octree::ViewConfig &v)
{
    if (!built_) throw std::logic_error("adaptive_octree: call build() before computeViews()");
    buildViews(v);
}

// --------------------------------------------------------------------------
// views (tree_view.cu:755-1134)
// --------------------------------------------------------------------------
void TreeEngine::prepareViews(size_t capacity, const adaptive_octree::ViewConfig &v)
{
    if (!(v.treeStructure | v.particleCountsPerBox | v.particleMapping)) return;
    Impl &m = *m_;
    cudaStream_t s = cfg_.stream;
    m.viewLeafCap = std::max(m.viewLeafCap, capacity);
    m.viewParticleCap = std::max(m.viewParticleCap, n_);
    m.viewPrepared.treeStructure |= v.treeStructure;
    m.viewPrepared.particleCountsPerBox |= v.particleCountsPerBox;
    m.viewPrepared.particleMapping |= v.particleMapping;
    m.viewScratch = true;
    const int b = cfg_.kind == 0 ? 3 : 1;
    const size_t L = std::max<size_t>(m.viewLeafCap, 1);
    const size_t I = (L - 1) / ((size_t(1) << b) - 1);
    const size_t nodes = L + I;
    m.vBox.grow(nodes * 8, m.vBox.bytes, s);
    m.vSplit.grow(nodes, m.vSplit.bytes, s);
    m.vDepth.grow(nodes, m.vDepth.bytes, s);
    m.vParent.grow(nodes * 4, m.vParent.bytes, s);
    m.vChild.grow(nodes * 4, m.vChild.bytes, s);
    m.vLevelOffset.grow(66 * 4, m.vLevelOffset.bytes, s);
    m.vMaxDepth.grow(16, m.vMaxDepth.bytes, s);
    if (m.viewPrepared.particleCountsPerBox)
    {
        m.vPbegin.grow(nodes * 4, m.vPbegin.bytes, s);
        m.vPcount.grow((nodes + 1) * 4, m.vPcount.bytes, s);
    }
    if (m.viewPrepared.particleMapping) m.vPmap.grow(std::max<size_t>(m.viewParticleCap, 1) * 8, m.vPmap.bytes, s);
    m.vLeafLevel.reserve(L, s);
    m.vLeafToNode.reserve(L * 4, s);
    m.vLevels.reserve(4 * 66 * 4, s);
    m.vCandStart.reserve(L * 8, s);
    m.vCandLevel.reserve(L, s);
    for (int k = 0; k < 2; ++k)
    {
        m.vLvKeys[k].reserve(L * 8, s);
        m.vLvVals[k].reserve(L * 4, s);
        m.vLayKeys[k].reserve(std::max<size_t>(I, 1) * 8, s);
        m.vLayVals[k].reserve(std::max<size_t>(I, 1) * 4, s);
    }
    m.vIntStartSfc.reserve(std::max<size_t>(I, 1) * 8, s);
    m.vIntLevelSfc.reserve(std::max<size_t>(I, 1), s);
    m.vIntM.reserve(std::max<size_t>(I, 1) * 4, s);
    m.vIntStartLay.reserve(std::max<size_t>(I, 1) * 8, s);
    m.vIntLevelLay.reserve(std::max<size_t>(I, 1), s);
    m.viewSort.ensure(L, sort::kDefaultSortConfig, s);
}

void TreeEngine::syncViewSizes()
{
    Impl &m = *m_;
    if (!m.viewScratch || hostLeaves_ > m.viewLeafCap) return;
    const size_t k = cfg_.kind == 0 ? 7 : 1;
    m.viewNodesLogical = hostLeaves_ + (hostLeaves_ - 1) / k;
    if (m.viewPrepared.particleMapping) m.mappingLogical = hostActive_;
}

void TreeEngine::buildViews(const adaptive_octree::ViewConfig &v)
{
    prepared_.treeStructure |= v.treeStructure;
    prepared_.particleCountsPerBox |= v.particleCountsPerBox;
    prepared_.particleMapping |= v.particleMapping;
    if (!(v.treeStructure | v.particleCountsPerBox | v.particleMapping)) return;
    Impl &m = *m_;
    cudaStream_t s = cfg_.stream;
    if (!m.viewScratch || (v.particleCountsPerBox && !m.viewPrepared.particleCountsPerBox) ||
        (v.particleMapping && (!m.viewPrepared.particleMapping || n_ > m.viewParticleCap)))
    {
        tv::flagResizeKernel<<<1, 1, 0, s>>>(m.st), noteLaunch();
        AOT_LAUNCH_CHECK();
        return;
    }
    const int b = cfg_.kind == 0 ? 3 : 1;
    const int leafCap = int(m.viewLeafCap);
    const int intCap = (leafCap - 1) / ((1 << b) - 1);
    const tv::ViewBufs vb = m.viewBufs();
    const u64 *K0 = m.K[0].as<u64>(), *K1 = m.K[1].as<u64>();
    const u32 *B0 = m.B[0].as<u32>(), *B1 = m.B[1].as<u32>();
    const KeyIndex idx = m.keyIndex(n_);
    const int counts = v.particleCountsPerBox ? 1 : 0;
    AOT_CHECK(cudaMemsetAsync(vb.leavesPerLevel, 0, 66 * sizeof(int), s));
    if (b == 3)
    {
        tv::classifyKernel<3><<<gridFor(leafCap, tv::kThreads), tv::kThreads, 0, s>>>(K0, K1, m.st, leafCap, vb), noteLaunch();
        tv::metadataKernel<3><<<1, 1, 0, s>>>(m.st, leafCap, vb), noteLaunch();
    }
    else
    {
        tv::classifyKernel<1><<<gridFor(leafCap, tv::kThreads), tv::kThreads, 0, s>>>(K0, K1, m.st, leafCap, vb), noteLaunch();
        tv::metadataKernel<1><<<1, 1, 0, s>>>(m.st, leafCap, vb), noteLaunch();
    }
    AOT_LAUNCH_CHECK();
    if (intCap > 0)
    {
        // stable order of internal nodes by level (non-internal boundaries last)
        u64 *lk[2] = {vb.lvKeys, vb.lvKeysAlt};
        u32 *lv[2] = {vb.lvVals, vb.lvValsAlt};
        const int w1 = sortWithIndices(s, lk, lv, size_t(leafCap - 1), 1, m.viewSort, &m.st->error);
        if (b == 3)
            tv::layoutKeysKernel<3><<<gridFor(intCap, tv::kThreads), tv::kThreads, 0, s>>>(lk[w1], lv[w1], intCap, vb), noteLaunch();
        else
            tv::layoutKeysKernel<1><<<gridFor(intCap, tv::kThreads), tv::kThreads, 0, s>>>(lk[w1], lv[w1], intCap, vb), noteLaunch();
        AOT_LAUNCH_CHECK();
        u64 *yk[2] = {vb.layKeys, vb.layKeysAlt};
        u32 *yv[2] = {vb.layVals, vb.layValsAlt};
        const int w2 = sortWithIndices(s, yk, yv, size_t(intCap), 8, m.viewSort, &m.st->error);
        tv::materializeKernel<<<gridFor(intCap, tv::kThreads), tv::kThreads, 0, s>>>(yk[w2], yv[w2], intCap, vb), noteLaunch();
        if (b == 3)
            tv::internalNodesKernel<3><<<gridFor(intCap, tv::kThreads), tv::kThreads, 0, s>>>(m.st, leafCap, intCap,
                                                                                              idx, counts, vb), noteLaunch();
        else
            tv::internalNodesKernel<1><<<gridFor(intCap, tv::kThreads), tv::kThreads, 0, s>>>(m.st, leafCap, intCap,
                                                                                              idx, counts, vb), noteLaunch();
        AOT_LAUNCH_CHECK();
    }
    if (b == 3)
        tv::leafNodesKernel<3><<<gridFor(leafCap, tv::kThreads), tv::kThreads, 0, s>>>(K0, K1, B0, B1, m.st, leafCap,
                                                                                      counts, vb), noteLaunch();
    else
        tv::leafNodesKernel<1><<<gridFor(leafCap, tv::kThreads), tv::kThreads, 0, s>>>(K0, K1, B0, B1, m.st, leafCap,
                                                                                      counts, vb), noteLaunch();
    AOT_LAUNCH_CHECK();
    if (v.particleMapping && n_ > 0)
    {
        tv::mappingKernel<<<gridFor(n_, tv::kThreads), tv::kThreads, 0, s>>>(B0, B1, m.st, leafCap, n_, vb), noteLaunch();
        AOT_LAUNCH_CHECK();
    }
}

// --------------------------------------------------------------------------
// getters
// --------------------------------------------------------------------------
void TreeEngine::buffer(int which, const void **ptr, size_t *len, size_t *cap, size_t *elem) const
{
    const Impl &m = *m_;
    const int a = hostActiveBuffer_;
    const size_t nodes = m.viewScratch ? m.viewNodesLogical : 0;
    const size_t nodeCap = m.viewScratch ? m.vBox.bytes / 8 : 0;
    const void *p = nullptr;
    size_t l = 0, c = 0, e = 1;
    switch (which)
    {
    case ParticleKeys: p = m.P[0].p; l = c = n_; e = 8; break;
    case Perm: p = m.Perm[0].p; l = c = n_; e = 4; break;
    case Cornerstone: p = m.K[a].p; l = hostLeaves_ + 1; c = physCap_ + 1; e = 8; break;
    case LeafCounts: p = m.N[a].p; l = hostLeaves_; c = physCap_; e = 4; break;
    case NearFieldCounts:
        if (cfg_.kind == 1) throw std::logic_error("Tree: Binary NFCount is not implemented yet");
        p = m.NF[a].p; l = hostLeaves_; c = physCap_; e = 4; break;
    case SfcBoxIndex: p = m.vBox.p; l = nodes; c = nodeCap; e = 8; break;
    case HasBoxSplit: p = m.vSplit.p; l = nodes; c = nodeCap; e = 1; break;
    case BoxDepth: p = m.vDepth.p; l = nodes; c = nodeCap; e = 1; break;
    case ParentIndex: p = m.vParent.p; l = nodes; c = nodeCap; e = 4; break;
    case ChildIndex: p = m.vChild.p; l = nodes; c = nodeCap; e = 4; break;
    case LevelOffset:
        p = m.vLevelOffset.p;
        l = c = m.viewScratch ? (cfg_.kind == 0 ? 23 : 65) : 0;
        e = 4;
        break;
    case ParticleBeginIndex:
        p = m.vPbegin.p;
        l = (m.viewScratch && m.viewPrepared.particleCountsPerBox) ? nodes : 0;
        c = m.vPbegin.bytes / 4;
        e = 4;
        break;
    case ParticleCounts:
        p = m.vPcount.p;
        l = (m.viewScratch && m.viewPrepared.particleCountsPerBox) ? nodes + 1 : 0;
        c = m.vPcount.bytes / 4;
        e = 4;
        break;
    case LeafBegins: p = m.B[a].p; l = hostLeaves_ + 1; c = physCap_ + 1; e = 4; break;
    case SfcParticleIndex:
        p = m.vPmap.p;
        l = (m.viewScratch && m.viewPrepared.particleMapping) ? m.mappingLogical : 0;
        c = m.vPmap.bytes / 8;
        e = 8;
        break;
    default: throw std::invalid_argument("adaptive_octree: unknown buffer");
    }
    if (ptr) *ptr = p;
    if (len) *len = l;
    if (cap) *cap = c;
    if (elem) *elem = e;
}

const int *TreeEngine::numLeavesDevice() const { return &m_->st->numLeaves; }
const int *TreeEngine::numNodesDevice() const { return &m_->st->numNodes; }
const unsigned *TreeEngine::numActiveParticlesDevice() const { return &m_->st->numActiveParticles; }

unsigned TreeEngine::maxAchievedDepth() const
{
    const Impl &m = *m_;
    cudaStream_t s = cfg_.stream;
    if (cfg_.kind == 1 && !(cfg_.views.treeStructure | cfg_.views.particleCountsPerBox | cfg_.views.particleMapping))
    {
        // kdtree3d.cu: maxAchievedDepth from the cornerstone when no view is configured
        std::vector<u64> k(hostLeaves_ + 1);
        AOT_CHECK(cudaMemcpyAsync(k.data(), m.K[hostActiveBuffer_].p, k.size() * 8, cudaMemcpyDeviceToHost, s));
        waitStream(s);
        unsigned d = 0;
        for (size_t i = 0; i + 1 < k.size(); ++i) d = std::max(d, unsigned(clz64(k[i + 1] - k[i])));
        return d;
    }
    if (!m.viewScratch) return 0;
    u8 v = 0;
    AOT_CHECK(cudaMemcpyAsync(&v, m.vMaxDepth.p, 1, cudaMemcpyDeviceToHost, s));
    waitStream(s);
    return v;
}

}  // namespace aot
