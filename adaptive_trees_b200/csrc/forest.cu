// forest.cu -- host orchestration of the forest engine (forest.hpp).
//
// build():  keys + segmented sort of all systems, the roots, then build
//           rounds over all systems until none changes (at most maxDepth,
//           as rebalanceBuild, octree.cu:159-180), one state readback per
//           round; each system's leafCapacity is replayed from its own round
//           history with the same capacity model as a single tree.
// update(): keys + segmented sort, a full begin-index refresh, then the
//           configured number of fixed passes with per-system capacity
//           rejection (updateOctreeGraphGpu, octree_rebalance.cuh:1177-1322);
//           no host synchronisation.
#include "forest.hpp"

#include <algorithm>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>

#include "capacity.hpp"
#include "engine_util.cuh"
#include "forest.cuh"
#include "forest_levels.cuh"
#include "forest_sort.cuh"

namespace aot
{
struct ForestEngine::Impl
{
    EngineConfig cfg;
    int S = 0;
    size_t total = 0;
    std::vector<forest::System> systems;
    // segmented sort: tiles of the sort configuration `tileConfig`
    u32 numTiles = 0;
    int tileConfig = -1;
    cudaEvent_t tuneStart = nullptr, tuneEnd = nullptr;  // sort tuner timing
    DevMem systemsD, tileSys, tileBegin, tileEnd, segFirstTile, segBase;
    DevMem P[2], Perm[2], hist, bins, tileCounters, status;
    // leaf arrays (entries = all systems' leaves + sentinels)
    size_t entryCap = 0;
    DevMem K[2], B[2], SEG[2], N, ops, offs, dirty, scanStatus, scanTile;
    size_t scanTiles = 0;
    // state
    DevMem st, sys, history, frozen;
    forest::State *hst = nullptr;       // pinned mirrors (block cache)
    forest::SysState *hsys = nullptr;
    size_t hstBytes = 0, hsysBytes = 0;
    std::vector<OctreeCapacity> capModel;
    std::vector<size_t> leafCap;
    bool built = false;
    // build by levels: the unit arena, the key sample and the control words
    DevMem lvRows, lvChild, lvLeaves, lvOffset, lvUsys, lvSysRoot, lvBins, lvCtl, sample, sortBar;
    size_t lvCap = 0;
    size_t lastEntries = 0;  // entries of the last build (the first guess of the next)
    int buildMode = 0;
    bool lastByLevels = false;
    KeygenParams<float> kpf{};
    KeygenParams<double> kpd{};

    ~Impl()
    {
        if (hst) blockcache::giveHost(hst, hstBytes);
        if (hsys) blockcache::giveHost(hsys, hsysBytes);
        if (tuneStart) cudaEventDestroy(tuneStart);
        if (tuneEnd) cudaEventDestroy(tuneEnd);
    }

    // Tile table of the segmented sort for configuration `config`: every
    // system in tiles of that configuration's size (a host build and upload,
    // done when the configuration changes).
    void buildTiles(int config, cudaStream_t stream)
    {
        if (config == tileConfig) return;
        const u32 tile = u32(sort::configTile(config));
        std::vector<u32> tSys, tBeg, tEnd;
        std::vector<u32> first(static_cast<size_t>(S), 0xffffffffu);
        std::vector<u32> base(static_cast<size_t>(S), 0u);
        for (int s = 0; s < S; ++s)
        {
            const forest::System &sy = systems[s];
            base[s] = sy.base;
            if (sy.n) first[s] = u32(tSys.size());
            for (u32 b = 0; b < sy.n; b += tile)
            {
                tSys.push_back(u32(s));
                tBeg.push_back(sy.base + b);
                tEnd.push_back(sy.base + std::min<u32>(sy.n, b + tile));
            }
        }
        waitStream(stream);  // the old tables may still be read
        numTiles = u32(tSys.size());
        auto upload = [](DevMem &d, const void *src, size_t bytes) {
            d.reserve(std::max<size_t>(bytes, 16));
            if (bytes) AOT_CHECK(cudaMemcpy(d.p, src, bytes, cudaMemcpyHostToDevice));
        };
        upload(tileSys, tSys.data(), tSys.size() * 4);
        upload(tileBegin, tBeg.data(), tBeg.size() * 4);
        upload(tileEnd, tEnd.data(), tEnd.size() * 4);
        upload(segFirstTile, first.data(), first.size() * 4);
        upload(segBase, base.data(), base.size() * 4);
        status.release();
        status.reserve(std::max<size_t>(numTiles, 1) * sort::configPasses(config) * sort::kRadix * 8);
        tileConfig = config;
    }

    forest::Bufs bufs() const
    {
        forest::Bufs f{};
        for (int k = 0; k < 2; ++k)
        {
            f.K[k] = K[k].as<u64>();
            f.B[k] = B[k].as<u32>();
            f.SEG[k] = SEG[k].as<int>();
        }
        f.N = N.as<u32>();
        f.ops = ops.as<int>();
        f.offs = offs.as<i64>();
        f.dirty = dirty.as<int>();
        f.scanStatus = scanStatus.as<u64>();
        f.scanTile = scanTile.as<u32>();
        f.st = st.as<forest::State>();
        f.sys = sys.as<forest::SysState>();
        f.systems = systemsD.as<forest::System>();
        f.numSystems = S;
        f.history = history.as<long long>();
        f.P = P[0].as<u64>();
        return f;
    }
};

ForestEngine::ForestEngine(const void *const *x, const void *const *y, const void *const *z, const size_t *n,
                           int numSystems, const EngineConfig &cfg)
    : m_(std::make_unique<Impl>())
{
    Impl &m = *m_;
    if (numSystems <= 0) throw std::invalid_argument("forest: need at least one system");
    if (!x || !y || !z || !n) throw std::invalid_argument("forest: null coordinate or count array");
    if (cfg.kind != 0) throw std::invalid_argument("forest: only octrees are batched");
    if (cfg.nf) throw std::invalid_argument("forest: only LeafCount refinement is batched");
    if (cfg.bucket == 0) throw std::invalid_argument("adaptive_octree: particle limit must be positive");
    if (cfg.iterations == 0) throw std::invalid_argument("adaptive_octree: updateIterations must be positive");
    if (cfg.views.treeStructure | cfg.views.particleCountsPerBox | cfg.views.particleMapping)
        throw std::invalid_argument("forest: tree views are not batched");
    m.cfg = cfg;
    m.S = numSystems;
    m.systems.resize(size_t(numSystems));
    size_t total = 0;
    for (int s = 0; s < numSystems; ++s)
    {
        if (n[s] > 0 && (!x[s] || !y[s] || !z[s]))
            throw std::invalid_argument("adaptive_octree: coordinate device pointers must not be null");
        m.systems[s] = forest::System{x[s], y[s], z[s], u32(total), u32(n[s])};
        total += n[s];
        if (total > size_t(std::numeric_limits<std::uint32_t>::max()))
            throw std::invalid_argument("forest: more than 2^32 - 1 particles in total");
    }
    m.total = total;
    m.kpf.q = makeQuantBox<float>(cfg.box);
    m.kpd.q = makeQuantBox<double>(cfg.box);
    m.kpf.h = m.kpd.h = hilbertTables();
    m.capModel.assign(size_t(numSystems), OctreeCapacity{});
    m.leafCap.assign(size_t(numSystems), 0);

    {
        const size_t bytes = m.systems.size() * sizeof(forest::System);
        m.systemsD.reserve(std::max<size_t>(bytes, 16));
        if (bytes) AOT_CHECK(cudaMemcpy(m.systemsD.p, m.systems.data(), bytes, cudaMemcpyHostToDevice));
    }
    m.buildTiles(sortTuning(true, total).config, cfg.stream);
    for (int k = 0; k < 2; ++k)
    {
        m.P[k].reserve(std::max<size_t>(total, 1) * 8);
        m.Perm[k].reserve(std::max<size_t>(total, 1) * 4);
    }
    m.hist.reserve(size_t(numSystems) * sort::kPassSlots * sort::kRadix * 4);
    m.bins.reserve(size_t(numSystems) * sort::kPassSlots * sort::kRadix * 4);
    m.tileCounters.reserve(sort::kPassSlots * 4);
    m.st.reserve(sizeof(forest::State));
    AOT_CHECK(cudaMemsetAsync(m.st.p, 0, sizeof(forest::State), cfg.stream));
    m.sys.reserve(size_t(numSystems) * sizeof(forest::SysState));
    AOT_CHECK(cudaMemsetAsync(m.sys.p, 0, size_t(numSystems) * sizeof(forest::SysState), cfg.stream));
    m.history.reserve(size_t(std::max(cfg.maxDepth, 1u)) * numSystems * sizeof(long long));
    m.frozen.reserve(size_t(numSystems));
    AOT_CHECK(cudaMemsetAsync(m.frozen.p, 0, size_t(numSystems), cfg.stream));
    waitStream(cfg.stream);
    m.hst = static_cast<forest::State *>(blockcache::takeHost(sizeof(forest::State), &m.hstBytes));
    m.hsys = static_cast<forest::SysState *>(
        blockcache::takeHost(size_t(numSystems) * sizeof(forest::SysState), &m.hsysBytes));
    std::memset(m.hst, 0, sizeof(forest::State));
    std::memset(m.hsys, 0, size_t(numSystems) * sizeof(forest::SysState));
    ensurePhysical(size_t(4) * numSystems + 4096);
}

// The buffers go back to the block cache: no queued work may still use them.
ForestEngine::~ForestEngine()
{
    if (m_) (void)cudaStreamSynchronize(m_->cfg.stream);
}

int ForestEngine::numSystems() const { return m_->S; }
size_t ForestEngine::numParticles() const { return m_->total; }

void ForestEngine::setCoordinates(int s, const void *x, const void *y, const void *z)
{
    Impl &m = *m_;
    if (s < 0 || s >= m.S) throw std::invalid_argument("forest: system index out of range");
    if (m.systems[s].n > 0 && (!x || !y || !z))
        throw std::invalid_argument("adaptive_octree: coordinate device pointers must not be null");
    m.systems[s].x = x;
    m.systems[s].y = y;
    m.systems[s].z = z;
    AOT_CHECK(cudaMemcpyAsync(m.systemsD.as<forest::System>() + s, &m.systems[s], sizeof(forest::System),
                              cudaMemcpyHostToDevice, m.cfg.stream));
    waitStream(m.cfg.stream);
}

// Leaf arrays for `entries` entries; the active arrays keep their contents.
void ForestEngine::ensurePhysical(size_t entries)
{
    Impl &m = *m_;
    if (entries <= m.entryCap && m.K[0].p) return;
    cudaStream_t s = m.cfg.stream;
    const size_t c = std::max(entries, m.entryCap + m.entryCap / 2);
    for (int k = 0; k < 2; ++k)
    {
        m.K[k].grow((c + 1) * 8, m.K[k].bytes, s);
        m.B[k].grow((c + 1) * 4, m.B[k].bytes, s);
        m.SEG[k].grow((c + 1) * 4, m.SEG[k].bytes, s);
    }
    m.N.grow((c + 1) * 4, m.N.bytes, s);
    m.ops.reserve((c + 1) * 4, s);
    m.offs.grow((c + 2) * 8, m.offs.bytes, s);  // a build round grows the arrays between scan and scatter
    m.dirty.reserve((c + 1) * 4, s);
    m.scanTiles = (c + 2 + rb::kScanTile - 1) / rb::kScanTile;
    m.scanStatus.reserve((m.scanTiles + 1) * 8, s);
    m.scanTile.reserve(16, s);
    m.entryCap = c;
}

void ForestEngine::sortParticles(bool withSample)
{
    Impl &m = *m_;
    cudaStream_t s = m.cfg.stream;
    if (m.total)
    {
        cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
        AOT_CHECK(cudaStreamIsCapturing(s, &capture));
        if (capture != cudaStreamCaptureStatusNone)
        {
            sortKeys(m.tileConfig);  // under capture the tables stay as they are
        }
        else if (m.cfg.tuneSort && sortNeedsTuning(true, m.total))
        {
            // every configuration sorts identically: the keys of the last timed
            // run stand, and the tables follow the chosen configuration
            if (!m.tuneStart) AOT_CHECK(cudaEventCreate(&m.tuneStart));
            if (!m.tuneEnd) AOT_CHECK(cudaEventCreate(&m.tuneEnd));
            auto time = [](int c, void *ctx) -> float {
                ForestEngine &e = *static_cast<ForestEngine *>(ctx);
                Impl &im = *e.m_;
                im.buildTiles(c, im.cfg.stream);
                AOT_CHECK(cudaEventRecord(im.tuneStart, im.cfg.stream));
                e.sortKeys(c);
                AOT_CHECK(cudaEventRecord(im.tuneEnd, im.cfg.stream));
                AOT_CHECK(cudaEventSynchronize(im.tuneEnd));
                float ms = 0.f;
                AOT_CHECK(cudaEventElapsedTime(&ms, im.tuneStart, im.tuneEnd));
                return ms;
            };
            const int best = sortTune(true, m.total, time, this);
            m.buildTiles(best, s);
        }
        else
        {
            const int config = sortTuning(true, m.total).config;
            m.buildTiles(config, s);
            if (withSample && sortPersistent(config)) return;  // keys, sort, active counts and sample in one launch
            sortKeys(config);
        }
    }
    const size_t ns = withSample ? (m.total + kSampleStride - 1) >> kSampleShift : 0;
    if (ns) m.sample.reserve(ns * sizeof(u64), s);
    const unsigned grid = std::min<unsigned>(gridFor(std::max(size_t(m.S), ns), 256), unsigned(smCount()) * 8u);
    forest::activeKernel<<<std::max(grid, 1u), 256, 0, s>>>(m.bufs(), ns ? m.sample.as<u64>() : nullptr, ns),
        noteLaunch();
    AOT_LAUNCH_CHECK();
}

// Keys of every system into P[0] (hist: with the 8-bit digit histograms).
void ForestEngine::launchKeygen(bool hist)
{
    Impl &m = *m_;
    cudaStream_t s = m.cfg.stream;
    const unsigned grid = std::max(1u, std::min<unsigned>(m.numTiles, unsigned(smCount()) * 8u));
    u64 *keys = m.P[0].as<u64>();
    u32 *keygenHist = hist ? m.hist.as<u32>() : nullptr;
    const Impl &cm = m;
    auto launch = [&](auto real) {
        using Real = decltype(real);
        const KeygenParams<Real> &prm = [&]() -> const KeygenParams<Real> & {
            if constexpr (sizeof(Real) == 4) return cm.kpf;
            else return cm.kpd;
        }();
        if (m.cfg.hilbert)
            forest::keygenKernel<Real, Curve::Hilbert><<<grid, forest::kThreads, 0, s>>>(
                m.systemsD.as<forest::System>(), m.tileSys.as<u32>(), m.tileBegin.as<u32>(), m.tileEnd.as<u32>(),
                m.numTiles, prm, keys, keygenHist), noteLaunch();
        else
            forest::keygenKernel<Real, Curve::Morton><<<grid, forest::kThreads, 0, s>>>(
                m.systemsD.as<forest::System>(), m.tileSys.as<u32>(), m.tileBegin.as<u32>(), m.tileEnd.as<u32>(),
                m.numTiles, prm, keys, keygenHist), noteLaunch();
    };
    if (m.cfg.real == 0) launch(float{});
    else launch(double{});
    AOT_LAUNCH_CHECK();
}

// Keys (one launch), then the segmented sort, the active counts and the key
// sample of a build by levels in one cooperative launch (forest::sortKernel),
// for the 8-bit sort configurations; false (nothing done) for the others.
bool ForestEngine::sortPersistent(int config)
{
    Impl &m = *m_;
    cudaStream_t s = m.cfg.stream;
    const sort::SortConfig sc = sort::kSortConfigs[config];
    if (sc.bits != sort::kRadixBits || config != m.tileConfig || sort::configPasses(config) != sort::kMaxPasses)
        return false;
    const void *fn = nullptr;
    size_t smem = 0;
    // 3 CTAs per SM: the pass loop stays in registers (at 4 it spills and
    // runs slower)
    switch (sc.items)
    {
    case 8:
        fn = reinterpret_cast<const void *>(&forest::sortKernel<8>);
        smem = sizeof(sort::SharedPass<8, 8>);
        break;
    case 10:
        fn = reinterpret_cast<const void *>(&forest::sortKernel<10>);
        smem = sizeof(sort::SharedPass<8, 10>);
        break;
    case 16:
        fn = reinterpret_cast<const void *>(&forest::sortKernel<16>);
        smem = sizeof(sort::SharedPass<8, 16>);
        break;
    default: return false;
    }
    AOT_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int perSm = 0;
    AOT_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, sort::kThreads, smem));
    if (perSm <= 0) return false;
    const unsigned grid = unsigned(perSm) * unsigned(smCount());
    const int passes = sort::configPasses(config);
    const size_t ns = (m.total + kSampleStride - 1) >> kSampleShift;
    m.sample.reserve(std::max<size_t>(ns, 1) * sizeof(u64), s);
    m.sortBar.reserve(sizeof(GridBarrier), s);
    AOT_CHECK(cudaMemsetAsync(m.hist.p, 0, size_t(m.S) * sort::kPassSlots * sort::kRadix * 4, s));
    AOT_CHECK(cudaMemsetAsync(m.tileCounters.p, 0, sort::kPassSlots * 4, s));
    AOT_CHECK(cudaMemsetAsync(m.status.p, 0, size_t(m.numTiles) * passes * sort::kRadix * 8, s));
    AOT_CHECK(cudaMemsetAsync(m.sortBar.p, 0, sizeof(GridBarrier), s));
    launchKeygen(true);
    forest::SortArgs p{};
    p.f = m.bufs();
    p.tiles = sort::SegmentTiles{m.tileSys.as<u32>(),      m.tileBegin.as<u32>(), m.tileEnd.as<u32>(),
                                 m.segFirstTile.as<u32>(), m.segBase.as<u32>(),  nullptr};
    p.numTiles = m.numTiles;
    for (int k = 0; k < 2; ++k)
    {
        p.keys[k] = m.P[k].as<u64>();
        p.vals[k] = m.Perm[k].as<u32>();
    }
    p.hist = m.hist.as<u32>();
    p.bins = m.bins.as<u32>();
    p.tileCounters = m.tileCounters.as<u32>();
    p.status = m.status.as<u64>();
    p.error = &m.st.as<forest::State>()->error;
    p.sample = m.sample.as<u64>();
    p.ns = ns;
    p.bar = m.sortBar.as<GridBarrier>();
    void *args[] = {&p};
    AOT_CHECK(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(sort::kThreads), args, smem, s));
    noteLaunch();
    AOT_LAUNCH_CHECK();
    return true;
}

// Keys of every system and the segmented sort with sort configuration
// `config`, whose tile table must be in place; the result lands in P[0] /
// Perm[0] (an even pass count).
void ForestEngine::sortKeys(int config)
{
    Impl &m = *m_;
    cudaStream_t s = m.cfg.stream;
    if (config != m.tileConfig) throw std::logic_error("forest: the tile table is not the sort configuration's");
    const int bitsPer = sort::kSortConfigs[config].bits;
    const int passes = sort::configPasses(config);
    if (passes & 1) throw std::logic_error("forest: sort configurations must have an even pass count");
    AOT_CHECK(cudaMemsetAsync(m.hist.p, 0, size_t(m.S) * sort::kPassSlots * sort::kRadix * 4, s));
    AOT_CHECK(cudaMemsetAsync(m.tileCounters.p, 0, sort::kPassSlots * 4, s));
    AOT_CHECK(cudaMemsetAsync(m.status.p, 0, size_t(m.numTiles) * passes * sort::kRadix * 8, s));
    u64 *keys = m.P[0].as<u64>();
    // 8-bit digits: the histograms come with the keys; otherwise a pass of their own
    const bool fused = bitsPer == sort::kRadixBits;
    launchKeygen(fused);
    if (!fused)
        forest::segHistKernel<7><<<m.numTiles, forest::kThreads, 0, s>>>(m.tileSys.as<u32>(), m.tileBegin.as<u32>(),
                                                                      m.tileEnd.as<u32>(), keys, passes,
                                                                      m.hist.as<u32>()),
            noteLaunch();
    forest::binsKernel<<<unsigned(m.S), sort::kRadix, 0, s>>>(m.systemsD.as<forest::System>(), m.S, m.hist.as<u32>(),
                                                              m.bins.as<u32>(), passes),
        noteLaunch();
    AOT_LAUNCH_CHECK();
    sort::setPassSmemAll();
    u64 *k[2] = {m.P[0].as<u64>(), m.P[1].as<u64>()};
    u32 *v[2] = {m.Perm[0].as<u32>(), m.Perm[1].as<u32>()};
    for (int p = 0; p < passes; ++p)
    {
        const int in = p & 1, out = in ^ 1;
        const int shift = p * bitsPer;
        const sort::SegmentTiles tiles{m.tileSys.as<u32>(),      m.tileBegin.as<u32>(), m.tileEnd.as<u32>(),
                                       m.segFirstTile.as<u32>(), m.segBase.as<u32>(),
                                       m.bins.as<u32>() + size_t(p) * m.S * sort::kRadix};
        sort::launchSegmentPass(config, s, m.numTiles, tiles, k[in], p == 0 ? nullptr : v[in], k[out], v[out], shift,
                                m.tileCounters.as<u32>() + p, m.status.as<u64>() + size_t(p) * m.numTiles * sort::kRadix,
                                &m.st.as<forest::State>()->error, std::min(bitsPer, 64 - shift)),
            noteLaunch();
        AOT_LAUNCH_CHECK();
    }
}

// One decision round (build) or fixed pass (update) over all systems.
void ForestEngine::pass(bool build, const unsigned char *frozenDevice)
{
    Impl &m = *m_;
    cudaStream_t s = m.cfg.stream;
    const forest::Bufs f = m.bufs();
    const unsigned sysGrid = gridFor(size_t(m.S), 256);
    const unsigned wide = unsigned(smCount()) * 8u;
    forest::beginPassKernel<<<sysGrid, 256, 0, s>>>(f, frozenDevice), noteLaunch();
    AOT_CHECK(cudaMemsetAsync(m.scanStatus.p, 0, (m.scanTiles + 1) * 8, s));
    forest::decideKernel<<<wide, forest::kThreads, 0, s>>>(f, m.cfg.bucket), noteLaunch();
    if (build) forest::checkKernel<true><<<sysGrid, 256, 0, s>>>(f), noteLaunch();
    else forest::checkKernel<false><<<sysGrid, 256, 0, s>>>(f), noteLaunch();
    forest::scanKernel<<<unsigned(m.scanTiles), rb::kScanThreads, 0, s>>>(f), noteLaunch();
    AOT_LAUNCH_CHECK();
    if (build)
    {
        // the proposal decides the room the scatter needs
        AOT_CHECK(cudaMemcpyAsync(m.hst, m.st.p, sizeof(forest::State), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        if (m.hst->error) throw std::runtime_error("forest: a device scan gave up waiting (bounded look-back)");
        if (!m.hst->changed) return;
        ensurePhysical(size_t(m.hst->proposal));
    }
    const forest::Bufs g = m.bufs();
    forest::scatterKernel<<<wide, forest::kThreads, 0, s>>>(g), noteLaunch();
    if (build) forest::commitKernel<true><<<1, 256, 0, s>>>(g), noteLaunch();
    else forest::commitKernel<false><<<1, 256, 0, s>>>(g), noteLaunch();
    forest::refreshKernel<false><<<wide, forest::kThreads, 0, s>>>(g), noteLaunch();
    AOT_LAUNCH_CHECK();
}

// Host mirrors of the device state; model: also the state readback of each
// system's capacity model (as doBuffersNeedResize of a single tree).
void ForestEngine::readState(bool model)
{
    Impl &m = *m_;
    cudaStream_t s = m.cfg.stream;
    AOT_CHECK(cudaMemcpyAsync(m.hst, m.st.p, sizeof(forest::State), cudaMemcpyDeviceToHost, s));
    AOT_CHECK(cudaMemcpyAsync(m.hsys, m.sys.p, size_t(m.S) * sizeof(forest::SysState), cudaMemcpyDeviceToHost, s));
    waitStream(s);
    if (m.hst->error) throw std::runtime_error("forest: a device scan gave up waiting (bounded look-back)");
    if (model)
        for (int i = 0; i < m.S; ++i) m.capModel[i].stateRead(size_t(std::max(m.hsys[i].leaves, 0)));
}

void ForestEngine::setBuildMode(int mode)
{
    if (mode != 0 && mode != 1) throw std::invalid_argument("forest: build mode must be 0 (levels) or 1 (rounds)");
    m_->buildMode = mode;
}

bool ForestEngine::lastBuildByLevels() const { return m_->lastByLevels; }

// The converged build of all systems in one cooperative launch
// (forest::levelBuildKernel).  False where the rounds must run instead: a
// system whose rounds stop at maxDepth before converging, an arrival round
// beyond the tracked ones, LeafCount thresholds that wrap, or a device that
// cannot hold the grid.
bool ForestEngine::levelBuild()
{
    Impl &m = *m_;
    cudaStream_t s = m.cfg.stream;
    if (u64(m.cfg.bucket) * 512u > 0xffffffffull) return false;
    const bool hil = m.cfg.hilbert;
    const void *fn = hil ? reinterpret_cast<const void *>(&forest::levelBuildKernel<true>)
                         : reinterpret_cast<const void *>(&forest::levelBuildKernel<false>);
    int perSm = 0;
    AOT_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, lb::kThreads, 0));
    if (perSm <= 0) return false;
    const unsigned grid = unsigned(perSm) * unsigned(smCount());
    const size_t S = size_t(m.S);
    constexpr size_t kHeadBytes = (sizeof(lb::Control) + 255) & ~size_t(255);
    constexpr size_t kCtlBytes = kHeadBytes + sizeof(forest::LevelStatus);
    size_t cap = std::max<size_t>(m.lvCap, m.total / std::max(1u, m.cfg.bucket) + 4096);
    ensurePhysical(std::max(m.lastEntries, 2 * S + 4 * (m.total / std::max(1u, m.cfg.bucket)) + 4096));
    lb::Control hc{};
    forest::LevelStatus hl{};
    for (;;)
    {
        if (cap >= (size_t(1) << 31)) return false;
        m.lvRows.reserve(cap * lb::kRow * sizeof(u32), s);
        m.lvChild.reserve(cap * 8 * sizeof(u32), s);
        m.lvLeaves.reserve(cap * sizeof(u32), s);
        m.lvOffset.reserve(cap * sizeof(u32), s);
        m.lvUsys.reserve(cap * sizeof(u32), s);
        m.lvSysRoot.reserve(S * sizeof(u32), s);
        m.lvBins.reserve(S * (lb::kContribBins + lb::kArrivals) * sizeof(unsigned long long), s);
        m.lvCtl.reserve(kCtlBytes, s);
        m.lvCap = cap;
        forest::LevelArgs p{};
        lb::Arena &a = p.a;
        a.rows = m.lvRows.as<u32>();
        a.child = m.lvChild.as<u32>();
        a.leaves = m.lvLeaves.as<u32>();
        a.offset = m.lvOffset.as<u32>();
        a.usys = m.lvUsys.as<u32>();
        a.sysRoot = m.lvSysRoot.as<u32>();
        a.ctl = m.lvCtl.as<lb::Control>();
        a.contrib = m.lvBins.as<unsigned long long>();
        a.landed = a.contrib + S * lb::kContribBins;
        a.cap = u32(cap);
        p.idx = KeyIndex{m.P[0].as<u64>(), m.sample.as<u64>(), m.total, (m.total + kSampleStride - 1) >> kSampleShift};
        p.f = m.bufs();
        p.ls = reinterpret_cast<forest::LevelStatus *>(m.lvCtl.as<unsigned char>() + kHeadBytes);
        p.capacity = u32(std::min<size_t>(m.entryCap, 0xffffffffu));
        p.bucket = m.cfg.bucket;
        p.maxDepth = int(m.cfg.maxDepth);
        p.h = m.kpd.h;
        AOT_CHECK(cudaMemsetAsync(m.lvCtl.p, 0, kCtlBytes, s));
        void *args[] = {&p};
        AOT_CHECK(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(lb::kThreads), args, 0, s));
        noteLaunch();
        AOT_LAUNCH_CHECK();
        AOT_CHECK(cudaMemcpyAsync(&hc, m.lvCtl.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
        AOT_CHECK(cudaMemcpyAsync(&hl, p.ls, sizeof(hl), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        if (hl.bar.error) throw std::runtime_error("forest: a grid barrier of the level build gave up waiting");
        if (hc.overflow)
        {
            cap *= 2;
            continue;
        }
        if (hc.late) return false;
        if (hl.entriesOverflow)
        {
            ensurePhysical(size_t(hl.entries));
            continue;
        }
        if (hl.tooManyRounds) return false;
        if (hl.historyMismatch) throw std::logic_error("forest: level build history does not end at the tree");
        m.lastEntries = size_t(hl.entries);
        return true;
    }
}

void ForestEngine::build()
{
    Impl &m = *m_;
    cudaStream_t s = m.cfg.stream;
    waitStream(s);
    for (auto &c : m.capModel) c.buildStart();
    const bool tryLevels = m.buildMode == 0;
    sortParticles(tryLevels);
    m.lastByLevels = tryLevels && levelBuild();
    if (!m.lastByLevels)
    {
        ensurePhysical(size_t(2) * m.S);
        const forest::Bufs f = m.bufs();
        forest::initKernel<<<gridFor(size_t(m.S), 256), 256, 0, s>>>(f), noteLaunch();
        AOT_LAUNCH_CHECK();
        for (unsigned r = 0; r < m.cfg.maxDepth; ++r)
        {
            pass(true, nullptr);
            if (!m.hst->changed) break;
        }
    }
    // per-system leafCapacity from each system's round history
    readState(false);
    std::vector<long long> hist(size_t(std::max(m.cfg.maxDepth, 1u)) * m.S);
    AOT_CHECK(cudaMemcpy(hist.data(), m.history.p, hist.size() * sizeof(long long), cudaMemcpyDeviceToHost));
    size_t entries = 0;
    for (int i = 0; i < m.S; ++i)
    {
        forest::SysState &ss = m.hsys[i];
        std::vector<long long> rounds(size_t(ss.iteration));
        for (int r = 0; r < ss.iteration; ++r) rounds[r] = hist[size_t(r) * m.S + i];
        const size_t leaves = size_t(ss.leaves);
        const size_t cap = m.capModel[i].finishBuild(rounds.data(), rounds.size(), leaves);
        const size_t maxLeaves = (size_t(std::numeric_limits<int>::max()) - 1) / 8 * 7 + 1;
        if (cap > maxLeaves) throw std::length_error("adaptive_octree: buffer capacity exceeds node index range");
        m.capModel[i].prepare(cap);
        m.leafCap[i] = cap;
        ss.cap = int(cap);
        ss.needsResize = 0;
        entries += cap + 1;
    }
    AOT_CHECK(cudaMemcpyAsync(m.sys.p, m.hsys, size_t(m.S) * sizeof(forest::SysState), cudaMemcpyHostToDevice, s));
    ensurePhysical(entries);
    if (!m.lastByLevels)  // the level build writes the counts itself
    {
        forest::materializeKernel<<<unsigned(smCount()) * 8u, 256, 0, s>>>(m.bufs()), noteLaunch();
        AOT_LAUNCH_CHECK();
    }
    m.built = true;
    readState(true);
}

void ForestEngine::beginUpdate(const unsigned char *frozen)
{
    Impl &m = *m_;
    if (!m.built) throw std::logic_error("adaptive_octree: call build() before update()");
    cudaStream_t s = m.cfg.stream;
    if (frozen)
        AOT_CHECK(cudaMemcpyAsync(m.frozen.p, frozen, size_t(m.S), cudaMemcpyHostToDevice, s));
    else
        AOT_CHECK(cudaMemsetAsync(m.frozen.p, 0, size_t(m.S), s));
    AOT_CHECK(cudaMemsetAsync(&m.st.as<forest::State>()->changedPasses, 0, sizeof(int), s));
    sortParticles(false);
    const forest::Bufs f = m.bufs();
    forest::refreshKernel<true><<<unsigned(smCount()) * 8u, forest::kThreads, 0, s>>>(f), noteLaunch();
    AOT_LAUNCH_CHECK();
}

void ForestEngine::endUpdate()
{
    Impl &m = *m_;
    forest::materializeKernel<<<unsigned(smCount()) * 8u, 256, 0, m.cfg.stream>>>(m.bufs()), noteLaunch();
    AOT_LAUNCH_CHECK();
}

void ForestEngine::update(const unsigned char *frozen)
{
    beginUpdate(frozen);
    for (unsigned i = 0; i < m_->cfg.iterations; ++i) pass(false, m_->frozen.as<unsigned char>());
    endUpdate();
}

// A pass after every system converged finds nothing to change, and its
// scatter, commit and refresh return at once (State::changed = 0), so a group
// of passes may overshoot convergence at the cost of its decisions only.
void ForestEngine::updateUntilConverged(const unsigned char *frozen, unsigned maxPasses, unsigned *changedPasses)
{
    if (maxPasses == 0) throw std::invalid_argument("forest: updateUntilConverged needs maxPasses >= 1");
    beginUpdate(frozen);
    Impl &m = *m_;
    cudaStream_t s = m.cfg.stream;
    const unsigned group = std::max(1u, m.cfg.iterations);
    unsigned launched = 0;
    while (launched < maxPasses)
    {
        const unsigned k = std::min(group, maxPasses - launched);
        for (unsigned i = 0; i < k; ++i) pass(false, m.frozen.as<unsigned char>());
        launched += k;
        if (launched == maxPasses) break;
        AOT_CHECK(cudaMemcpyAsync(m.hst, m.st.p, sizeof(forest::State), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        if (m.hst->error) throw std::runtime_error("forest: a device scan gave up waiting (bounded look-back)");
        if (!m.hst->changed) break;
    }
    endUpdate();
    if (changedPasses)
    {
        AOT_CHECK(cudaMemcpyAsync(m.hst, m.st.p, sizeof(forest::State), cudaMemcpyDeviceToHost, s));
        waitStream(s);
        if (m.hst->error) throw std::runtime_error("forest: a device scan gave up waiting (bounded look-back)");
        *changedPasses = unsigned(m.hst->changedPasses);
    }
}

bool ForestEngine::needsResize()
{
    Impl &m = *m_;
    if (!m.built) return false;
    readState(true);
    for (int i = 0; i < m.S; ++i)
        if (m.hsys[i].needsResize) return true;
    return false;
}

void ForestEngine::resizeBuffers()
{
    Impl &m = *m_;
    if (!m.built) throw std::logic_error("adaptive_octree: call build() before resizeBuffers()");
    readState(true);
    size_t entries = 0;
    for (int i = 0; i < m.S; ++i)
    {
        forest::SysState &ss = m.hsys[i];
        if (ss.needsResize)
        {
            // resizeBuffers (octree.cu:539-551): 25% more capacity
            const size_t cap = m.leafCap[i] + (m.leafCap[i] + 3) / 4;
            const size_t maxLeaves = (size_t(std::numeric_limits<int>::max()) - 1) / 8 * 7 + 1;
            if (cap > maxLeaves) throw std::length_error("adaptive_octree: buffer capacity exceeds node index range");
            m.capModel[i].prepare(cap);
            m.leafCap[i] = cap;
            ss.cap = int(cap);
            ss.needsResize = 0;
        }
        entries += m.leafCap[i] + 1;
    }
    ensurePhysical(entries);
    AOT_CHECK(cudaMemcpyAsync(m.sys.p, m.hsys, size_t(m.S) * sizeof(forest::SysState), cudaMemcpyHostToDevice,
                              m.cfg.stream));
    waitStream(m.cfg.stream);
}

void ForestEngine::buffer(int s, int which, const void **ptr, size_t *len) const
{
    const Impl &m = *m_;
    if (s < 0 || s >= m.S) throw std::invalid_argument("forest: system index out of range");
    const forest::System &sy = m.systems[s];
    const forest::SysState &ss = m.hsys[s];
    const int a = m.hst->activeBuffer;
    switch (which)
    {
    case ParticleKeys:
        *ptr = m.P[0].as<u64>() + sy.base;
        *len = sy.n;
        break;
    case Perm:
        *ptr = m.Perm[0].as<u32>() + sy.base;
        *len = sy.n;
        break;
    case Cornerstone:
        *ptr = m.K[a].as<u64>() + ss.start;
        *len = m.built ? size_t(ss.leaves) + 1 : 0;
        break;
    case LeafCounts:
        *ptr = m.N.as<u32>() + ss.start;
        *len = m.built ? size_t(ss.leaves) : 0;
        break;
    default:
        throw std::invalid_argument("forest: unknown buffer");
    }
}

ForestEngine::SystemInfo ForestEngine::info(int s) const
{
    const Impl &m = *m_;
    if (s < 0 || s >= m.S) throw std::invalid_argument("forest: system index out of range");
    const forest::SysState &ss = m.hsys[s];
    return SystemInfo{m.systems[s].n, ss.active, m.built ? size_t(ss.leaves) : 0, m.leafCap[s],
                      ss.needsResize != 0};
}
}  // namespace aot
