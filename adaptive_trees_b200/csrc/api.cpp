// api.cpp -- adaptive_octree::Octree<Real> / KDTree3D<Real> and the C ABI over TreeEngine.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>
#include <new>
#include <ostream>
#include <string>

#include "adaptive_octree/tree.hpp"
#include "adaptive_trees_b200.h"
#include "engine.hpp"
#include "forest.hpp"
#include "particle_io.hpp"
#include "serve.hpp"

namespace adaptive_octree
{
namespace
{
template <class Real>
aot::EngineConfig octreeEngineConfig(const OctreeConfig<Real> &c)
{
    aot::EngineConfig e;
    e.kind = 0;
    e.real = sizeof(Real) == 4 ? 0 : 1;
    e.bucket = c.maxParticlesPerLeaf;
    e.maxDepth = c.maxDepth;
    e.iterations = c.updateIterations;
    e.nf = c.splitCriterion == SplitCriterion::NFCount;
    e.hilbert = c.sfcKind == SfcKind::Hilbert;
    const double b[6] = {double(c.box.xmin), double(c.box.xmax), double(c.box.ymin),
                         double(c.box.ymax), double(c.box.zmin), double(c.box.zmax)};
    std::memcpy(e.box, b, sizeof(b));
    e.views = c.views;
    e.stream = c.stream;
    return e;
}
template <class Real>
aot::EngineConfig binaryEngineConfig(const KDTree3DConfig<Real> &c)
{
    aot::EngineConfig e;
    e.kind = 1;
    e.real = sizeof(Real) == 4 ? 0 : 1;
    e.bucket = c.maxParticlesPerLeaf;
    e.maxDepth = c.maxDepth;
    e.iterations = c.updateIterations;
    const double b[6] = {double(c.box.xmin), double(c.box.xmax), double(c.box.ymin),
                         double(c.box.ymax), double(c.box.zmin), double(c.box.zmax)};
    std::memcpy(e.box, b, sizeof(b));
    e.views = c.views;
    e.stream = c.stream;
    return e;
}
template <class T>
const DeviceVector<T> &view(const aot::TreeEngine &e, int which, DeviceVector<T> &slot)
{
    const void *p = nullptr;
    size_t len = 0, cap = 0, elem = 0;
    e.buffer(which, &p, &len, &cap, &elem);
    slot = DeviceVector<T>(static_cast<const T *>(p), len, cap);
    return slot;
}
void printSummary(std::ostream &out, const aot::TreeEngine &e, const char *name)
{
    out << name << ": " << e.numParticles() << " particle slots, " << e.numActiveParticles() << " active, "
        << e.leafCapacity() << " leaf capacity, " << e.numNodes() << " view nodes\n";
}
}  // namespace

// ---------------------------------------------------------------- Octree<Real>
template <class Real>
Octree<Real>::Octree(const Real *x, const Real *y, const Real *z, std::size_t n, Config config)
    : engine_(std::make_unique<aot::TreeEngine>(x, y, z, n, octreeEngineConfig(config)))
{
}
template <class Real> Octree<Real>::~Octree() = default;
template <class Real> Octree<Real>::Octree(Octree &&) noexcept = default;
template <class Real> Octree<Real> &Octree<Real>::operator=(Octree &&) noexcept = default;
template <class Real> void Octree<Real>::print(std::ostream &out) const { printSummary(out, *engine_, "Octree"); }
template <class Real> void Octree<Real>::build() { engine_->build(); }
template <class Real> void Octree<Real>::update() { engine_->update(); }
template <class Real> void Octree<Real>::computeViews(ViewConfig v) { engine_->computeViews(v); }
template <class Real> void Octree<Real>::computeViews() { engine_->computeViews(engine_->config().views); }
template <class Real> bool Octree<Real>::doBuffersNeedResize() const { return engine_->doBuffersNeedResize(); }
template <class Real> void Octree<Real>::resizeBuffers() { engine_->resizeBuffers(); }
template <class Real> const NodeIndex *Octree<Real>::numLeaves_d() const { return engine_->numLeavesDevice(); }
template <class Real> const NodeIndex *Octree<Real>::numNodes_d() const { return engine_->numNodesDevice(); }
template <class Real> const unsigned *Octree<Real>::numActiveParticles_d() const
{
    return engine_->numActiveParticlesDevice();
}
template <class Real> const DeviceVector<KeyType> &Octree<Real>::particleKeys_d() const
{
    return view<KeyType>(*engine_, 0, views_.particleKeys);
}
template <class Real> const DeviceVector<PermIndex> &Octree<Real>::perm_d() const
{
    return view<PermIndex>(*engine_, 1, views_.perm);
}
template <class Real> const DeviceVector<KeyType> &Octree<Real>::cornerstone_d() const
{
    return view<KeyType>(*engine_, 2, views_.cornerstone);
}
template <class Real> const DeviceVector<unsigned> &Octree<Real>::leafCounts_d() const
{
    return view<unsigned>(*engine_, 3, views_.leafCounts);
}
template <class Real> const DeviceVector<unsigned> &Octree<Real>::nearFieldCounts_d() const
{
    return view<unsigned>(*engine_, 4, views_.nearFieldCounts);
}
template <class Real> const DeviceVector<KeyType> &Octree<Real>::sfcBoxIndex_d() const
{
    return view<KeyType>(*engine_, 5, views_.sfcBoxIndex);
}
template <class Real> const DeviceVector<std::uint8_t> &Octree<Real>::hasBoxSplit_d() const
{
    return view<std::uint8_t>(*engine_, 6, views_.hasBoxSplit);
}
template <class Real> const DeviceVector<std::uint8_t> &Octree<Real>::boxDepth_d() const
{
    return view<std::uint8_t>(*engine_, 7, views_.boxDepth);
}
template <class Real> const DeviceVector<NodeIndex> &Octree<Real>::parentIndex_d() const
{
    return view<NodeIndex>(*engine_, 8, views_.parentIndex);
}
template <class Real> const DeviceVector<NodeIndex> &Octree<Real>::childIndex_d() const
{
    return view<NodeIndex>(*engine_, 9, views_.childIndex);
}
template <class Real> const DeviceVector<NodeIndex> &Octree<Real>::levelOffset_d() const
{
    return view<NodeIndex>(*engine_, 10, views_.levelOffset);
}
template <class Real> unsigned Octree<Real>::maxAchievedDepth() const { return engine_->maxAchievedDepth(); }
template <class Real> const DeviceVector<unsigned> &Octree<Real>::particleBeginIndex_d() const
{
    return view<unsigned>(*engine_, 11, views_.particleBeginIndex);
}
template <class Real> const DeviceVector<unsigned> &Octree<Real>::particleCounts_d() const
{
    return view<unsigned>(*engine_, 12, views_.particleCounts);
}
template <class Real> const DeviceVector<KeyType> &Octree<Real>::sfcParticleIndex_d() const
{
    return view<KeyType>(*engine_, 13, views_.sfcParticleIndex);
}
template <class Real> std::size_t Octree<Real>::numParticles() const { return engine_->numParticles(); }
template <class Real> std::size_t Octree<Real>::numActiveParticles() const { return engine_->numActiveParticles(); }
template <class Real> std::size_t Octree<Real>::numNodes() const { return engine_->numNodes(); }
template <class Real> SplitCriterion Octree<Real>::splitCriterion() const
{
    return engine_->config().nf ? SplitCriterion::NFCount : SplitCriterion::LeafCount;
}
template <class Real> SfcKind Octree<Real>::sfcKind() const
{
    return engine_->config().hilbert ? SfcKind::Hilbert : SfcKind::Morton;
}
template class Octree<float>;
template class Octree<double>;

// ---------------------------------------------------------------- KDTree3D<Real>
template <class Real>
KDTree3D<Real>::KDTree3D(const Real *x, const Real *y, const Real *z, std::size_t n, Config config)
    : engine_(std::make_unique<aot::TreeEngine>(x, y, z, n, binaryEngineConfig(config)))
{
}
template <class Real> KDTree3D<Real>::~KDTree3D() = default;
template <class Real> KDTree3D<Real>::KDTree3D(KDTree3D &&) noexcept = default;
template <class Real> KDTree3D<Real> &KDTree3D<Real>::operator=(KDTree3D &&) noexcept = default;
template <class Real> void KDTree3D<Real>::print(std::ostream &out) const { printSummary(out, *engine_, "KDTree3D"); }
template <class Real> void KDTree3D<Real>::build() { engine_->build(); }
template <class Real> void KDTree3D<Real>::update() { engine_->update(); }
template <class Real> void KDTree3D<Real>::computeViews(ViewConfig v) { engine_->computeViews(v); }
template <class Real> void KDTree3D<Real>::computeViews() { engine_->computeViews(engine_->config().views); }
template <class Real> bool KDTree3D<Real>::doBuffersNeedResize() const { return engine_->doBuffersNeedResize(); }
template <class Real> void KDTree3D<Real>::resizeBuffers() { engine_->resizeBuffers(); }
template <class Real> const NodeIndex *KDTree3D<Real>::numLeaves_d() const { return engine_->numLeavesDevice(); }
template <class Real> const NodeIndex *KDTree3D<Real>::numNodes_d() const { return engine_->numNodesDevice(); }
template <class Real> const unsigned *KDTree3D<Real>::numActiveParticles_d() const
{
    return engine_->numActiveParticlesDevice();
}
template <class Real> const DeviceVector<KeyType> &KDTree3D<Real>::particleKeys_d() const
{
    return view<KeyType>(*engine_, 0, views_.particleKeys);
}
template <class Real> const DeviceVector<PermIndex> &KDTree3D<Real>::perm_d() const
{
    return view<PermIndex>(*engine_, 1, views_.perm);
}
template <class Real> const DeviceVector<KeyType> &KDTree3D<Real>::cornerstone_d() const
{
    return view<KeyType>(*engine_, 2, views_.cornerstone);
}
template <class Real> const DeviceVector<unsigned> &KDTree3D<Real>::leafCounts_d() const
{
    return view<unsigned>(*engine_, 3, views_.leafCounts);
}
template <class Real> const DeviceVector<KeyType> &KDTree3D<Real>::sfcBoxIndex_d() const
{
    return view<KeyType>(*engine_, 5, views_.sfcBoxIndex);
}
template <class Real> const DeviceVector<std::uint8_t> &KDTree3D<Real>::hasBoxSplit_d() const
{
    return view<std::uint8_t>(*engine_, 6, views_.hasBoxSplit);
}
template <class Real> const DeviceVector<std::uint8_t> &KDTree3D<Real>::boxDepth_d() const
{
    return view<std::uint8_t>(*engine_, 7, views_.boxDepth);
}
template <class Real> const DeviceVector<NodeIndex> &KDTree3D<Real>::parentIndex_d() const
{
    return view<NodeIndex>(*engine_, 8, views_.parentIndex);
}
template <class Real> const DeviceVector<NodeIndex> &KDTree3D<Real>::childIndex_d() const
{
    return view<NodeIndex>(*engine_, 9, views_.childIndex);
}
template <class Real> const DeviceVector<NodeIndex> &KDTree3D<Real>::levelOffset_d() const
{
    return view<NodeIndex>(*engine_, 10, views_.levelOffset);
}
template <class Real> unsigned KDTree3D<Real>::maxAchievedDepth() const { return engine_->maxAchievedDepth(); }
template <class Real> const DeviceVector<unsigned> &KDTree3D<Real>::particleBeginIndex_d() const
{
    return view<unsigned>(*engine_, 11, views_.particleBeginIndex);
}
template <class Real> const DeviceVector<unsigned> &KDTree3D<Real>::particleCounts_d() const
{
    return view<unsigned>(*engine_, 12, views_.particleCounts);
}
template <class Real> const DeviceVector<KeyType> &KDTree3D<Real>::sfcParticleIndex_d() const
{
    return view<KeyType>(*engine_, 13, views_.sfcParticleIndex);
}
template <class Real> std::size_t KDTree3D<Real>::numParticles() const { return engine_->numParticles(); }
template <class Real> std::size_t KDTree3D<Real>::numActiveParticles() const { return engine_->numActiveParticles(); }
template <class Real> std::size_t KDTree3D<Real>::numNodes() const { return engine_->numNodes(); }
template class KDTree3D<float>;
template class KDTree3D<double>;
}  // namespace adaptive_octree

// =========================================================================
// C ABI
// =========================================================================
struct ao_tree
{
    std::unique_ptr<aot::TreeEngine> engine;
};

struct ao_batch
{
    std::unique_ptr<aot::ForestEngine> engine;
};

struct ao_server
{
    std::unique_ptr<aot::Server> server;
};

struct ao_manifest
{
    aot::io::Manifest m;
};

namespace
{
thread_local std::string g_lastError;

ao_status fail(ao_status s, const char *msg)
{
    g_lastError = msg ? msg : "";
    return s;
}

template <class F>
ao_status guarded(F &&f)
{
    try
    {
        f();
        return AO_OK;
    }
    catch (const std::invalid_argument &e)
    {
        return fail(AO_ERR_INVALID_ARGUMENT, e.what());
    }
    catch (const std::length_error &e)
    {
        return fail(AO_ERR_LENGTH, e.what());
    }
    catch (const std::logic_error &e)
    {
        return fail(AO_ERR_LOGIC, e.what());
    }
    catch (const aot::CudaError &e)
    {
        return fail(e.code == cudaErrorMemoryAllocation ? AO_ERR_OUT_OF_MEMORY : AO_ERR_CUDA, e.what());
    }
    catch (const std::bad_alloc &e)
    {
        return fail(AO_ERR_OUT_OF_MEMORY, e.what());
    }
    catch (const std::exception &e)
    {
        return fail(AO_ERR_RUNTIME, e.what());
    }
    catch (...)
    {
        return fail(AO_ERR_RUNTIME, "unknown error");
    }
}

// Tree<Real, Kind>::backendConfig (tree.hpp:108-133) + backend defaults.
aot::EngineConfig engineConfig(int kind, int real, const ao_config &c, void *stream)
{
    if (kind != AO_OCTREE && kind != AO_BINARY) throw std::invalid_argument("ao_tree_create: unknown tree kind");
    if (real != AO_FLOAT32 && real != AO_FLOAT64) throw std::invalid_argument("ao_tree_create: unknown real type");
    if (c.max_depth < -1 || c.update_iterations < -1) throw std::invalid_argument("Tree: use -1 for backend defaults");
    aot::EngineConfig e;
    e.kind = kind;
    e.real = real;
    e.bucket = c.max_particles_per_leaf;
    e.maxDepth = c.max_depth >= 0 ? unsigned(c.max_depth) : (kind == AO_OCTREE ? 21u : 63u);
    e.iterations = c.update_iterations >= 0 ? unsigned(c.update_iterations) : (kind == AO_OCTREE ? 2u : 6u);
    std::memcpy(e.box, c.box, sizeof(e.box));
    e.views.treeStructure = c.views_tree_structure != 0;
    e.views.particleCountsPerBox = c.views_particle_counts != 0;
    e.views.particleMapping = c.views_particle_mapping != 0;
    e.stream = static_cast<cudaStream_t>(stream);
    if (kind == AO_OCTREE)
    {
        e.nf = c.split_criterion == AO_NF_COUNT;
        e.hilbert = c.sfc_kind == AO_HILBERT;
    }
    else
    {
        if (c.split_criterion != AO_LEAF_COUNT)
            throw std::invalid_argument("Tree: Binary NFCount is not implemented yet");
        if (c.sfc_kind != AO_MORTON) throw std::invalid_argument("Tree: Binary uses longest-side keys, not Hilbert");
    }
    return e;
}
}  // namespace

extern "C" {

const char *ao_last_error(void) { return g_lastError.c_str(); }

ao_status ao_tree_create(int kind, int real_type, const void *x, const void *y, const void *z, size_t n,
                         const ao_config *config, void *stream, ao_tree **out)
{
    return guarded([&] {
        if (!out || !config) throw std::invalid_argument("ao_tree_create: null argument");
        *out = nullptr;
        auto e = std::make_unique<aot::TreeEngine>(x, y, z, n, engineConfig(kind, real_type, *config, stream));
        *out = new ao_tree{std::move(e)};
    });
}

ao_status ao_tree_destroy(ao_tree *tree)
{
    return guarded([&] { delete tree; });
}

#define AO_NEED_TREE()                                                     \
    if (!tree) throw std::invalid_argument("null ao_tree handle")

ao_status ao_tree_build(ao_tree *tree)
{
    return guarded([&] {
        AO_NEED_TREE();
        tree->engine->build();
    });
}

ao_status ao_tree_update(ao_tree *tree)
{
    return guarded([&] {
        AO_NEED_TREE();
        tree->engine->update();
    });
}

ao_status ao_tree_set_profiling(ao_tree *tree, int on)
{
    return guarded([&] {
        AO_NEED_TREE();
        tree->engine->setProfiling(on != 0);
    });
}

ao_status ao_tree_set_build_mode(ao_tree *tree, int mode)
{
    return guarded([&] {
        AO_NEED_TREE();
        tree->engine->setBuildMode(mode);
    });
}

ao_status ao_tree_build_path(ao_tree *tree, int *by_levels, int *rounds)
{
    return guarded([&] {
        AO_NEED_TREE();
        if (by_levels) *by_levels = tree->engine->lastBuildByLevels() ? 1 : 0;
        if (rounds) *rounds = tree->engine->buildRounds();
    });
}

ao_status ao_tree_stage_times(ao_tree *tree, ao_stage_times *out)
{
    return guarded([&] {
        AO_NEED_TREE();
        if (!out) throw std::invalid_argument("ao_tree_stage_times: null output");
        const aot::TreeEngine::StageTimes t = tree->engine->stageTimes();
        out->keys_and_sort_ms = t.keysAndSortMs;
        out->refresh_ms = t.refreshMs;
        out->passes_ms = t.passesMs;
        out->finish_ms = t.finishMs;
        out->total_ms = t.totalMs;
        out->near_field_ms = t.nearFieldMs;
        out->near_field_first_ms = t.nearFieldFirstMs;
        out->near_field_launches = t.nearFieldLaunches;
        out->call = t.call;
        out->valid = t.valid ? 1 : 0;
    });
}

ao_status ao_tree_update_until_converged(ao_tree *tree, int max_passes, int *changed_passes)
{
    return guarded([&] {
        AO_NEED_TREE();
        if (max_passes < 1) throw std::invalid_argument("ao_tree_update_until_converged: max_passes must be >= 1");
        unsigned changed = 0;
        tree->engine->updateUntilConverged(unsigned(max_passes), changed_passes ? &changed : nullptr);
        if (changed_passes) *changed_passes = int(changed);
    });
}

ao_status ao_tree_compute_views(ao_tree *tree, const ao_view_config *views)
{
    return guarded([&] {
        AO_NEED_TREE();
        adaptive_octree::ViewConfig v = tree->engine->config().views;
        if (views)
        {
            v.treeStructure = views->tree_structure != 0;
            v.particleCountsPerBox = views->particle_counts_per_box != 0;
            v.particleMapping = views->particle_mapping != 0;
        }
        tree->engine->computeViews(v);
    });
}

ao_status ao_tree_needs_resize(ao_tree *tree, int *out)
{
    return guarded([&] {
        AO_NEED_TREE();
        if (!out) throw std::invalid_argument("ao_tree_needs_resize: null output");
        *out = tree->engine->doBuffersNeedResize() ? 1 : 0;
    });
}

ao_status ao_tree_resize_buffers(ao_tree *tree)
{
    return guarded([&] {
        AO_NEED_TREE();
        tree->engine->resizeBuffers();
    });
}

ao_status ao_tree_get_buffer(ao_tree *tree, int which, const void **dptr, size_t *len, size_t *capacity)
{
    return guarded([&] {
        AO_NEED_TREE();
        tree->engine->buffer(which, dptr, len, capacity, nullptr);
    });
}

ao_status ao_tree_counters(ao_tree *tree, const int **num_leaves_d, const int **num_nodes_d,
                           const unsigned **num_active_particles_d)
{
    return guarded([&] {
        AO_NEED_TREE();
        if (num_leaves_d) *num_leaves_d = tree->engine->numLeavesDevice();
        if (num_nodes_d) *num_nodes_d = tree->engine->numNodesDevice();
        if (num_active_particles_d) *num_active_particles_d = tree->engine->numActiveParticlesDevice();
    });
}

ao_status ao_tree_get_info(ao_tree *tree, ao_tree_info *info)
{
    return guarded([&] {
        AO_NEED_TREE();
        if (!info) throw std::invalid_argument("ao_tree_get_info: null output");
        const aot::TreeEngine &e = *tree->engine;
        size_t leaves = 0;
        e.buffer(aot::TreeEngine::LeafCounts, nullptr, &leaves, nullptr, nullptr);
        info->num_particles = e.numParticles();
        info->num_active_particles = e.numActiveParticles();
        info->num_nodes = e.numNodes();
        info->num_leaves = leaves;
        info->leaf_capacity = e.leafCapacity();
        info->max_achieved_depth = e.maxAchievedDepth();
        info->split_criterion = e.config().nf ? AO_NF_COUNT : AO_LEAF_COUNT;
        info->sfc_kind = e.config().kind == AO_BINARY ? -1 : (e.config().hilbert ? AO_HILBERT : AO_MORTON);
        info->kernel_launches = aot::TreeEngine::kernelLaunches();
    });
}

ao_status ao_compute_sfc_keys(int kind, int real_type, const void *x, const void *y, const void *z, size_t n,
                              const double *box, int sfc_kind, unsigned max_depth, unsigned long long *keys_d,
                              unsigned *perm_d, void *stream)
{
    return guarded([&] {
        if (kind != AO_OCTREE && kind != AO_BINARY) throw std::invalid_argument("ao_compute_sfc_keys: unknown kind");
        if (real_type != AO_FLOAT32 && real_type != AO_FLOAT64)
            throw std::invalid_argument("ao_compute_sfc_keys: unknown real type");
        if (n > 0 && (!x || !y || !z || !keys_d || !box))
            throw std::invalid_argument("ao_compute_sfc_keys: null argument");
        aot::TreeEngine::computeKeys(kind, real_type, x, y, z, n, box, sfc_kind == AO_HILBERT, max_depth, keys_d,
                                     perm_d, static_cast<cudaStream_t>(stream));
    });
}

ao_status ao_sort_pairs(void *scratch, size_t *scratch_bytes, const unsigned long long *keys_in,
                        unsigned long long *keys_out, const unsigned *values_in, unsigned *values_out, size_t n,
                        int begin_bit, int end_bit, void *stream)
{
    return guarded([&] {
        aot::TreeEngine::sortPairs(scratch, scratch_bytes, keys_in, keys_out, values_in, values_out, n, begin_bit,
                                   end_bit, static_cast<cudaStream_t>(stream));
    });
}

ao_status ao_sort_pairs_check(const void *scratch, size_t n, void *stream)
{
    return guarded([&] {
        if (n > 0 && aot::TreeEngine::sortPairsFailed(scratch, n, static_cast<cudaStream_t>(stream)))
            throw std::runtime_error("ao_sort_pairs: a bounded look-back wait gave up; the output is not sorted");
    });
}

ao_status ao_selftest_bounded_wait(int which, unsigned spin_limit, int *error_word)
{
    return guarded([&] {
        const int e = aot::TreeEngine::boundedWaitProbe(which, spin_limit);
        if (error_word) *error_word = e;
        if (e != 0)
            throw std::runtime_error(std::string("ao_selftest_bounded_wait: the ") +
                                     (which == 0 ? "radix sort" : "decide+scan") +
                                     " look-back wait gave up after its limit and the kernel returned");
    });
}

ao_status ao_sort_config_count(int *count)
{
    return guarded([&] {
        if (!count) throw std::invalid_argument("ao_sort_config_count: null output");
        *count = aot::sortConfigCount();
    });
}

ao_status ao_sort_config_info(int config, int *digit_bits, int *items_per_thread)
{
    return guarded([&] {
        if (!digit_bits || !items_per_thread) throw std::invalid_argument("ao_sort_config_info: null output");
        const aot::SortTuning t = aot::sortConfigInfo(config);
        *digit_bits = t.digitBits;
        *items_per_thread = t.itemsPerThread;
    });
}

ao_status ao_sort_tuning(int segmented, size_t n, int *config, int *digit_bits, int *items_per_thread, int *tuned)
{
    return guarded([&] {
        if (!config || !digit_bits || !items_per_thread || !tuned)
            throw std::invalid_argument("ao_sort_tuning: null output");
        const aot::SortTuning t = aot::sortTuning(segmented != 0, n);
        *config = t.config;
        *digit_bits = t.digitBits;
        *items_per_thread = t.itemsPerThread;
        *tuned = t.tuned ? 1 : 0;
    });
}

ao_status ao_sort_set_autotune(int on)
{
    return guarded([&] { aot::sortSetAutotune(on != 0); });
}

ao_status ao_sort_force_config(int config)
{
    return guarded([&] { aot::sortForceConfig(config); });
}

ao_status ao_sort_forget_tuning(void)
{
    return guarded([&] { aot::sortForgetTuning(); });
}

ao_status ao_tree_gather(ao_tree *tree, const void *src, void *dst, size_t elem_bytes)
{
    return guarded([&] {
        if (!tree) throw std::invalid_argument("ao_tree_gather: null tree");
        tree->engine->gather(src, dst, elem_bytes);
    });
}

ao_status ao_batch_create(int real_type, int num_systems, const void *const *x, const void *const *y,
                          const void *const *z, const size_t *counts, const ao_config *config, void *stream,
                          ao_batch **out)
{
    return guarded([&] {
        if (!out || !config) throw std::invalid_argument("ao_batch_create: null argument");
        *out = nullptr;
        const aot::EngineConfig cfg = engineConfig(AO_OCTREE, real_type, *config, stream);
        auto b = std::make_unique<ao_batch>();
        b->engine = std::make_unique<aot::ForestEngine>(x, y, z, counts, num_systems, cfg);
        *out = b.release();
    });
}

ao_status ao_batch_destroy(ao_batch *batch)
{
    return guarded([&] { delete batch; });
}

ao_status ao_batch_build(ao_batch *batch)
{
    return guarded([&] {
        if (!batch) throw std::invalid_argument("ao_batch_build: null batch");
        batch->engine->build();
    });
}

ao_status ao_batch_set_build_mode(ao_batch *batch, int mode)
{
    return guarded([&] {
        if (!batch) throw std::invalid_argument("ao_batch_set_build_mode: null batch");
        batch->engine->setBuildMode(mode);
    });
}

ao_status ao_batch_build_path(ao_batch *batch, int *by_levels)
{
    return guarded([&] {
        if (!batch) throw std::invalid_argument("ao_batch_build_path: null batch");
        if (by_levels) *by_levels = batch->engine->lastBuildByLevels() ? 1 : 0;
    });
}

ao_status ao_batch_update(ao_batch *batch, const unsigned char *frozen)
{
    return guarded([&] {
        if (!batch) throw std::invalid_argument("ao_batch_update: null batch");
        batch->engine->update(frozen);
    });
}

ao_status ao_batch_update_until_converged(ao_batch *batch, const unsigned char *frozen, int max_passes,
                                          int *changed_passes)
{
    return guarded([&] {
        if (!batch) throw std::invalid_argument("ao_batch_update_until_converged: null batch");
        if (max_passes < 1) throw std::invalid_argument("ao_batch_update_until_converged: max_passes must be >= 1");
        unsigned changed = 0;
        batch->engine->updateUntilConverged(frozen, unsigned(max_passes), changed_passes ? &changed : nullptr);
        if (changed_passes) *changed_passes = int(changed);
    });
}

ao_status ao_batch_needs_resize(ao_batch *batch, int *any)
{
    return guarded([&] {
        if (!batch || !any) throw std::invalid_argument("ao_batch_needs_resize: null argument");
        *any = batch->engine->needsResize() ? 1 : 0;
    });
}

ao_status ao_batch_resize_buffers(ao_batch *batch)
{
    return guarded([&] {
        if (!batch) throw std::invalid_argument("ao_batch_resize_buffers: null batch");
        batch->engine->resizeBuffers();
    });
}

ao_status ao_batch_set_coordinates(ao_batch *batch, int system, const void *x, const void *y, const void *z)
{
    return guarded([&] {
        if (!batch) throw std::invalid_argument("ao_batch_set_coordinates: null batch");
        batch->engine->setCoordinates(system, x, y, z);
    });
}

ao_status ao_batch_get_buffer(ao_batch *batch, int system, int which, const void **ptr, size_t *size)
{
    return guarded([&] {
        if (!batch || !ptr || !size) throw std::invalid_argument("ao_batch_get_buffer: null argument");
        if (which < AO_BUF_PARTICLE_KEYS || which > AO_BUF_LEAF_COUNTS)
            throw std::invalid_argument("ao_batch_get_buffer: a batch exposes keys, perm, cornerstone and counts");
        batch->engine->buffer(system, which, ptr, size);
    });
}

ao_status ao_batch_get_info(ao_batch *batch, int system, ao_batch_system_info *info)
{
    return guarded([&] {
        if (!batch || !info) throw std::invalid_argument("ao_batch_get_info: null argument");
        const aot::ForestEngine::SystemInfo s = batch->engine->info(system);
        info->num_particles = s.particles;
        info->num_active_particles = s.active;
        info->num_leaves = s.leaves;
        info->leaf_capacity = s.leafCapacity;
        info->needs_resize = s.needsResize ? 1 : 0;
    });
}

ao_status ao_serve_create(int slots, size_t memory_budget_bytes, ao_server **out)
{
    return guarded([&] {
        if (!out) throw std::invalid_argument("ao_serve_create: null argument");
        *out = nullptr;
        if (slots <= 0) throw std::invalid_argument("ao_serve_create: need at least one slot");
        if (memory_budget_bytes == 0) throw std::invalid_argument("ao_serve_create: the memory budget must be positive");
        auto s = std::make_unique<ao_server>();
        s->server = std::make_unique<aot::Server>(slots, memory_budget_bytes);
        *out = s.release();
    });
}

ao_status ao_serve_destroy(ao_server *server)
{
    return guarded([&] { delete server; });
}

ao_status ao_serve_submit(ao_server *server, const ao_request *request, long long *ticket)
{
    return guarded([&] {
        if (!server || !request || !ticket) throw std::invalid_argument("ao_serve_submit: null argument");
        aot::ServeRequest r;
        r.op = request->op;
        r.tree = request->tree;
        if (request->op == AO_REQUEST_BUILD)
            r.cfg = engineConfig(request->kind, request->real_type, request->config, nullptr);
        r.n = request->n;
        r.x = request->x;
        r.y = request->y;
        r.z = request->z;
        r.digest = request->want_digest != 0;
        *ticket = server->server->submit(r);
    });
}

ao_status ao_serve_wait(ao_server *server, long long ticket, ao_request_result *result)
{
    aot::ServeResult r;
    const ao_status s = guarded([&] {
        if (!server || !result) throw std::invalid_argument("ao_serve_wait: null argument");
        r = server->server->wait(ticket);
        result->status = r.status;
        result->queued_ms = r.queuedMs;
        result->latency_ms = r.latencyMs;
        result->num_leaves = r.leaves;
        result->resizes = r.resizes;
        result->digest = r.digest;
    });
    if (s != AO_OK) return s;
    if (r.status != AO_OK) return fail(static_cast<ao_status>(r.status), r.message.c_str());
    return AO_OK;
}

ao_status ao_serve_drain(ao_server *server)
{
    return guarded([&] {
        if (!server) throw std::invalid_argument("ao_serve_drain: null server");
        server->server->drain();
    });
}

ao_status ao_serve_get_stats(ao_server *server, ao_serve_stats *stats)
{
    return guarded([&] {
        if (!server || !stats) throw std::invalid_argument("ao_serve_get_stats: null argument");
        const aot::ServeStats s = server->server->stats();
        stats->submitted = s.submitted;
        stats->completed = s.completed;
        stats->failed = s.failed;
        stats->resident_trees = s.residentTrees;
        stats->resident_bytes = s.residentBytes;
        stats->peak_bytes = s.peakBytes;
        stats->particles = s.particles;
        stats->p50_ms = s.p50Ms;
        stats->p99_ms = s.p99Ms;
        stats->mean_ms = s.meanMs;
        stats->max_ms = s.maxMs;
        stats->particles_per_s = s.particlesPerS;
        stats->span_s = s.spanS;
    });
}

ao_status ao_serve_reset_stats(ao_server *server)
{
    return guarded([&] {
        if (!server) throw std::invalid_argument("ao_serve_reset_stats: null server");
        server->server->resetStats();
    });
}

ao_status ao_release_cached_memory(void)
{
    return guarded([&] { aot::blockcache::trim(); });
}

ao_status ao_read_particles(const char *path, int layout, double **x, double **y, double **z, size_t *n)
{
    return guarded([&] {
        if (!path || !x || !y || !z || !n) throw std::invalid_argument("ao_read_particles: null argument");
        *x = *y = *z = nullptr;
        *n = 0;
        std::vector<double> vx, vy, vz;
        if (layout == AO_LAYOUT_BINARY_XYZ) aot::io::readBinary(path, vx, vy, vz);
        else if (layout == AO_LAYOUT_CHARGE_XYZ) aot::io::readText(path, 1, vx, vy, vz);
        else if (layout == AO_LAYOUT_XYZ_CHARGE) aot::io::readText(path, 0, vx, vy, vz);
        else throw std::invalid_argument("ao_read_particles: unknown layout");
        const size_t bytes = std::max<size_t>(vx.size(), 1) * sizeof(double);
        double *px = static_cast<double *>(std::malloc(bytes));
        double *py = static_cast<double *>(std::malloc(bytes));
        double *pz = static_cast<double *>(std::malloc(bytes));
        if (!px || !py || !pz)
        {
            std::free(px);
            std::free(py);
            std::free(pz);
            throw std::bad_alloc();
        }
        std::memcpy(px, vx.data(), vx.size() * sizeof(double));
        std::memcpy(py, vy.data(), vy.size() * sizeof(double));
        std::memcpy(pz, vz.data(), vz.size() * sizeof(double));
        *x = px;
        *y = py;
        *z = pz;
        *n = vx.size();
    });
}

ao_status ao_free(void *p)
{
    std::free(p);
    return AO_OK;
}

ao_status ao_read_manifest(const char *path, ao_manifest **out)
{
    return guarded([&] {
        if (!path || !out) throw std::invalid_argument("ao_read_manifest: null argument");
        *out = nullptr;
        auto m = std::make_unique<ao_manifest>();
        m->m = aot::io::readManifest(path);
        *out = m.release();
    });
}

ao_status ao_manifest_info(const ao_manifest *manifest, const char **dataset, size_t *slots, double *box6,
                           size_t *frames)
{
    return guarded([&] {
        if (!manifest) throw std::invalid_argument("ao_manifest_info: null manifest");
        if (dataset) *dataset = manifest->m.dataset.c_str();
        if (slots) *slots = manifest->m.slots;
        if (box6) std::memcpy(box6, manifest->m.box, sizeof(manifest->m.box));
        if (frames) *frames = manifest->m.frames.size();
    });
}

ao_status ao_manifest_frame(const ao_manifest *manifest, size_t i, int *index, long long *id, int *layout,
                            const char **path)
{
    return guarded([&] {
        if (!manifest) throw std::invalid_argument("ao_manifest_frame: null manifest");
        if (i >= manifest->m.frames.size()) throw std::invalid_argument("ao_manifest_frame: no such frame");
        const auto &f = manifest->m.frames[i];
        if (index) *index = f.index;
        if (id) *id = f.id;
        if (layout) *layout = f.layout;
        if (path) *path = f.path.c_str();
    });
}

ao_status ao_manifest_destroy(ao_manifest *manifest)
{
    return guarded([&] { delete manifest; });
}

ao_status ao_sort_pairs_noalloc(const unsigned long long *keys_in, unsigned long long *keys_out,
                                const unsigned *values_in, unsigned *values_out, size_t n, int begin_bit,
                                int end_bit, void *stream)
{
    return guarded([&] {
        aot::sortPairsNoAlloc(keys_in, keys_out, values_in, values_out, n, begin_bit, end_bit,
                              static_cast<cudaStream_t>(stream));
    });
}

ao_status ao_sort_pairs_noalloc_check(size_t n, void *stream)
{
    return guarded([&] {
        if (aot::sortPairsNoAllocFailed(n, static_cast<cudaStream_t>(stream)))
            throw std::runtime_error(
                "ao_sort_pairs_noalloc: a bounded look-back wait gave up; the output is not sorted");
    });
}

}  // extern "C"
