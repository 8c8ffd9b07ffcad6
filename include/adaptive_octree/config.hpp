// config.hpp -- public types, configuration and macros of the B200 adaptive-tree engine.
//
// Mirrors the public surface of nrottstegge/Adaptive_Trees
// (include/adaptive_octree/config.hpp:14-180): the same macros, type aliases,
// sentinels, enums, defaults, Box, ViewConfig and the per-backend configs.
// Differences at this boundary:
//   * device buffers are returned as const adaptive_octree::DeviceVector<T>&
//     (engine-owned storage with size/capacity/empty/data and conversions to
//     host and device containers such as thrust::host_vector<T> and
//     thrust::device_vector<T>), not as const thrust::device_vector<T>&;
//   * CUDA failures inside the library throw adaptive_octree::CudaError
//     instead of exiting the process (the reference's library code calls
//     std::exit through checkGpuErrors).  The checkGpuErrors macro itself
//     keeps its meaning for callers' code: report and exit.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include <cuda_runtime_api.h>

#if defined(__CUDACC__)
#define AO_HOST_DEVICE __host__ __device__
#else
#define AO_HOST_DEVICE
#endif

// The reference's public macros (config.hpp:14-33), for callers' code.
#ifndef HOST_DEVICE_FUN
#define HOST_DEVICE_FUN AO_HOST_DEVICE
#endif

// NVTX ranges around callers' phases when ADAPTIVE_OCTREE_PROFILING is
// defined; no-ops otherwise.
#ifdef ADAPTIVE_OCTREE_PROFILING
#include <nvtx3/nvToolsExt.h>
#define ADAPTIVE_OCTREE_NVTX_RANGE_PUSH(name) nvtxRangePushA(name)
#define ADAPTIVE_OCTREE_NVTX_RANGE_POP() nvtxRangePop()
#else
#define ADAPTIVE_OCTREE_NVTX_RANGE_PUSH(name) ((void)0)
#define ADAPTIVE_OCTREE_NVTX_RANGE_POP() ((void)0)
#endif

// checkGpuErrors(call): on failure prints the call, file and line and exits.
// ADAPTIVE_OCTREE_CHECK_CUDA(call): on failure throws std::runtime_error.
#define checkGpuErrors(errcode) ::adaptive_octree::detail::checkErr((errcode), __FILE__, __LINE__, #errcode)
#define ADAPTIVE_OCTREE_CHECK_CUDA(operation) ::adaptive_octree::detail::checkCudaResult((operation), #operation)

// Symbols of the C++ classes exported by the shared library.
#if defined(__GNUC__)
#define AO_CXX_API __attribute__((visibility("default")))
#else
#define AO_CXX_API
#endif

namespace adaptive_octree
{
using KeyType = unsigned long long;
using NodeIndex = int;
using PermIndex = std::uint32_t;

inline constexpr NodeIndex invalidNodeIndex = -1;
inline constexpr KeyType invalidParticleKey = std::numeric_limits<KeyType>::max();
inline constexpr KeyType invalidParticleNodeIndex = static_cast<KeyType>(invalidNodeIndex);
inline constexpr unsigned maxOctreeDepth = std::numeric_limits<KeyType>::digits / 3;
inline constexpr unsigned maxBinaryDepth = std::numeric_limits<KeyType>::digits - 1;
inline constexpr KeyType maxKey = KeyType(1) << maxBinaryDepth;

enum class TreeType { Octree, Binary };
enum class SplitCriterion { LeafCount, NFCount };
enum class SfcKind { Morton, Hilbert };

namespace defaults
{
inline constexpr unsigned maxParticlesPerLeaf = 64;
inline constexpr unsigned octreeUpdateIterations = 2;
inline constexpr unsigned binaryUpdateIterations = 6;
inline constexpr unsigned long long nearFieldLimit = 1ULL * maxParticlesPerLeaf * maxParticlesPerLeaf * 27;
inline constexpr std::uint64_t mergeBufferRatio = 1;
inline constexpr std::uint64_t splitBufferRatio = 1;
// Capacity growth adds 1/bufferGrowthDivisor (25%).
inline constexpr std::size_t bufferGrowthDivisor = 4;
}  // namespace defaults

template <class Real>
struct Box
{
    Real xmin = Real{0}, xmax = Real{1};
    Real ymin = Real{0}, ymax = Real{1};
    Real zmin = Real{0}, zmax = Real{1};
};

// Escaped particles keep their input slot and sort after the active keys.
template <class Real>
inline constexpr Real escapedParticleCoordinate = std::numeric_limits<Real>::max();

template <class Real>
AO_HOST_DEVICE constexpr bool isEscapedParticle(Real x, Real y, Real z)
{
    return x == escapedParticleCoordinate<Real> && y == escapedParticleCoordinate<Real> &&
           z == escapedParticleCoordinate<Real>;
}

struct ViewConfig
{
    bool treeStructure = false;
    bool particleCountsPerBox = false;
    bool particleMapping = false;
};

template <class Real>
struct OctreeConfig
{
    unsigned maxDepth = maxOctreeDepth;  // build iteration limit, as in the reference
    unsigned maxParticlesPerLeaf = defaults::maxParticlesPerLeaf;
    SplitCriterion splitCriterion = SplitCriterion::LeafCount;
    SfcKind sfcKind = SfcKind::Morton;
    Box<Real> box{};
    ViewConfig views{};
    unsigned updateIterations = defaults::octreeUpdateIterations;
    cudaStream_t stream = nullptr;
    // The reference prompts on stdin when this is true; this engine never
    // reads stdin and accepts the field only for source compatibility.
    bool interactive = false;
};

template <class Real>
struct KDTree3DConfig
{
    unsigned maxDepth = maxBinaryDepth;
    unsigned maxParticlesPerLeaf = defaults::maxParticlesPerLeaf;
    Box<Real> box{};
    ViewConfig views{};
    unsigned updateIterations = defaults::binaryUpdateIterations;
    cudaStream_t stream = nullptr;
};

template <class Real>
struct TreeConfig
{
    // -1 uses the backend default; explicit depth zero is valid.
    int maxDepth = -1;
    unsigned maxParticlesPerLeaf = defaults::maxParticlesPerLeaf;
    int updateIterations = -1;
    Box<Real> box{};
    cudaStream_t stream = nullptr;
    SplitCriterion splitCriterion = SplitCriterion::LeafCount;
    // NFCount and Hilbert are available only in Octree mode.
    SfcKind sfcKind = SfcKind::Morton;
    ViewConfig views{};
};

// A CUDA runtime failure inside the engine.
class CudaError : public std::runtime_error
{
public:
    CudaError(int code, const std::string &what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

namespace detail
{
inline void checkErr(cudaError_t error, const char *file, int line, const char *expression)
{
    if (error == cudaSuccess) return;
    std::fprintf(stderr, "CUDA error: %s failed at %s:%d with %s (%s)\n", expression, file, line,
                 cudaGetErrorName(error), cudaGetErrorString(error));
    std::exit(EXIT_FAILURE);
}

inline void checkCudaResult(cudaError_t error, const char *operation)
{
    if (error != cudaSuccess) throw std::runtime_error(std::string(operation) + ": " + cudaGetErrorString(error));
}

// A host container of T with contiguous storage: value_type T, resize(n),
// data() -> T* (std::vector<T>, thrust::host_vector<T>).
template <class C, class T, class = void>
struct IsHostContainer : std::false_type
{
};
template <class C, class T>
struct IsHostContainer<C, T,
                       std::void_t<typename C::value_type, decltype(std::declval<C &>().resize(std::size_t(0))),
                                   decltype(std::declval<C &>().data())>>
    : std::bool_constant<std::is_same_v<typename C::value_type, T> &&
                         std::is_same_v<decltype(std::declval<C &>().data()), T *>>
{
};

// A device container of T whose data() is a fancy pointer with get() -> T*
// (thrust::device_vector<T>); constructible with a size.
template <class C, class T, class = void>
struct IsDeviceContainer : std::false_type
{
};
template <class C, class T>
struct IsDeviceContainer<C, T, std::void_t<typename C::value_type, decltype(std::declval<C &>().data().get())>>
    : std::bool_constant<std::is_same_v<typename C::value_type, T> &&
                         std::is_same_v<decltype(std::declval<C &>().data().get()), T *> &&
                         std::is_constructible_v<C, std::size_t>>
{
};

inline void copyOrThrow(void *dst, const void *src, std::size_t bytes, cudaMemcpyKind kind)
{
    if (!bytes) return;
    const cudaError_t e = cudaMemcpy(dst, src, bytes, kind);
    if (e != cudaSuccess) throw CudaError(int(e), std::string("DeviceVector copy: ") + cudaGetErrorString(e));
}
}  // namespace detail

// An engine-owned device array as the getters return it.  size() is the
// logical length reported by the last host synchronisation (build() or
// doBuffersNeedResize()), capacity() the allocation; data() is a device
// pointer that stays valid until the next build() or resizeBuffers() (so
// thrust::raw_pointer_cast(tree.perm_d().data()) works as with the
// reference).  Like the reference's const thrust::device_vector<T>&, a getter
// returns a reference to storage held by the tree; the tree refreshes it at
// each getter call, so reacquire it after update().
//
// Copies (all synchronous, cudaMemcpy on the legacy stream):
//   thrust::host_vector<T> h = tree.particleKeys_d();   // or std::vector<T>
//   thrust::device_vector<T> d = tree.particleKeys_d(); // a device copy
// so callers written against the reference's getters, which assign them to
// host vectors (tests/tree_test.cu:313-317), compile unchanged.
template <class T>
class DeviceVector
{
public:
    using value_type = T;
    using size_type = std::size_t;
    DeviceVector() = default;
    DeviceVector(const T *data, std::size_t size, std::size_t capacity) : data_(data), size_(size), cap_(capacity) {}
    const T *data() const { return data_; }
    std::size_t size() const { return size_; }
    std::size_t capacity() const { return cap_; }
    bool empty() const { return size_ == 0; }

    std::vector<T> to_host() const
    {
        std::vector<T> out(size_);
        detail::copyOrThrow(out.data(), data_, size_ * sizeof(T), cudaMemcpyDeviceToHost);
        return out;
    }
    template <class C, std::enable_if_t<detail::IsHostContainer<C, T>::value, int> = 0>
    operator C() const
    {
        C out;
        out.resize(size_);
        detail::copyOrThrow(out.data(), data_, size_ * sizeof(T), cudaMemcpyDeviceToHost);
        return out;
    }
    template <class C, std::enable_if_t<detail::IsDeviceContainer<C, T>::value, long> = 0>
    operator C() const
    {
        C out(size_);
        detail::copyOrThrow(out.data().get(), data_, size_ * sizeof(T), cudaMemcpyDeviceToDevice);
        return out;
    }

private:
    const T *data_ = nullptr;
    std::size_t size_ = 0, cap_ = 0;
};

// The arrays a tree's getters return references to.
struct GetterViews
{
    DeviceVector<KeyType> particleKeys, cornerstone, sfcBoxIndex, sfcParticleIndex;
    DeviceVector<PermIndex> perm;
    DeviceVector<unsigned> leafCounts, nearFieldCounts, particleBeginIndex, particleCounts;
    DeviceVector<std::uint8_t> hasBoxSplit, boxDepth;
    DeviceVector<NodeIndex> parentIndex, childIndex, levelOffset;
};
}  // namespace adaptive_octree
