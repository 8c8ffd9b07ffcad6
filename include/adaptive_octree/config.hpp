// config.hpp -- public types and configuration of the B200 adaptive-tree engine.
//
// Mirrors the public surface of nrottstegge/Adaptive_Trees
// (include/adaptive_octree/config.hpp:36-160): the same type aliases,
// sentinels, enums, defaults, Box, ViewConfig and the per-backend configs.
// Differences at this boundary:
//   * device buffers are returned as adaptive_octree::DeviceVector<T> (a
//     read-only view: data/size/capacity/empty/to_host), not as
//     thrust::device_vector<T>;
//   * CUDA failures throw adaptive_octree::CudaError instead of exiting the
//     process (config.hpp:164-172 of the reference calls std::exit).
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime_api.h>

#if defined(__CUDACC__)
#define AO_HOST_DEVICE __host__ __device__
#else
#define AO_HOST_DEVICE
#endif

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

// Read-only view of an engine-owned device array.  size() is the logical
// length reported by the last host synchronisation (build() or
// doBuffersNeedResize()), capacity() the allocation; data() is a device
// pointer that stays valid until the next build() or resizeBuffers().
template <class T>
class DeviceVector
{
public:
    using value_type = T;
    DeviceVector() = default;
    DeviceVector(const T *data, std::size_t size, std::size_t capacity) : data_(data), size_(size), cap_(capacity) {}
    const T *data() const { return data_; }
    std::size_t size() const { return size_; }
    std::size_t capacity() const { return cap_; }
    bool empty() const { return size_ == 0; }
    // Synchronous copy to the host (cudaMemcpy on the legacy stream).
    std::vector<T> to_host() const
    {
        std::vector<T> out(size_);
        if (size_)
        {
            const cudaError_t e = cudaMemcpy(out.data(), data_, size_ * sizeof(T), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) throw CudaError(int(e), cudaGetErrorString(e));
        }
        return out;
    }

private:
    const T *data_ = nullptr;
    std::size_t size_ = 0, cap_ = 0;
};
}  // namespace adaptive_octree
