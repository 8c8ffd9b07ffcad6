// common.cuh -- shared device/host definitions of the B200 adaptive-tree engine.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "adaptive_octree/config.hpp"
#include "engine.hpp"

namespace aot
{
using u8 = std::uint8_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;
using i64 = std::int64_t;

using adaptive_octree::KeyType;
using adaptive_octree::NodeIndex;

constexpr unsigned kOctLevels = 21;        // 3 x 21 = 63 key bits (sfc_keys.cuh:33-36)
constexpr unsigned kBinDepth = 63;         // maxBinaryDepth (config.hpp:47)
constexpr u64 kMaxKey = u64(1) << 63;      // root exclusive end (config.hpp:48)
constexpr u64 kInvalidKey = ~u64(0);       // escaped particle key (config.hpp:43)

// Device-resident tree state.  The first eight fields keep the layout of the
// reference's RebalanceState (helpers.cuh:109-120) so numLeaves_d(),
// numNodes_d() and numActiveParticles_d() point at the same members.
struct DeviceState
{
    int changed;
    int converged;
    int numLeaves;
    int newNumLeaves;
    int needsResize;
    int numNodes;
    int activeBuffer;
    unsigned numActiveParticles;
    // engine-private
    int overflow;        // physical buffer too small for a build proposal
    int error;           // a bounded device wait gave up (see kErrLookback)
    int iteration;       // build rounds that changed the tree
    int dirtyCount;      // dirty-leaf list length of the last materialisation
    int updatePasses;    // update passes that changed the tree since the last update() began
    int doneBlocks;      // completion counter of the scatter kernel
    int rounds;          // build rounds completed (changed or found converged)
    int pad;
    long long proposal;  // leaf count proposed by the last decision scan
    long long logicalCap;  // binary build: the reference's leafCapacity
};

// Pass modes of the scatter/commit kernels.
constexpr int kModeUpdate = 0;       // reference graph pass: exceeding leafCapacity sets needsResize
constexpr int kModeOctreeBuild = 1;  // build: buffers grow on the host, exceeding them is an overflow
constexpr int kModeBinaryBuild = 2;  // build: leafCapacity grows by 25% steps until the proposal fits

constexpr int kErrLookback = 1;


inline unsigned ceilDiv(size_t n, unsigned b) { return unsigned((n + b - 1) / b); }

// --------------------------------------------------------------------------
// integer helpers
// --------------------------------------------------------------------------
__host__ __device__ inline int clz64(u64 x)
{
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return x ? __builtin_clzll(x) : 64;
#endif
}
// octree node key range at a level (nodeRange, sfc_keys.cuh:92-97)
__host__ __device__ inline u64 octRange(unsigned level) { return u64(1) << (3u * (kOctLevels - level)); }
// octree level of a power-of-8 range (treeLevel, sfc_keys.cuh:100-104)
__host__ __device__ inline unsigned octLevel(u64 range) { return unsigned(clz64(range - 1) - 1) / 3u; }
// octal digit of a key at a level (octalDigit, sfc_keys.cuh:108-112)
__host__ __device__ inline unsigned octDigit(u64 key, unsigned level)
{
    return unsigned(key >> (3u * (kOctLevels - level))) & 7u;
}

// First index in a[0, n) whose key is >= v (lowerBound, helpers.cuh:65-85).
// Branch-free halving; `a` is read through the read-only path.
__device__ __forceinline__ size_t lowerBoundDev(const u64 *__restrict__ a, size_t n, u64 v)
{
    size_t lo = 0;
    while (n > 0)
    {
        const size_t half = n >> 1;
        const u64 m = __ldg(a + lo + half);
        const bool less = m < v;
        lo = less ? lo + half + 1 : lo;
        n = less ? n - half - 1 : half;
    }
    return lo;
}

// First index in a[0, n) whose key is > v (upperBound, helpers.cuh:87-107).
__device__ __forceinline__ size_t upperBoundDev(const u64 *__restrict__ a, size_t n, u64 v)
{
    size_t lo = 0;
    while (n > 0)
    {
        const size_t half = n >> 1;
        const u64 m = __ldg(a + lo + half);
        const bool le = !(v < m);
        lo = le ? lo + half + 1 : lo;
        n = le ? n - half - 1 : half;
    }
    return lo;
}

// First index in a[0, n) whose key is >= v, 32-bit index arithmetic.
__device__ __forceinline__ u32 lowerBound32(const u64 *__restrict__ a, u32 n, u64 v)
{
    u32 lo = 0;
    while (n > 0)
    {
        const u32 half = n >> 1;
        const bool less = __ldg(a + lo + half) < v;
        lo = less ? lo + half + 1 : lo;
        n = less ? n - half - 1 : half;
    }
    return lo;
}

// Sorted-key search accelerated by a sampled index.  `sample[j]` holds
// keys[j * kSampleStride]; the search first narrows to one stride window with
// the sample (small, L2-resident) and then searches that window of the keys.
// Key counts are below 2^32 (32-bit permutation), so indices are 32-bit.
constexpr unsigned kSampleShift = 5;
constexpr unsigned kSampleStride = 1u << kSampleShift;

// Lower bound of t in the sorted A[b, e) by a whole warp: each step probes 32
// points that split the range into 33 parts and keeps the part the ballot
// points to, so a range of n keys takes about log33(n) dependent loads
// instead of log2(n).  Every lane returns the answer.
__device__ __forceinline__ u32 warpLowerBound(const u64 *A, u32 b, u32 e, u64 t, int lane)
{
    while (e > b)
    {
        const u32 n = e - b;
        const u32 p = b + u32((u64(lane) + 1) * n / 33u);  // p < e; p_k = b + k when n <= 32
        const unsigned below = __ballot_sync(0xffffffffu, __ldg(A + p) < t);
        const int c = __popc(below);  // a prefix of the lanes: A is sorted
        const u32 pLow = __shfl_sync(0xffffffffu, p, c > 0 ? c - 1 : 0);
        const u32 pHigh = __shfl_sync(0xffffffffu, p, c < 32 ? c : 31);
        if (c > 0) b = pLow + 1;
        if (c < 32) e = pHigh;
    }
    return b;
}

struct KeyIndex
{
    const u64 *keys;
    const u64 *sample;
    size_t n;        // keys
    size_t ns;       // samples = ceil(n / stride)

    // lowerBound(keys, n, v)
    __device__ __forceinline__ u32 lower(u64 v) const
    {
        if (n == 0) return 0;
        // first sample >= v; the answer lies in the window before it
        const u32 s = lowerBound32(sample, u32(ns), v);
        if (s == 0) return 0;
        const u32 base = (s - 1) << kSampleShift;
        u32 len = u32(n) - base;
        if (len > kSampleStride) len = kSampleStride;
        return base + lowerBound32(keys + base, len, v);
    }

    // lowerBound(keys, n, v) for a target expected near index `hint`:
    // gallop up to Probes probes each way from the hint (a window of
    // 2^Probes - 1 keys), then fall back to lower().
    template <int Probes = 4>
    __device__ __forceinline__ u32 lowerNear(u32 hint, u64 v) const
    {
        const u32 m = u32(n);
        if (hint < m && __ldg(keys + hint) < v)
        {
            u32 base = hint, step = 1;  // keys[base] < v
#pragma unroll
            for (int k = 0; k < Probes; ++k)
            {
                const u32 probe = base + step;
                if (probe >= m || __ldg(keys + probe) >= v)
                {
                    const u32 end = probe < m ? probe : m;
                    return base + 1 + lowerBound32(keys + base + 1, end - base - 1, v);
                }
                base = probe;
                step <<= 1;
            }
            return lower(v);
        }
        u32 top = hint < m ? hint : m, step = 1;  // answer <= top
#pragma unroll
        for (int k = 0; k < Probes; ++k)
        {
            if (top < step) return lowerBound32(keys, top, v);
            const u32 probe = top - step;
            if (__ldg(keys + probe) < v) return probe + 1 + lowerBound32(keys + probe + 1, top - probe - 1, v);
            top = probe;
            step <<= 1;
        }
        return lower(v);
    }
    // number of keys in [a, b)
    __device__ __forceinline__ unsigned count(u64 a, u64 b) const { return lower(b) - lower(a); }
};

}  // namespace aot
