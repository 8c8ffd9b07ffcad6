// keygen.cuh -- particle coordinates -> SFC keys, fused with the sort's digit histogram.
//
// Replaces computeSfcKeysKernel (sfc_keys.cuh:501-532) and
// computeSfcKeysBinaryKernel (kdtree3d_rebalance.cuh:247-273).  Each CTA
// streams coordinates with 128-bit loads (4 floats or 2 doubles per axis per
// thread step), writes the keys with 128-bit stores and accumulates the digit
// counts of all eight radix passes in shared memory, so the sort never
// re-reads the keys for its histogram.  The identity permutation is not
// written: the first sort pass generates it from the input index.
#pragma once

#include "radix_sort.cuh"
#include "sfc.cuh"

namespace aot
{
enum class Curve : int { Morton = 0, Hilbert = 1, Binary = 2 };

template <class Real>
struct KeygenParams
{
    QuantBox<Real> q;
    BinaryGeometry g;
    HilbertTables h;
};

// sPair: the two-level Hilbert table (hilbertPairEntry) in shared memory.
template <class Real, Curve C>
__device__ __forceinline__ u64 particleKey(Real x, Real y, Real z, const KeygenParams<Real> &p,
                                           const unsigned short *sPair)
{
    if constexpr (C == Curve::Binary)
    {
        return binaryKey<Real>(x, y, z, p.g);
    }
    else
    {
        if (isEscaped<Real>(x, y, z)) return kInvalidKey;
        const u32 ix = quantise(x, p.q.xmin, p.q.ilx, p.q.bx);
        const u32 iy = quantise(y, p.q.ymin, p.q.ily, p.q.by);
        const u32 iz = quantise(z, p.q.zmin, p.q.ilz, p.q.bz);
        if constexpr (C == Curve::Hilbert) return hilbertKeyPairs(ix, iy, iz, sPair);
        else return mortonKey(ix, iy, iz);
    }
}

constexpr int kKeygenThreads = 256;

// Vec: particles per thread step (4 for float4, 2 for double2, 1 scalar).
template <class Real, Curve C, int Vec>
static __global__ void __launch_bounds__(kKeygenThreads)
    keygenKernel(const Real *__restrict__ x, const Real *__restrict__ y, const Real *__restrict__ z, size_t n,
                 const KeygenParams<Real> prm, u64 *__restrict__ keys, u32 *__restrict__ hist, int histPasses)
{
    __shared__ u32 sh[sort::kMaxPasses][sort::kRadix];
    __shared__ unsigned short sPair[C == Curve::Hilbert ? kHilbertPairEntries : 1];
    for (int i = threadIdx.x; i < sort::kMaxPasses * sort::kRadix; i += blockDim.x) (&sh[0][0])[i] = 0;
    if constexpr (C == Curve::Hilbert)
    {
        // the one-level tables staged in shared memory, then the pair table from them
        __shared__ unsigned char sEnc[48 * 8], sNext[48 * 8];
        for (int i = threadIdx.x; i < 48 * 8; i += blockDim.x)
        {
            sEnc[i] = prm.h.enc[i];
            sNext[i] = prm.h.encNext[i];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kHilbertPairEntries; i += blockDim.x)
            sPair[i] = hilbertPairEntry(i, sEnc, sNext);
    }
    __syncthreads();

    auto count = [&](u64 k) {
#pragma unroll
        for (int p = 0; p < sort::kMaxPasses; ++p)
            if (p < histPasses) atomicAdd(&sh[p][(k >> (p * sort::kRadixBits)) & (sort::kRadix - 1)], 1u);
    };

    const size_t groups = n / Vec;
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t gi = blockIdx.x * size_t(blockDim.x) + threadIdx.x; gi < groups; gi += stride)
    {
        const size_t base = gi * Vec;
        Real vx[Vec], vy[Vec], vz[Vec];
        if constexpr (Vec == 4)
        {
            const float4 a = __ldcs(reinterpret_cast<const float4 *>(x) + gi);
            const float4 b = __ldcs(reinterpret_cast<const float4 *>(y) + gi);
            const float4 c = __ldcs(reinterpret_cast<const float4 *>(z) + gi);
            vx[0] = a.x; vx[1] = a.y; vx[2] = a.z; vx[3] = a.w;
            vy[0] = b.x; vy[1] = b.y; vy[2] = b.z; vy[3] = b.w;
            vz[0] = c.x; vz[1] = c.y; vz[2] = c.z; vz[3] = c.w;
        }
        else if constexpr (Vec == 2)
        {
            const double2 a = __ldcs(reinterpret_cast<const double2 *>(x) + gi);
            const double2 b = __ldcs(reinterpret_cast<const double2 *>(y) + gi);
            const double2 c = __ldcs(reinterpret_cast<const double2 *>(z) + gi);
            vx[0] = a.x; vx[1] = a.y;
            vy[0] = b.x; vy[1] = b.y;
            vz[0] = c.x; vz[1] = c.y;
        }
        else
        {
            vx[0] = x[base];
            vy[0] = y[base];
            vz[0] = z[base];
        }
        u64 k[Vec];
#pragma unroll
        for (int j = 0; j < Vec; ++j)
        {
            k[j] = particleKey<Real, C>(vx[j], vy[j], vz[j], prm, sPair);
            count(k[j]);
        }
        if constexpr (Vec == 4)
        {
            ulonglong2 *o = reinterpret_cast<ulonglong2 *>(keys + base);
            o[0] = make_ulonglong2(k[0], k[1]);  // default policy: the sort reads the keys next
            o[1] = make_ulonglong2(k[2], k[3]);
        }
        else if constexpr (Vec == 2)
        {
            *reinterpret_cast<ulonglong2 *>(keys + base) = make_ulonglong2(k[0], k[1]);
        }
        else
        {
            keys[base] = k[0];
        }
    }
    // tail particles that do not fill a vector
    for (size_t i = groups * Vec + blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += stride)
    {
        const u64 k = particleKey<Real, C>(x[i], y[i], z[i], prm, sPair);
        keys[i] = k;
        count(k);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < histPasses * sort::kRadix; i += blockDim.x)
    {
        const u32 v = (&sh[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

}  // namespace aot
