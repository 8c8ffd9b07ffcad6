// forest_sort.cuh -- the segmented sort of every system of a forest in one
// persistent (cooperative) launch.
//
// After the keys and their digit histograms (keygenKernel, a launch of its
// own at full occupancy), the phases of the launch-per-stage path
// (binsKernel, one segmentOnesweepKernel per pass, activeKernel), separated
// by grid barriers instead of launch boundaries:
//   bins       per system (one CTA each) and pass, the global start of each
//              digit;
//   passes     the 8 onesweep passes; in each, CTAs take tiles from the pass's
//              counter until it runs out.  A tile's look-back waits only for
//              tiles taken before it, by CTAs that are resident and do not
//              wait for later tiles, so every wait ends;
//   active     each system's active count (escaped keys sort last) and the
//              key sample of a build by levels.
// Only the 8-bit configurations (key generation counts their digits) run here.
#pragma once

#include <utility>

#include "forest.cuh"
#include "grid_barrier.cuh"

namespace aot
{
namespace forest
{
struct SortArgs
{
    Bufs f;                   // systems, per-system state, sorted keys (f.P = keys[0])
    sort::SegmentTiles tiles; // the tile table (bins set per pass)
    u32 numTiles;
    u64 *keys[2];
    u32 *vals[2];
    u32 *hist;                // [system][pass slot][digit], zero on entry
    u32 *bins;                // [pass][system][digit]
    u32 *tileCounters;        // [pass], zero on entry
    u64 *status;              // [pass][tile][digit], zero on entry
    int *error;               // bounded look-back gave up
    u64 *sample;              // every 32nd sorted key (nullptr: none)
    size_t ns;
    GridBarrier *bar;
};

// A barrier gave up: the forest's error word tells the host (the keys are
// not sorted, and what follows on the stream leaves them alone).
__device__ __forceinline__ void fail(const SortArgs &p)
{
    if (threadIdx.x == 0) atomicExch(p.error, kErrLookback);
}

// Pass Q of the sort: every buffer and shift a compile-time choice among the
// kernel's parameters, so that nothing of it has to stay in registers.
template <int Items, int Q>
__device__ __forceinline__ void sortPass(const SortArgs &p)
{
    constexpr int shift = Q * sort::kRadixBits;
    constexpr int bits = 64 - shift < sort::kRadixBits ? 64 - shift : sort::kRadixBits;
    while (sort::onesweepTile<8, Items>(
        sort::SegmentTiles{p.tiles.tileSeg, p.tiles.tileBegin, p.tiles.tileEnd, p.tiles.segFirstTile, p.tiles.segBase,
                           p.bins + size_t(Q) * p.f.numSystems * sort::kRadix},
        p.keys[Q & 1], Q == 0 ? nullptr : p.vals[Q & 1], p.keys[(Q & 1) ^ 1], p.vals[(Q & 1) ^ 1], shift,
        p.tileCounters + Q, p.status + size_t(Q) * p.numTiles * sort::kRadix, p.error, bits, sort::kLookbackSpins,
        p.numTiles))
        __syncthreads();
}

template <int Items, int... Q>
__device__ __forceinline__ bool sortPasses(const SortArgs &p, std::integer_sequence<int, Q...>)
{
    // each pass, then a barrier; stop at the first barrier that gives up
    return ((sortPass<Items, Q>(p), gridBarrier(p.bar)) && ...);
}

// Three CTAs per SM: the registers of the pass loop fit without spills.
template <int Items>
static __global__ void __launch_bounds__(sort::kThreads, 3) sortKernel(SortArgs p)
{
    static_assert(sort::kThreads == sort::kRadix, "one digit per thread in the bins phase");
    extern __shared__ __align__(16) unsigned char smemRaw[];
    u32 *sh = reinterpret_cast<u32 *>(smemRaw);
    for (int sys = blockIdx.x; sys < p.f.numSystems; sys += gridDim.x)
        systemBins(p.f.systems, p.f.numSystems, sys, p.hist, p.bins, sort::kMaxPasses, sh);
    if (!gridBarrier(p.bar)) return fail(p);
    if (!sortPasses<Items>(p, std::make_integer_sequence<int, sort::kMaxPasses>{})) return fail(p);
    activeAndSample(p.f, p.sample, p.ns, size_t(blockIdx.x) * blockDim.x + threadIdx.x,
                    size_t(gridDim.x) * blockDim.x);
}

}  // namespace forest
}  // namespace aot
