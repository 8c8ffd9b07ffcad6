// radix_sort.cuh -- onesweep LSD radix sort of 64-bit keys carrying 32-bit values.
//
// Replaces cub::DeviceRadixSort::SortPairs on the particle keys
// (octree.cu:301-304, kdtree3d.cu:168-170) and on the view's internal-node keys
// (tree_view.cu:664-689).  Stable: equal keys keep their input order, which
// for the particle sort makes Perm ascend within runs of equal keys.
//
// Structure (one read of the keys per digit):
//   1. a histogram kernel counts all digit positions at once (fused into key
//      generation for the particle sort with 8-bit digits, so the keys are
//      never re-read);
//   2. a tiny kernel turns the counts into per-digit global start offsets;
//   3. one onesweep kernel per digit: each CTA takes a tile of keys in
//      arrival order (atomic tile counter), ranks them per warp with ballots,
//      publishes its per-digit counts, resolves its global offsets by
//      decoupled look-back over earlier tiles, reorders the tile in shared
//      memory and writes digit runs out contiguously.
// The digit width and the keys per thread are template parameters; the
// configurations compiled in are listed in kSortConfigs, and the sort tuner
// (sortTune in engine.cu) picks one per device and problem size by timing them.
// The look-back wait is bounded: after kLookbackSpins polls it records
// kErrLookback in the device error word and proceeds, so a broken invariant
// surfaces as an error status instead of a hung GPU.
#pragma once

#include "common.cuh"

namespace aot
{
namespace sort
{
constexpr int kRadixBits = 8;              // digit width of the default configuration
constexpr int kRadix = 1 << kRadixBits;     // largest radix: stride of every per-pass digit array
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 10;                  // keys per thread of the default configuration
constexpr int kTile = kThreads * kItems;
constexpr int kMaxPasses = 8;               // passes of 8-bit digits over 64-bit keys
constexpr int kPassSlots = 10;              // most passes of any configuration (7-bit digits)
constexpr int kMinTile = kThreads * 8;      // smallest tile of any configuration
constexpr u64 kFlagAgg = u64(1) << 62;
constexpr u64 kFlagPrefix = u64(2) << 62;
constexpr u64 kValueMask = (u64(1) << 62) - 1;
constexpr unsigned kLookbackSpins = 1u << 22;
constexpr int kLookbackWindow = 8;

__device__ __forceinline__ u64 ldRelaxed(const u64 *p)
{
    u64 v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void stRelaxed(u64 *p, u64 v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned laneMaskLt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Per-sort scratch laid out by the host (see SortScratch):
//   hist[kMaxPasses][256] u32 counts, bins[kMaxPasses][256] u32 exclusive
//   starts, tileCounters[kMaxPasses] u32, status[kMaxPasses][tiles][256] u64.
struct Scratch
{
    u32 *hist;
    u32 *bins;
    u32 *tileCounters;
    u64 *status;
    int *error;
    size_t tiles;
};

// Histogram of the Bits-wide digits of keys[0, n) for passes covering
// [beginBit, endBit); pass p's counts go to hist[p * kRadix + digit].
template <int Bits = kRadixBits>
static __global__ void __launch_bounds__(kThreads) histogramKernel(const u64 *__restrict__ keys, size_t n, int beginBit,
                                                             int passes, u32 *__restrict__ hist, int endBit = 64)
{
    constexpr int R = 1 << Bits;
    __shared__ u32 sh[kPassSlots][R];
    for (int i = threadIdx.x; i < kPassSlots * R; i += kThreads) (&sh[0][0])[i] = 0;
    __syncthreads();
    for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n; i += size_t(gridDim.x) * kThreads)
    {
        const u64 k = __ldg(keys + i);
        for (int p = 0; p < passes; ++p)
        {
            const int shift = beginBit + p * Bits;
            const int bits = endBit - shift < Bits ? endBit - shift : Bits;
            atomicAdd(&sh[p][(k >> shift) & ((1u << bits) - 1)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * R; i += kThreads)
    {
        const u32 v = (&sh[0][0])[i];
        if (v) atomicAdd(hist + (i / R) * kRadix + (i % R), v);
    }
}

// Exclusive scan of each pass' 256 digit counts (a narrower radix leaves the
// upper counts zero, so their starts are unused).
static __global__ void __launch_bounds__(kRadix) binsKernel(const u32 *__restrict__ hist, u32 *__restrict__ bins, int passes)
{
    __shared__ u32 s[kRadix];
    const int d = threadIdx.x;
    for (int p = 0; p < passes; ++p)
    {
        const u32 v = hist[p * kRadix + d];
        s[d] = v;
        __syncthreads();
        // Hillis-Steele inclusive scan over 256 entries
        for (int off = 1; off < kRadix; off <<= 1)
        {
            const u32 t = d >= off ? s[d - off] : 0u;
            __syncthreads();
            s[d] += t;
            __syncthreads();
        }
        bins[p * kRadix + d] = s[d] - v;
        __syncthreads();
    }
}

template <int Bits, int Items>
struct SharedPass
{
    static constexpr int R = 1 << Bits;
    static constexpr int T = kThreads * Items;
    u64 keys[T];
    u32 vals[T];
    u32 stage[T];              // the tile's input values, staged by one bulk copy (16-byte aligned)
    u64 valuesReady;           // mbarrier of that copy
    u32 staged;                // values in `stage` (a multiple of 4)
    u32 warpHist[kWarps][R];   // per-warp digit counts, then exclusive warp offsets
    u32 localStart[R];
    u32 gstart[R];             // global position of local index 0 of each digit (mod 2^32)
    u32 count[R];
    u32 warpSums[kWarps];
    u32 tile;
};

// The compiled configurations: digit width, keys per thread and the CTAs per
// SM they are built for (their shared memory and a 64-register budget allow
// 4 CTAs for tiles of up to 3072 keys).  Each gives an even number of passes
// over 64-bit keys (8 or 10), so the sorted data ends where it started.
struct SortConfig
{
    int bits, items;
};
constexpr SortConfig kSortConfigs[] = {{8, 10}, {8, 16}, {8, 8}, {7, 12}, {7, 16}};
constexpr int kNumSortConfigs = int(sizeof(kSortConfigs) / sizeof(kSortConfigs[0]));
constexpr int kDefaultSortConfig = 0;
constexpr int configTile(int c) { return kThreads * kSortConfigs[c].items; }
constexpr int configPasses(int c, int bits = 64)
{
    return (bits + kSortConfigs[c].bits - 1) / kSortConfigs[c].bits;
}

// Lanes of the warp whose (valid) digit equals this lane's: eight ballots, one
// per digit bit, instead of __match_any_sync.
__device__ __forceinline__ unsigned peerLanes(unsigned digit, int bits, unsigned validMask)
{
    unsigned peers = validMask;
#pragma unroll
    for (int b = 0; b < kRadixBits; ++b)
    {
        if (b < bits)
        {
            const bool set = (digit >> b) & 1u;
            const unsigned m = __ballot_sync(0xffffffffu, set);
            peers &= set ? m : ~m;
        }
    }
    return peers;
}

// Shared-memory address of a pointer into shared memory.
__device__ __forceinline__ unsigned smemAddr(const void *p) { return unsigned(__cvta_generic_to_shared(p)); }

// mbarrier and bulk-copy helpers (PTX ISA: mbarrier, cp.async.bulk)
__device__ __forceinline__ void mbarInit(u64 *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fenceMbarInit() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbarArriveExpectTx(u64 *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbarArrive(u64 *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(u64 *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Global -> shared copy of `bytes` (a multiple of 16; both addresses 16-byte
// aligned) that completes on `bar`.  No multicast: the source is this GPU's memory.
__device__ __forceinline__ void bulkLoad(void *dst, const void *src, unsigned bytes, u64 *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smemAddr(dst)),
                 "l"(src), "r"(bytes), "r"(smemAddr(bar))
                 : "memory");
}
constexpr unsigned kStageSpins = 1u << 22;  // bounded wait for the staged values

// Tile geometry of a pass over one contiguous key array keys[0, n).  The
// accessors are cheap and recomputed where used, so that nothing extra stays
// live in registers across the pass.
template <int Tile>
struct ContiguousTiles
{
    static constexpr bool kStageValues = true;  // tiles start at multiples of Tile (16-byte aligned values)
    size_t n;
    const u32 *bins;  // [radix] global start of each digit
    // the tile's keys are [base(t), min(base(t) + Tile, end(t)))
    __device__ __forceinline__ size_t base(size_t tile) const { return tile * size_t(Tile); }
    __device__ __forceinline__ size_t end(size_t) const { return n; }
    // the tile publishes an inclusive prefix without look-back
    __device__ __forceinline__ bool chainStart(size_t tile) const { return tile == 0; }
    __device__ __forceinline__ const u32 *digitBase(size_t) const { return bins; }
    // generated first-pass value of the key at global index i: i - valueOffset
    __device__ __forceinline__ u32 valueOffset(size_t) const { return 0; }
};

// Tile geometry of a segmented pass (the systems of a forest): tile t holds
// the keys [tileBegin[t], tileEnd[t]) of segment tileSeg[t] (at most one tile,
// never straddling segments); a look-back chain ends at the segment's first
// tile; digit starts are per segment, and generated values are indices within
// the segment.
struct SegmentTiles
{
    static constexpr bool kStageValues = false;  // tiles start anywhere: plain loads
    const u32 *tileSeg, *tileBegin, *tileEnd, *segFirstTile, *segBase;
    const u32 *bins;  // [segments][kRadix] global start of each digit of this pass
    __device__ __forceinline__ size_t base(size_t tile) const { return tileBegin[tile]; }
    __device__ __forceinline__ size_t end(size_t tile) const { return tileEnd[tile]; }
    __device__ __forceinline__ bool chainStart(size_t tile) const { return u32(tile) == segFirstTile[tileSeg[tile]]; }
    __device__ __forceinline__ const u32 *digitBase(size_t tile) const { return bins + size_t(tileSeg[tile]) * kRadix; }
    __device__ __forceinline__ u32 valueOffset(size_t tile) const { return segBase[tileSeg[tile]]; }
};

// One onesweep pass: the Bits-wide digit at bit `shift` (`bits` <= Bits
// wide) of the tiles of `tiles`, Items keys per thread.  valsIn == nullptr
// means values are generated (first pass).  Threads below the radix own one
// digit each in the per-digit steps.  A look-back that polls an unpublished
// tile more than spinLimit times records kErrLookback and goes on with the
// prefix it has: every write stays inside the output, the result is wrong
// and the host reports the error.  A persistent CTA calls it until it returns
// false: the tile counter has passed numTiles (which a launch of one CTA per
// tile never reaches).  Persistent use needs unstaged values
// (Tiles::kStageValues false): the staging barrier is not set up again.
template <int Bits, int Items, class Tiles>
__device__ __forceinline__ bool onesweepTile(const Tiles &tiles, const u64 *__restrict__ keysIn,
                                             const u32 *__restrict__ valsIn, u64 *__restrict__ keysOut,
                                             u32 *__restrict__ valsOut, int shift, u32 *tileCounter, u64 *status,
                                             int *error, int bits, unsigned spinLimit = kLookbackSpins,
                                             u32 numTiles = 0xffffffffu)
{
    using Smem = SharedPass<Bits, Items>;
    constexpr int R = Smem::R;
    constexpr int T = Smem::T;
    static_assert(R <= kThreads && R <= kRadix, "one digit per thread");
    static_assert(Items % 2 == 0, "ranks are packed in pairs");
    const unsigned dmask = (1u << bits) - 1;
    extern __shared__ __align__(16) unsigned char smemRaw[];
    Smem &sm = *reinterpret_cast<Smem *>(smemRaw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    const bool stage = Tiles::kStageValues && valsIn != nullptr;
    for (int i = tid; i < kWarps * R; i += kThreads) (&sm.warpHist[0][0])[i] = 0;
    if (tid == 0)
    {
        sm.tile = atomicAdd(tileCounter, 1u);
        if (stage)
        {
            mbarInit(&sm.valuesReady, 1);
            fenceMbarInit();
        }
    }
    __syncthreads();
    const size_t tile = sm.tile;
    if (tile >= numTiles) return false;
    const size_t tileBase = tiles.base(tile);
    const size_t warpBase = tileBase + size_t(warp) * (32 * Items);
    if (stage && tid == 0)
    {
        // the values travel to shared memory while the keys are ranked
        const size_t end = tiles.end(tile);
        const u32 count = u32((end - tileBase) < size_t(T) ? end - tileBase : size_t(T));
        const bool aligned = (reinterpret_cast<uintptr_t>(valsIn + tileBase) & 15u) == 0;
        const u32 bulk = aligned ? (count & ~3u) : 0u;
        sm.staged = bulk;
        if (bulk)
        {
            mbarArriveExpectTx(&sm.valuesReady, bulk * 4u);
            bulkLoad(sm.stage, valsIn + tileBase, bulk * 4u, &sm.valuesReady);
        }
        else
        {
            mbarArrive(&sm.valuesReady);
        }
    }

    u64 key[Items];
#pragma unroll
    for (int i = 0; i < Items; ++i)
    {
        const size_t idx = warpBase + size_t(i) * 32 + lane;
        key[i] = idx < tiles.end(tile) ? __ldcs(keysIn + idx) : 0ull;
    }
    // Rank within the warp, items in memory order (item-major, lane-minor):
    // the lowest lane of each digit group adds the group size to the warp's
    // counter and broadcasts the old value.
    u32 *wh = sm.warpHist[warp];
    const unsigned ltMask = laneMaskLt();
    u32 rank2[Items / 2];
#pragma unroll
    for (int i = 0; i < Items; ++i)
    {
        const size_t idx = warpBase + size_t(i) * 32 + lane;
        const bool valid = idx < tiles.end(tile);
        const unsigned validMask = __ballot_sync(0xffffffffu, valid);
        const unsigned d = unsigned(key[i] >> shift) & dmask;
        const unsigned peers = peerLanes(d, bits, validMask);
        const int leader = __ffs(peers) - 1;
        u32 base = 0;
        if (valid && lane == leader) base = atomicAdd(&wh[d], u32(__popc(peers)));
        base = __shfl_sync(0xffffffffu, base, leader < 0 ? 0 : leader);
        __syncwarp();
        const u32 r = base + __popc(peers & ltMask);
        if (i & 1) rank2[i >> 1] |= r << 16;
        else rank2[i >> 1] = r;
    }
    __syncthreads();
    // Per digit: warp exclusive offsets and tile total (thread = digit).
    if (tid < R)
    {
        const int d = tid;
        u32 acc = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w)
        {
            const u32 c = sm.warpHist[w][d];
            sm.warpHist[w][d] = acc;
            acc += c;
        }
        sm.count[d] = acc;
    }
    __syncthreads();
    // Publish this tile's digit counts early (a chain's first tile publishes
    // final prefixes), then build the tile-local order; the look-back comes
    // last so earlier tiles have had time to publish inclusive prefixes.
    {
        const int d = tid;
        const u32 cnt = d < R ? sm.count[d] : 0u;
        if (d < R) stRelaxed(status + tile * R + d, (tiles.chainStart(tile) ? kFlagPrefix : kFlagAgg) | u64(cnt));
        // exclusive scan of the tile's digit counts -> local starts
        u32 v = cnt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const u32 t = __shfl_up_sync(0xffffffffu, v, off);
            if (lane >= off) v += t;
        }
        if (lane == 31) sm.warpSums[warp] = v;
        __syncthreads();
        u32 wOff = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w)
            if (w < warp) wOff += sm.warpSums[w];
        if (d < R) sm.localStart[d] = wOff + v - cnt;
    }
    __syncthreads();
    // Reorder the tile in shared memory.
    u32 staged = 0;
    bool copyPending = false;
    if (stage)
    {
        unsigned spins = 0;
        while (!mbarTryWait(&sm.valuesReady, 0))
        {
            if (++spins > kStageSpins)
            {
                atomicExch(error, kErrLookback);
                copyPending = true;
                break;
            }
        }
        staged = copyPending ? 0u : sm.staged;
    }
#pragma unroll
    for (int i = 0; i < Items; ++i)
    {
        const size_t idx = warpBase + size_t(i) * 32 + lane;
        if (idx < tiles.end(tile))
        {
            const unsigned d = unsigned(key[i] >> shift) & dmask;
            const u32 r = (rank2[i >> 1] >> ((i & 1) * 16)) & 0xffffu;
            const u32 pos = sm.localStart[d] + sm.warpHist[warp][d] + r;
            sm.keys[pos] = key[i];
            const u32 li = u32(idx - tileBase);
            sm.vals[pos] = valsIn ? (li < staged ? sm.stage[li] : __ldcs(valsIn + idx))
                                  : u32(idx) - tiles.valueOffset(tile);
        }
    }
    // Look-back: global start of each digit for this tile.
    if (tid < R)
    {
        const int d = tid;
        const u64 total = sm.count[d];
        u64 excl = 0;
        if (!tiles.chainStart(tile))
        {
            // Walk back over earlier tiles, eight status words per round trip,
            // summing aggregates until an inclusive prefix is found (the
            // chain's first tile always holds one).
            long long j = (long long)tile - 1;
            unsigned spins = 0;
            while (j >= 0)
            {
                u64 w8[kLookbackWindow];
#pragma unroll
                for (int k = 0; k < kLookbackWindow; ++k)
                    w8[k] = j - k >= 0 ? ldRelaxed(status + size_t(j - k) * R + d) : kFlagPrefix;
                int k = 0;
                bool done = false;
                for (; k < kLookbackWindow; ++k)
                {
                    const u64 flag = w8[k] & ~kValueMask;
                    if (flag == 0) break;
                    excl += w8[k] & kValueMask;
                    if (flag == kFlagPrefix)
                    {
                        done = true;
                        break;
                    }
                }
                if (done) break;
                j -= k;
                if (k < kLookbackWindow)  // tile j has not published yet
                {
                    if (++spins > spinLimit)
                    {
                        atomicExch(error, kErrLookback);
                        break;
                    }
                    if (spins > 64) __nanosleep(64);
                }
            }
            stRelaxed(status + tile * R + d, kFlagPrefix | (excl + total));
        }
        // modulo 2^32: gstart + j is exact for every key of digit d
        sm.gstart[d] = tiles.digitBase(tile)[d] + u32(excl) - sm.localStart[d];
    }
    __syncthreads();
    const size_t remain = tiles.end(tile) - tileBase;
    const int valid = remain < size_t(T) ? int(remain) : T;
#pragma unroll 4
    for (int j = tid; j < valid; j += kThreads)
    {
        const u64 k = sm.keys[j];
        const unsigned d = unsigned(k >> shift) & dmask;
        const u32 out = sm.gstart[d] + u32(j);
        keysOut[out] = k;
        valsOut[out] = sm.vals[j];
    }
    if (copyPending)
    {
        // the CTA does not leave with its copy still in flight (bounded again)
        for (unsigned spins = 0; spins < kStageSpins && !mbarTryWait(&sm.valuesReady, 0); ++spins)
        {
        }
    }
    return true;
}

// CTAs per SM each configuration is built for.
template <int Bits, int Items>
constexpr int passMinBlocks()
{
    return Items <= 12 ? 4 : 3;
}

// One onesweep pass over keys[0, n): digit at bit `shift` (`bits` wide).
// valsIn == nullptr means values are the input indices (first pass).  The
// look-back status holds one word per tile and digit of the radix.
template <int Bits, int Items>
static __global__ void __launch_bounds__(kThreads, passMinBlocks<Bits, Items>())
    onesweepKernel(const u64 *__restrict__ keysIn, const u32 *__restrict__ valsIn, u64 *__restrict__ keysOut,
                   u32 *__restrict__ valsOut, size_t n, int shift, const u32 *__restrict__ bins, u32 *tileCounter,
                   u64 *status, int *error, int bits)
{
    onesweepTile<Bits, Items>(ContiguousTiles<kThreads * Items>{n, bins}, keysIn, valsIn, keysOut, valsOut, shift,
                              tileCounter, status, error, bits);
}

// One onesweep pass over the segments of a forest: every segment is sorted
// on its own (stable within the segment), in place in the global arrays.
template <int Bits, int Items>
static __global__ void __launch_bounds__(kThreads, passMinBlocks<Bits, Items>())
    segmentOnesweepKernel(SegmentTiles tiles, const u64 *__restrict__ keysIn, const u32 *__restrict__ valsIn,
                          u64 *__restrict__ keysOut, u32 *__restrict__ valsOut, int shift, u32 *tileCounter,
                          u64 *status, int *error, int bits)
{
    onesweepTile<Bits, Items>(tiles, keysIn, valsIn, keysOut, valsOut, shift, tileCounter, status, error, bits);
}

// ---------------------------------------------------------------------------
// Host-side dispatch over kSortConfigs (one instantiation per configuration):
// X(index, digit bits, keys per thread), in the order of kSortConfigs.
// ---------------------------------------------------------------------------
#define AOT_SORT_CONFIGS(X) X(0, 8, 10) X(1, 8, 16) X(2, 8, 8) X(3, 7, 12) X(4, 7, 16)

inline size_t passSmem(int c)
{
    switch (c)
    {
#define AOT_CASE(i, B, I) \
    case i: return sizeof(SharedPass<B, I>);
        AOT_SORT_CONFIGS(AOT_CASE)
#undef AOT_CASE
    default: throw std::invalid_argument("sort: unknown configuration");
    }
}

// Opts every pass kernel of this translation unit into its dynamic shared
// memory, once per device.
static inline void setPassSmemAll()
{
    static bool done[64] = {};
    int dev = 0;
    AOT_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && done[dev]) return;
#define AOT_CASE(i, B, I)                                                                                        \
    AOT_CHECK(cudaFuncSetAttribute(onesweepKernel<B, I>, cudaFuncAttributeMaxDynamicSharedMemorySize,           \
                                   int(sizeof(SharedPass<B, I>))));                                              \
    AOT_CHECK(cudaFuncSetAttribute(segmentOnesweepKernel<B, I>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                   int(sizeof(SharedPass<B, I>))));
    AOT_SORT_CONFIGS(AOT_CASE)
#undef AOT_CASE
    if (dev >= 0 && dev < 64) done[dev] = true;
}

// One contiguous pass of configuration c over n keys.
static inline void launchPass(int c, cudaStream_t s, const u64 *keysIn, const u32 *valsIn, u64 *keysOut, u32 *valsOut,
                       size_t n, int shift, const u32 *bins, u32 *tileCounter, u64 *status, int *error, int bits)
{
    const unsigned tiles = unsigned((n + size_t(configTile(c)) - 1) / size_t(configTile(c)));
    switch (c)
    {
#define AOT_CASE(i, B, I)                                                                                        \
    case i:                                                                                                      \
        onesweepKernel<B, I><<<tiles, kThreads, sizeof(SharedPass<B, I>), s>>>(                                  \
            keysIn, valsIn, keysOut, valsOut, n, shift, bins, tileCounter, status, error, bits);                 \
        break;
        AOT_SORT_CONFIGS(AOT_CASE)
#undef AOT_CASE
    default: throw std::invalid_argument("sort: unknown configuration");
    }
}

// One segmented pass of configuration c over `numTiles` tiles.
static inline void launchSegmentPass(int c, cudaStream_t s, unsigned numTiles, const SegmentTiles &tiles, const u64 *keysIn,
                              const u32 *valsIn, u64 *keysOut, u32 *valsOut, int shift, u32 *tileCounter,
                              u64 *status, int *error, int bits)
{
    switch (c)
    {
#define AOT_CASE(i, B, I)                                                                                        \
    case i:                                                                                                      \
        segmentOnesweepKernel<B, I><<<numTiles, kThreads, sizeof(SharedPass<B, I>), s>>>(                       \
            tiles, keysIn, valsIn, keysOut, valsOut, shift, tileCounter, status, error, bits);                   \
        break;
        AOT_SORT_CONFIGS(AOT_CASE)
#undef AOT_CASE
    default: throw std::invalid_argument("sort: unknown configuration");
    }
}

// Histogram of configuration c's digits.
static inline void launchHistogram(int c, cudaStream_t s, unsigned blocks, const u64 *keys, size_t n, int beginBit, int passes,
                            u32 *hist, int endBit)
{
    if (kSortConfigs[c].bits == 8)
        histogramKernel<8><<<blocks, kThreads, 0, s>>>(keys, n, beginBit, passes, hist, endBit);
    else
        histogramKernel<7><<<blocks, kThreads, 0, s>>>(keys, n, beginBit, passes, hist, endBit);
}

}  // namespace sort
}  // namespace aot
