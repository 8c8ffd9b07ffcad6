// forest.cuh -- kernels of the forest engine: many independent octrees
// ("systems") built and updated together, each launch covering all systems.
//
// Each system is the reference's Tree<Real, Octree> with LeafCount
// refinement (calculateNodeOp, octree_rebalance.cuh:174-249; graph passes
// 1177-1322) on its own particles; the forest only changes how the work is
// laid out on the device:
//   * particles of all systems are concatenated; system s owns
//     [base_s, base_s + n_s) of the key and permutation arrays, and its keys
//     are sorted on their own by a segmented onesweep sort (tiles never
//     straddle systems; see sort::SegmentTiles);
//   * the leaf arrays hold every system's cornerstone one after the other,
//     each including its end sentinel 2^63, with the owning system of every
//     entry in SEG.  A decision, scan and scatter over all entries therefore
//     rebalances all systems at once; a sentinel is always kept, and a
//     sibling group only counts when its first entry and its end entry belong
//     to the leaf's own system;
//   * capacity is per system: an update pass that would exceed a system's
//     leafCapacity is rejected for that system alone (its leaves are kept and
//     needsResize is set), exactly as the pass of a single tree.
// Begin indices B are global particle indices; counts are their differences.
#pragma once

#include "keygen.cuh"
#include "rebalance.cuh"

namespace aot
{
namespace forest
{
constexpr int kThreads = 256;

// One system (host-written).
struct System
{
    const void *x, *y, *z;
    u32 base;  // first particle (global index)
    u32 n;
};

// Per-system device state.
struct SysState
{
    int start;        // first entry (leaf 0) in the active leaf arrays
    int leaves;       // leaves in the active leaf arrays
    u32 active;       // active (non-escaped) particles
    int cap;          // leafCapacity: update passes reject proposals above it
    int needsResize;  // an update pass was rejected for capacity
    int changed;      // some decision of this pass is not 1
    int proposal;     // entries (leaves + sentinel) proposed by this pass
    int rejected;     // this pass keeps every leaf of the system
    int frozen;       // update passes leave the system alone (host-set)
    int iteration;    // build rounds that changed the system
    int startNew;     // start after this pass
    int sentinelNew;  // sentinel entry after this pass
};

// Forest-wide device state.
struct State
{
    int entries;       // active entries: all systems' leaves and sentinels
    int activeBuffer;
    int changed;       // some system applies changes in this pass
    int dirtyCount;
    int error;
    int changedPasses;   // update passes that changed some system since update began
    long long proposal;  // entries after this pass
};

struct Bufs
{
    u64 *K[2];
    u32 *B[2];
    int *SEG[2];
    u32 *N;        // leaf counts of the active arrays (materialised)
    int *ops;      // decisions of the pass
    i64 *offs;     // their exclusive scan
    int *dirty;    // new entries that need a begin index
    u64 *scanStatus;
    u32 *scanTile;
    State *st;
    SysState *sys;
    const System *systems;
    int numSystems;
    long long *history;  // [round][system]: leaves after each build round that changed the system
    const u64 *P;        // sorted keys
    __device__ __forceinline__ u64 *k(int a) const { return a ? K[1] : K[0]; }
    __device__ __forceinline__ u32 *b(int a) const { return a ? B[1] : B[0]; }
    __device__ __forceinline__ int *seg(int a) const { return a ? SEG[1] : SEG[0]; }
};

// --------------------------------------------------------------------------
// keys and the segmented sort
// --------------------------------------------------------------------------
// Keys of every system's particles and (hist != nullptr) the per-system
// histograms of the eight 8-bit digits, hist[system][pass slot][digit].  Each
// CTA takes a contiguous range of tiles, so its shared histogram is flushed
// only where the system changes.
// The keys of tiles [t0, t1) (a CTA's share), with the digit histograms
// counted in sh[kMaxPasses][kRadix] (zero on entry and on return) and flushed
// where the system changes.  sPair holds the two-level Hilbert table.
template <class Real, Curve C>
__device__ __forceinline__ void keygenTiles(const System *__restrict__ systems, const u32 *__restrict__ tileSys,
                                            const u32 *__restrict__ tileBegin, const u32 *__restrict__ tileEnd,
                                            u32 t0, u32 t1, const KeygenParams<Real> &prm, u64 *__restrict__ keys,
                                            u32 *__restrict__ hist, u32 *sh, const unsigned short *sPair)
{
    int cur = -1;
    auto flush = [&]() {
        __syncthreads();
        if (cur >= 0 && hist)
        {
            u32 *h = hist + size_t(cur) * sort::kPassSlots * sort::kRadix;
            for (int i = threadIdx.x; i < sort::kMaxPasses * sort::kRadix; i += blockDim.x)
            {
                const u32 v = sh[i];
                if (v)
                {
                    atomicAdd(h + i, v);
                    sh[i] = 0;
                }
            }
        }
        __syncthreads();
    };
    for (u32 t = t0; t < t1; ++t)
    {
        const int s = int(tileSys[t]);
        if (s != cur)
        {
            flush();
            cur = s;
        }
        const System sy = systems[s];
        const Real *x = static_cast<const Real *>(sy.x);
        const Real *y = static_cast<const Real *>(sy.y);
        const Real *z = static_cast<const Real *>(sy.z);
        const u32 end = tileEnd[t];
        for (u32 g = tileBegin[t] + threadIdx.x; g < end; g += blockDim.x)
        {
            const u32 l = g - sy.base;
            const u64 k = particleKey<Real, C>(x[l], y[l], z[l], prm, sPair);
            keys[g] = k;
            if (hist)
            {
#pragma unroll
                for (int p = 0; p < sort::kMaxPasses; ++p)
                    atomicAdd(&sh[p * sort::kRadix + int((k >> (p * sort::kRadixBits)) & (sort::kRadix - 1))], 1u);
            }
        }
    }
    flush();
}

template <class Real, Curve C>
static __global__ void __launch_bounds__(kThreads)
    keygenKernel(const System *__restrict__ systems, const u32 *__restrict__ tileSys,
                 const u32 *__restrict__ tileBegin, const u32 *__restrict__ tileEnd, u32 numTiles,
                 const KeygenParams<Real> prm, u64 *__restrict__ keys, u32 *__restrict__ hist)
{
    __shared__ u32 sh[sort::kMaxPasses * sort::kRadix];
    __shared__ unsigned short sPair[C == Curve::Hilbert ? kHilbertPairEntries : 1];
    for (int i = threadIdx.x; i < sort::kMaxPasses * sort::kRadix; i += blockDim.x) sh[i] = 0;
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
    const u32 per = (numTiles + gridDim.x - 1) / gridDim.x;
    const u32 t0 = blockIdx.x * per;
    keygenTiles<Real, C>(systems, tileSys, tileBegin, tileEnd, t0, min(numTiles, t0 + per), prm, keys, hist, sh, sPair);
}

// Per-system histograms of Bits-wide digits for `passes` passes, one CTA per
// tile of the segmented sort (the sort configurations whose digits are not
// the 8 bits key generation counts).  hist[system][pass slot][digit].
template <int Bits>
static __global__ void __launch_bounds__(kThreads)
    segHistKernel(const u32 *__restrict__ tileSys, const u32 *__restrict__ tileBegin, const u32 *__restrict__ tileEnd,
                  const u64 *__restrict__ keys, int passes, u32 *__restrict__ hist)
{
    constexpr int R = 1 << Bits;
    __shared__ u32 sh[sort::kPassSlots * R];
    for (int i = threadIdx.x; i < sort::kPassSlots * R; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const u32 t = blockIdx.x;
    for (u32 g = tileBegin[t] + threadIdx.x; g < tileEnd[t]; g += blockDim.x)
    {
        const u64 k = __ldg(keys + g);
        for (int p = 0; p < passes; ++p)
        {
            const int shift = p * Bits;
            const int bits = 64 - shift < Bits ? 64 - shift : Bits;
            atomicAdd(&sh[p * R + int((k >> shift) & ((1u << bits) - 1))], 1u);
        }
    }
    __syncthreads();
    u32 *h = hist + size_t(tileSys[t]) * sort::kPassSlots * sort::kRadix;
    for (int i = threadIdx.x; i < passes * R; i += blockDim.x)
    {
        const u32 v = sh[i];
        if (v) atomicAdd(h + (i / R) * sort::kRadix + (i % R), v);
    }
}

// Per system and pass: global start of each digit = base + exclusive scan of
// the system's digit counts.  bins[pass][system][digit].  One CTA of kRadix
// threads per system; s: kRadix words of shared scratch.
__device__ __forceinline__ void systemBins(const System *__restrict__ systems, int numSystems, int sys,
                                           const u32 *__restrict__ hist, u32 *__restrict__ bins, int passes, u32 *s)
{
    const int d = threadIdx.x;
    const u32 base = systems[sys].base;
    for (int p = 0; p < passes; ++p)
    {
        const u32 v = hist[(size_t(sys) * sort::kPassSlots + p) * sort::kRadix + d];
        s[d] = v;
        __syncthreads();
        for (int off = 1; off < sort::kRadix; off <<= 1)
        {
            const u32 t = d >= off ? s[d - off] : 0u;
            __syncthreads();
            s[d] += t;
            __syncthreads();
        }
        bins[(size_t(p) * numSystems + sys) * sort::kRadix + d] = base + s[d] - v;
        __syncthreads();
    }
}

static __global__ void __launch_bounds__(sort::kRadix)
    binsKernel(const System *__restrict__ systems, int numSystems, const u32 *__restrict__ hist,
               u32 *__restrict__ bins, int passes)
{
    __shared__ u32 s[sort::kRadix];
    systemBins(systems, numSystems, blockIdx.x, hist, bins, passes, s);
}

// With a sample array: also every 32nd key of the concatenated sorted keys
// (the key index of a build by levels).
__device__ __forceinline__ void activeAndSample(const Bufs &f, u64 *sample, size_t ns, size_t r, size_t size)
{
    for (size_t s = r; s < size_t(f.numSystems); s += size)
    {
        const System sy = f.systems[s];
        f.sys[s].active = sy.n ? u32(lowerBoundDev(f.P + sy.base, sy.n, kMaxKey)) : 0u;
    }
    if (sample)
        for (size_t j = r; j < ns; j += size) sample[j] = f.P[j << kSampleShift];
}

static __global__ void activeKernel(Bufs f, u64 *sample, size_t ns)
{
    activeAndSample(f, sample, ns, size_t(blockIdx.x) * blockDim.x + threadIdx.x, size_t(gridDim.x) * blockDim.x);
}

// --------------------------------------------------------------------------
// rebalance
// --------------------------------------------------------------------------
// Root of every system: entries 2s (leaf [0, 2^63)) and 2s + 1 (sentinel).
static __global__ void initKernel(Bufs f)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0)
    {
        State &st = *f.st;
        const int err = st.error;
        st = State{};
        st.error = err;
        st.entries = 2 * f.numSystems;
    }
    if (s >= f.numSystems) return;
    const System sy = f.systems[s];
    SysState &ss = f.sys[s];
    f.K[0][2 * s] = 0;
    f.K[0][2 * s + 1] = kMaxKey;
    f.B[0][2 * s] = sy.base;
    f.B[0][2 * s + 1] = sy.base + ss.active;
    f.SEG[0][2 * s] = s;
    f.SEG[0][2 * s + 1] = s;
    ss.start = 2 * s;
    ss.leaves = 1;
    ss.needsResize = 0;
    ss.iteration = 0;
    ss.frozen = 0;
}

// Per-pass reset; frozen (optional, one byte per system) marks systems an
// update leaves alone.
static __global__ void beginPassKernel(Bufs f, const unsigned char *frozen)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0)
    {
        f.st->changed = 0;
        f.st->dirtyCount = 0;
        *f.scanTile = 0;
    }
    if (s >= f.numSystems) return;
    SysState &ss = f.sys[s];
    ss.changed = 0;
    ss.proposal = 0;
    ss.rejected = 0;
    if (frozen) ss.frozen = frozen[s];
}

// siblingIndexAndLevel (octree_rebalance.cuh:26-50) inside one system.
__device__ __forceinline__ int siblingInSystem(const u64 *K, const int *SEG, int E, int i, unsigned &level)
{
    const u64 s = K[i];
    level = octLevel(K[i + 1] - s);
    if (level == 0) return -1;
    const int sib = int(octDigit(s, level));
    const int first = i - sib;
    if (first < 0 || first + 8 > E - 1) return -1;
    const int own = SEG[i];
    if (SEG[first] != own || SEG[first + 8] != own) return -1;
    return K[first + 8] == K[first] + octRange(level - 1) ? sib : -1;
}

// calculateNodeOp, LeafCount (octree_rebalance.cuh:174-249); sentinels stay.
__device__ __forceinline__ int leafOp(const u64 *K, const u32 *B, const int *SEG, int E, int i, unsigned bucket)
{
    if (K[i] == kMaxKey) return 1;
    unsigned level = 0;
    const int sib = siblingInSystem(K, SEG, E, i, level);
    if (sib > 0)
    {
        const int first = i - sib;
        if (u64(B[first + 8] - B[first]) <= u64(bucket)) return 0;
    }
    const u32 c = B[i + 1] - B[i];
    if (c > bucket * 512u && level + 3 < kOctLevels) return 4096;
    if (c > bucket * 64u && level + 2 < kOctLevels) return 512;
    if (c > bucket * 8u && level + 1 < kOctLevels) return 64;
    if (c > bucket && level < kOctLevels) return 8;
    return 1;
}

// Decisions of every entry, and per system the proposed entry count and
// whether anything changes.  Warps stride over the entries 32 at a time;
// lanes of one system combine their sums before one atomic.
static __global__ void __launch_bounds__(kThreads) decideKernel(Bufs f, unsigned bucket)
{
    const int a = f.st->activeBuffer;
    const int E = f.st->entries;
    const u64 *K = f.k(a);
    const u32 *B = f.b(a);
    const int *SEG = f.seg(a);
    const int lane = threadIdx.x & 31;
    const int warpsTotal = gridDim.x * (blockDim.x / 32);
    const int w0 = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    for (int base = w0 * 32; base < E; base += warpsTotal * 32)
    {
        const int i = base + lane;
        const bool valid = i < E;
        int op = 0, s = -1;
        if (valid)
        {
            op = leafOp(K, B, SEG, E, i, bucket);
            f.ops[i] = op;
            s = SEG[i];
        }
        const unsigned group = __match_any_sync(0xffffffffu, s);
        const int sum = __reduce_add_sync(group, op);
        const unsigned changedLanes = __ballot_sync(0xffffffffu, valid && op != 1) & group;
        if (valid && lane == __ffs(group) - 1)
        {
            atomicAdd(&f.sys[s].proposal, sum);
            if (changedLanes) atomicOr(&f.sys[s].changed, 1);
        }
    }
}

// Per system: does the pass apply?  Update passes (Build = false) keep every
// leaf of a system that is frozen, already needs a resize, or whose proposal
// exceeds its leafCapacity (the latter sets needsResize), as the capacity
// check of a single tree's pass (graphCheckCapacityKernel,
// octree_rebalance.cuh:1211-1232).
template <bool Build>
static __global__ void checkKernel(Bufs f)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= f.numSystems) return;
    SysState &ss = f.sys[s];
    bool reject = false;
    if (!Build)
    {
        if (ss.frozen || ss.needsResize) reject = true;
        else if (ss.changed && ss.proposal - 1 > ss.cap)
        {
            ss.needsResize = 1;
            reject = true;
        }
    }
    ss.rejected = reject ? 1 : 0;
    if (ss.changed && !reject) atomicOr(&f.st->changed, 1);
}

// Exclusive scan of the applied decisions (a rejected system keeps every
// entry): offs[0..E], proposal = offs[E].
static __global__ void __launch_bounds__(rb::kScanThreads) scanKernel(Bufs f)
{
    __shared__ i64 sWarp[rb::kScanThreads / 32];
    __shared__ u32 sTile;
    __shared__ i64 sPrefix;
    State *st = f.st;
    if (!st->changed) return;
    const int a = st->activeBuffer;
    const int E = st->entries;
    const int *SEG = f.seg(a);
    const u32 numTiles = u32((size_t(E) + 1 + rb::kScanTile - 1) / rb::kScanTile);
    if (threadIdx.x == 0) sTile = atomicAdd(f.scanTile, 1u);
    __syncthreads();
    const u32 tile = sTile;
    if (tile >= numTiles) return;
    const size_t first = size_t(tile) * rb::kScanTile + size_t(threadIdx.x) * rb::kScanItems;
    int ops[rb::kScanItems];
    i64 sum = 0;
#pragma unroll
    for (int j = 0; j < rb::kScanItems; ++j)
    {
        const size_t i = first + j;
        int op = 0;
        if (i < size_t(E)) op = f.sys[SEG[i]].rejected ? 1 : f.ops[i];
        ops[j] = op;
        sum += op;
    }
    i64 total;
    const i64 excl = rb::blockExclusiveScan(sum, sWarp, total);
    if (threadIdx.x == 0) sPrefix = rb::lookback(f.scanStatus, tile, total, &st->error);
    __syncthreads();
    i64 run = sPrefix + excl;
#pragma unroll
    for (int j = 0; j < rb::kScanItems; ++j)
    {
        const size_t i = first + j;
        if (i <= size_t(E))
        {
            f.offs[i] = run;
            if (i == size_t(E)) st->proposal = run;
        }
        run += ops[j];
    }
}

// processNode (octree_rebalance.cuh:253-365) for every entry into the
// inactive arrays, with the work list of new entries that need a begin index
// and each system's new start and sentinel.
static __global__ void __launch_bounds__(kThreads) scatterKernel(Bufs f)
{
    State *st = f.st;
    if (!st->changed) return;
    const int a = st->activeBuffer, b = a ^ 1;
    const int E = st->entries;
    const u64 *K = f.k(a);
    const u32 *B = f.b(a);
    const int *SEG = f.seg(a);
    u64 *Kn = f.k(b);
    u32 *Bn = f.b(b);
    int *SEGn = f.seg(b);
    const int lane = threadIdx.x & 31;
    const int warpsTotal = gridDim.x * (blockDim.x / 32);
    const int w0 = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    for (int base = w0 * 32; base < E; base += warpsTotal * 32)
    {
        const int i = base + lane;
        int nDirty = 0, op = 0;
        i64 ni = 0;
        if (i < E)
        {
            const int s = SEG[i];
            ni = f.offs[i];
            op = int(f.offs[i + 1] - ni);
            const u64 start = K[i];
            if (op >= 1)
            {
                if (i == f.sys[s].start) f.sys[s].startNew = int(ni);
                if (start == kMaxKey) f.sys[s].sentinelNew = int(ni);
            }
            if (op == 1)
            {
                Kn[ni] = start;
                Bn[ni] = B[i];
                SEGn[ni] = s;
            }
            else if (op > 1)
            {
                const unsigned level = octLevel(K[i + 1] - start);
                const u64 nr = octRange(level + rb::splitLevels(op));
                for (int c = 0; c < op; ++c)
                {
                    Kn[ni + c] = start + u64(c) * nr;
                    SEGn[ni + c] = s;
                }
                Bn[ni] = B[i];  // the first child starts where the parent did
                nDirty = op - 1;
            }
        }
        const int d0 = rb::warpAppend(&st->dirtyCount, nDirty);
        for (int c = 1; c <= nDirty; ++c) f.dirty[d0 + c - 1] = int(ni) + c;
    }
}

// Applies the pass: flips the arrays, moves every system's start and leaf
// count, and (build) records the leaf count of each system that changed.
template <bool Build>
static __global__ void commitKernel(Bufs f)
{
    State *st = f.st;
    if (!st->changed) return;
    __syncthreads();
    for (int s = threadIdx.x; s < f.numSystems; s += blockDim.x)
    {
        SysState &ss = f.sys[s];
        ss.start = ss.startNew;
        ss.leaves = ss.sentinelNew - ss.startNew;
        if (Build && ss.changed && !ss.rejected)
        {
            f.history[size_t(ss.iteration) * f.numSystems + s] = ss.leaves;
            ss.iteration += 1;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        st->activeBuffer ^= 1;
        st->entries = int(st->proposal);
        if (!Build) st->changedPasses += 1;
    }
}

// Begin indices of the new entries (All: of every entry): a leaf's is the
// lower bound of its key among its system's keys (calculateNodeCount,
// octree_rebalance.cuh:367-413), a sentinel's the system's active end.
template <bool All>
static __global__ void __launch_bounds__(kThreads) refreshKernel(Bufs f)
{
    const State *st = f.st;
    const int a = st->activeBuffer;
    const u64 *K = f.k(a);
    u32 *B = f.b(a);
    const int *SEG = f.seg(a);
    const int count = All ? st->entries : st->dirtyCount;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
    {
        const int i = All ? j : f.dirty[j];
        const int s = SEG[i];
        const System sy = f.systems[s];
        const u64 k = K[i];
        B[i] = sy.base + (k == kMaxKey ? f.sys[s].active : u32(lowerBoundDev(f.P + sy.base, sy.n, k)));
    }
}

// N = differences of B for the leaves of the active arrays (sentinels 0).
static __global__ void materializeKernel(Bufs f)
{
    const State *st = f.st;
    const int a = st->activeBuffer;
    const u64 *K = f.k(a);
    const u32 *B = f.b(a);
    const int E = st->entries;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < E; i += gridDim.x * blockDim.x)
        f.N[i] = K[i] == kMaxKey ? 0u : B[i + 1] - B[i];
}

}  // namespace forest
}  // namespace aot
