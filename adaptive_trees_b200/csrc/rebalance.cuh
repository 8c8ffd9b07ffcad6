// rebalance.cuh -- device kernels of the split/merge rebalance passes.
//
// One pass (octree or binary) is three kernels, all reading sizes and the
// A/B selection from DeviceState so a captured CUDA graph stays valid while
// the topology changes (the reference's graph path, octree_rebalance.cuh:
// 1177-1322 and kdtree3d_rebalance.cuh:160-245):
//   decide+scan   per-leaf op code and its exclusive prefix in ONE kernel
//                 (decoupled look-back over 2048-entry tiles); the tile that
//                 holds entry numLeaves records the proposed leaf count;
//   scatter       writes the proposal into the inactive buffer when it is
//                 accepted; the last CTA to finish applies the reference's
//                 capacity check and commit (graphCheckCapacityKernel +
//                 graphCommitNodesKernel) and the work lists for the refresh;
//   refresh       recomputes per-leaf quantities of new leaves only.
// Per leaf the engine keeps B[i] = lowerBound(P, K[i]) (B[L] = active count):
// the leaf count is B[i+1] - B[i] and a sibling group's count is
// B[first+8] - B[first], so LeafCount decisions need no count array and
// unchanged leaves keep B without a search.
#pragma once

#include "common.cuh"
#include "sfc.cuh"

namespace aot
{
namespace rb
{
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr u64 kFlagAgg = u64(1) << 62;
constexpr u64 kFlagPrefix = u64(2) << 62;
constexpr u64 kValueMask = (u64(1) << 62) - 1;
constexpr unsigned kLookbackSpins = 1u << 22;
constexpr int kScatterThreads = 256;
constexpr int kRefreshThreads = 256;

// Buffers of one tree (A/B pairs are indexed by DeviceState::activeBuffer).
struct TreeBufs
{
    u64 *K[2];    // leaf boundaries, numLeaves + 1 used
    u32 *B[2];    // begin index of every boundary in P
    u32 *NF[2];   // near-field counts (NFCount octrees)
    u8 *G[2];     // group-can-merge flag at each complete group's first leaf
    u32 *N[2];    // leaf counts, materialised for getters and views
    i64 *offs;    // decision scan, capacity + 1
    int *dirty;   // new leaves that need a search (and NF)
    u64 *scanStatus;
    u32 *scanTile;
    DeviceState *st;
    // A/B selection without dynamic indexing of the (by-value) arrays, which
    // would move the whole struct to local memory
    __device__ __forceinline__ u64 *k(int a) const { return a ? K[1] : K[0]; }
    __device__ __forceinline__ u32 *b(int a) const { return a ? B[1] : B[0]; }
    __device__ __forceinline__ u32 *nf(int a) const { return a ? NF[1] : NF[0]; }
    __device__ __forceinline__ u8 *g(int a) const { return a ? G[1] : G[0]; }
    __device__ __forceinline__ u32 *n(int a) const { return a ? N[1] : N[0]; }
};

__device__ __forceinline__ bool halted(const DeviceState *st)
{
    return st->converged | st->overflow | st->error;
}

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

// Block-wide exclusive scan of one value per thread (kScanThreads threads).
__device__ __forceinline__ i64 blockExclusiveScan(i64 v, i64 *sWarp, i64 &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    i64 inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        const i64 t = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += t;
    }
    if (lane == 31) sWarp[warp] = inc;
    __syncthreads();
    i64 wOff = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kScanThreads / 32; ++w)
    {
        const i64 s = sWarp[w];
        if (w < warp) wOff += s;
        tot += s;
    }
    total = tot;
    return wOff + inc - v;
}

// Decoupled look-back: returns the exclusive prefix of `tile` given its
// aggregate.  Called by one thread.  Polling an unpublished tile more than
// spinLimit times records kErrLookback and returns the prefix summed so far.
__device__ __forceinline__ i64 lookback(u64 *status, u32 tile, i64 aggregate, int *error,
                                        unsigned spinLimit = kLookbackSpins)
{
    if (tile == 0)
    {
        stRelaxed(status, kFlagPrefix | u64(aggregate));
        return 0;
    }
    stRelaxed(status + tile, kFlagAgg | u64(aggregate));
    i64 excl = 0;
    long long j = (long long)tile - 1;
    unsigned spins = 0;
    while (j >= 0)
    {
        u64 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = j - k >= 0 ? ldRelaxed(status + (j - k)) : kFlagPrefix;
        int k = 0;
        bool done = false;
        for (; k < 8; ++k)
        {
            const u64 flag = v[k] & ~kValueMask;
            if (flag == 0) break;
            excl += i64(v[k] & kValueMask);
            if (flag == kFlagPrefix)
            {
                done = true;
                break;
            }
        }
        if (done) break;
        j -= k;
        if (k < 8)
        {
            if (++spins > spinLimit)
            {
                atomicExch(error, kErrLookback);
                break;
            }
            if (spins > 64) __nanosleep(64);
        }
    }
    stRelaxed(status + tile, kFlagPrefix | u64(excl + aggregate));
    return excl;
}

// Generic single-pass decide+scan.  OpFn(i, L) returns the op code of leaf
// i < L; entry L is 0.  Writes offs[0..L] (exclusive), state->proposal and
// state->changed.
template <class OpFn>
__device__ void decideScan(const OpFn &opOf, TreeBufs tb)
{
    __shared__ i64 sWarp[kScanThreads / 32];
    __shared__ u32 sTile;
    __shared__ i64 sPrefix;
    __shared__ int sChanged;
    DeviceState *st = tb.st;
    if (halted(st) || st->needsResize) return;
    const int L = st->numLeaves;
    const size_t entries = size_t(L) + 1;
    const u32 numTiles = u32((entries + kScanTile - 1) / kScanTile);
    if (threadIdx.x == 0)
    {
        sTile = atomicAdd(tb.scanTile, 1u);
        sChanged = 0;
    }
    __syncthreads();
    const u32 tile = sTile;
    if (tile >= numTiles) return;
    const size_t first = size_t(tile) * kScanTile + size_t(threadIdx.x) * kScanItems;
    int ops[kScanItems];
    i64 sum = 0;
    bool changed = false;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j)
    {
        const size_t i = first + j;
        int op = 0;
        if (i < size_t(L))
        {
            op = opOf(int(i), L);
            changed |= op != 1;
        }
        ops[j] = op;
        sum += op;
    }
    if (changed) sChanged = 1;
    i64 total;
    const i64 excl = blockExclusiveScan(sum, sWarp, total);
    if (threadIdx.x == 0)
    {
        sPrefix = lookback(tb.scanStatus, tile, total, &st->error);
        if (sChanged) atomicOr(&st->changed, 1);
    }
    __syncthreads();
    i64 run = sPrefix + excl;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j)
    {
        const size_t i = first + j;
        if (i <= size_t(L))
        {
            tb.offs[i] = run;
            if (i == size_t(L)) st->proposal = run;
        }
        run += ops[j];
    }
}

// Warp-aggregated append of `count` consecutive items to a list; returns the
// first slot of this thread.
__device__ __forceinline__ int warpAppend(int *counter, int count)
{
    const int lane = threadIdx.x & 31;
    int inc = count;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        const int t = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += t;
    }
    const int warpTotal = __shfl_sync(0xffffffffu, inc, 31);
    int base = 0;
    if (lane == 31 && warpTotal) base = atomicAdd(counter, warpTotal);
    base = __shfl_sync(0xffffffffu, base, 31);
    return base + inc - count;
}

// Completion of a scatter kernel: the last CTA applies the capacity check and
// the commit (graphCheckCapacityKernel + graphCommitNodesKernel semantics,
// octree_rebalance.cuh:1211-1273).  `limit` is the leaf capacity the scatter
// wrote against: the reference's leafCapacity in kModeUpdate, the physical
// buffer size in the build modes (exceeding it is an overflow the host repairs
// by growing the buffers and repeating the round).  In kModeBinaryBuild the
// reference's leafCapacity (st->logicalCap) grows by 25% steps until the
// proposal fits, as its build loop does through needsResize/growBuffers
// (kdtree3d.cu:239-249).
__device__ __forceinline__ void commitIfLast(DeviceState *st, long long limit, int mode, bool binary,
                                             long long *history)
{
    __shared__ bool sLast;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        sLast = atomicAdd(&st->doneBlocks, 1) == int(gridDim.x) - 1;
    }
    __syncthreads();
    if (!sLast || threadIdx.x != 0) return;
    __threadfence();
    st->doneBlocks = 0;
    const long long total = st->proposal;
    if (st->needsResize || !st->changed)
    {
        st->converged = 1;
        if (mode != kModeUpdate) st->rounds += 1;
        return;
    }
    if (total > limit)
    {
        if (mode == kModeUpdate)
        {
            st->needsResize = 1;
            st->converged = 1;
        }
        else
        {
            st->overflow = 1;
        }
        return;
    }
    if (mode == kModeBinaryBuild)
    {
        long long c = st->logicalCap < 1 ? 1 : st->logicalCap;
        while (total > c) c += (c + 3) / 4;  // c >= 1 grows by >= 1 per step
        st->logicalCap = c;
    }
    st->newNumLeaves = int(total);
    st->numLeaves = int(total);
    if (binary) st->numNodes = (int(total) - 1) * 2 + 1;
    st->activeBuffer ^= 1;
    if (mode != kModeUpdate)
    {
        if (history) history[st->iteration] = total;
        st->iteration += 1;
        st->rounds += 1;
    }
    else
    {
        st->updatePasses += 1;
    }
}

// --------------------------------------------------------------------------
// Octree
// --------------------------------------------------------------------------
// siblingIndexAndLevel (octree_rebalance.cuh:26-50)
__device__ __forceinline__ int siblingIndex(const u64 *K, int L, int i, unsigned &level)
{
    const u64 s = K[i];
    level = octLevel(K[i + 1] - s);
    if (level == 0) return -1;
    const int sib = int(octDigit(s, level));
    const int first = i - sib;
    if (first < 0 || first > L - 8) return -1;
    return K[first + 8] == K[first] + octRange(level - 1) ? sib : -1;
}

// calculateNodeOp (octree_rebalance.cuh:174-249)
template <bool NF>
struct OctreeOp
{
    const u64 *K;
    const u32 *B;
    const u32 *NFc;
    const u8 *G;
    unsigned bucket;
    __device__ __forceinline__ int operator()(int i, int L) const
    {
        unsigned level = 0;
        const int sib = siblingIndex(K, L, i, level);
        if constexpr (!NF)
        {
            if (sib > 0)
            {
                const int first = i - sib;
                const u64 parent = u64(B[first + 8] - B[first]);
                if (parent <= u64(bucket)) return 0;
            }
            const u32 c = B[i + 1] - B[i];
            if (c > bucket * 512u && level + 3 < kOctLevels) return 4096;
            if (c > bucket * 64u && level + 2 < kOctLevels) return 512;
            if (c > bucket * 8u && level + 1 < kOctLevels) return 64;
            if (c > bucket && level < kOctLevels) return 8;
            return 1;
        }
        else
        {
            if (sib >= 0)
            {
                const int first = i - sib;
                if (first + 8 <= L && G[first]) return sib == 0 ? 1 : 0;
            }
            const u64 c = NFc[i], b = bucket;
            if (c > b * 262144 && level + 3 < kOctLevels) return 4096;
            if (c > b * 4096 && level + 2 < kOctLevels) return 512;
            if (c > b * 64 && level + 1 < kOctLevels) return 64;
            if (c > b && level < kOctLevels) return 8;
            return 1;
        }
    }
};

template <bool NF>
static __global__ void __launch_bounds__(kScanThreads) octDecideScanKernel(TreeBufs tb, unsigned bucket)
{
    const int a = tb.st->activeBuffer;
    const OctreeOp<NF> op{tb.k(a), tb.b(a), tb.nf(a), tb.g(a), bucket};
    decideScan(op, tb);
}

__device__ __forceinline__ int opAt(const i64 *offs, int i) { return int(offs[i + 1] - offs[i]); }

// log8ceil of a split op code (octree_rebalance.cuh:349): 8->1, 64->2, 512->3, 4096->4
__device__ __forceinline__ unsigned splitLevels(int op) { return op == 8 ? 1u : op == 64 ? 2u : op == 512 ? 3u : 4u; }

// processNode (octree_rebalance.cuh:253-365) for every old leaf, plus the
// work lists of the refresh: new leaves needing a search (and NF) and
// candidate group leaders needing a parent NF.
template <bool NF>
__device__ __forceinline__ void octScatterLeaf(const TreeBufs &tb, DeviceState *st, int i, int L, int a, int b,
                                               long long total)
{
    const int lane = threadIdx.x & 31;
    int nDirty = 0, op = 0;
    i64 ni = 0;
    u64 start = 0, nr = 0;
    u64 *Kn = tb.k(b);
    if (i < L)
    {
        const u64 *K = tb.k(a);
        const i64 *offs = tb.offs;
        op = opAt(offs, i);
        start = K[i];
        const unsigned level = octLevel(K[i + 1] - start);
        ni = offs[i];
        u32 *Bn = tb.b(b);
        if (op == 1)
        {
            Kn[ni] = start;
            Bn[ni] = tb.b(a)[i];
            if constexpr (NF)
            {
                // a merge leader becomes a new leaf; a kept leaf keeps its NF
                // and its group flag (both depend on the particles only; a
                // group completed in this pass holds a new leaf, and the
                // refresh of that leaf's parent rewrites the flag)
                const bool leader = i + 1 < L && opAt(offs, i + 1) == 0;
                if (leader)
                {
                    nDirty = 1;
                }
                else
                {
                    tb.nf(b)[ni] = tb.nf(a)[i];
                    tb.g(b)[ni] = tb.g(a)[i];
                }
            }
        }
        else if (op > 1)
        {
            nr = octRange(level + splitLevels(op));
            Bn[ni] = tb.b(a)[i];  // the first child starts where the parent did
            nDirty = NF ? op : op - 1;
        }
        if (i == 0)
        {
            Kn[total] = kMaxKey;
            tb.b(b)[total] = st->numActiveParticles;
        }
    }
    // work lists (warp-aggregated appends; list order is irrelevant)
    const int d0 = warpAppend(&st->dirtyCount, nDirty);
    if (nDirty && op == 1) tb.dirty[d0] = int(ni);
    // the children of the warp's split leaves, written by all lanes together
    // (consecutive children in consecutive lanes): each child finds its
    // leaf as the last lane whose exclusive child offset is <= its index
    const int children = op > 1 ? op : 0;
    int inc = children;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        const int t = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += t;
    }
    const int excl = inc - children;
    const int warpChildren = __shfl_sync(0xffffffffu, inc, 31);
    const int c0 = NF ? 0 : 1;  // LeafCount: the first child needs no search
    for (int base = 0; base < warpChildren; base += 32)
    {
        const int t = base + lane;
        int owner = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1)
        {
            const int cand = owner + step;
            const int ex = __shfl_sync(0xffffffffu, excl, cand & 31);
            if (cand < 32 && ex <= t) owner = cand;
        }
        const i64 niL = __shfl_sync(0xffffffffu, ni, owner);
        const u64 startL = __shfl_sync(0xffffffffu, start, owner);
        const u64 nrL = __shfl_sync(0xffffffffu, nr, owner);
        const int d0L = __shfl_sync(0xffffffffu, d0, owner);
        const int exL = __shfl_sync(0xffffffffu, excl, owner);
        if (t < warpChildren)
        {
            const int c = t - exL;
            Kn[niL + c] = startL + u64(c) * nrL;
            if (c >= c0) tb.dirty[d0L + c - c0] = int(niL) + c;
        }
    }
}

// processNode (octree_rebalance.cuh:253-365) for every old leaf, plus the
// work lists of the refresh: new leaves needing a search (and NF) and
// candidate group leaders needing a parent NF.  Persistent grid: each warp
// strides over the leaves 32 at a time, so every lane takes part in the
// warp-aggregated appends.
template <bool NF>
static __global__ void __launch_bounds__(kScatterThreads)
    octScatterKernel(TreeBufs tb, long long limit, int mode, long long *history)
{
    DeviceState *st = tb.st;
    if (halted(st)) return;  // uniform: the state does not change before the last CTA
    const long long total = st->proposal;
    const bool proceed = !st->needsResize && st->changed && total <= limit;
    if (proceed)
    {
        const int L = st->numLeaves;
        const int a = st->activeBuffer, b = a ^ 1;
        const int lane = threadIdx.x & 31;
        const int warpsTotal = gridDim.x * (blockDim.x / 32);
        const int w0 = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
        for (int base = w0 * 32; base < L; base += warpsTotal * 32) octScatterLeaf<NF>(tb, st, base + lane, L, a, b, total);
    }
    commitIfLast(st, limit, mode, false, history);
}

// Lower bound of v in the sorted keys when `lo` is already a lower bound of a
// key <= v (so the answer is >= lo): gallop forward from lo (exponential
// probes, then a binary search of the bracket).  Near-field cells hold few
// particles, so the upper end of a cell is usually found in the cache line of
// its lower end.  Far targets fall back to the sampled index.
__device__ __forceinline__ u32 lowerFrom(const KeyIndex &idx, u32 lo, u64 v)
{
    const u64 *P = idx.keys;
    const u32 n = u32(idx.n);
    if (lo >= n || __ldg(P + lo) >= v) return lo;
    u32 base = lo, step = 1;  // P[base] < v
    for (int k = 0; k < 12; ++k)
    {
        const u32 probe = base + step;
        if (probe >= n || __ldg(P + probe) >= v)
        {
            const u32 end = probe < n ? probe : n;
            return base + 1 + lowerBound32(P + base + 1, end - base - 1, v);
        }
        base = probe;
        step <<= 1;
    }
    return idx.lower(v);
}

// Begin index B[i] = lowerBound(P, K[i]) of new leaves (All: of every leaf and
// the end sentinel).  This is the whole count refresh of LeafCount trees: the
// counts are differences of B.
template <bool All>
static __global__ void __launch_bounds__(kRefreshThreads) octBeginKernel(TreeBufs tb, KeyIndex idx)
{
    DeviceState *st = tb.st;
    if (halted(st)) return;
    const int a = st->activeBuffer;
    const int L = st->numLeaves;
    const u64 *K = tb.k(a);
    u32 *B = tb.b(a);
    if (All && blockIdx.x == 0 && threadIdx.x == 0) B[L] = st->numActiveParticles;
    const int count = All ? L : st->dirtyCount;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
    {
        const int i = All ? j : tb.dirty[j];
        B[i] = u32(idx.lower(K[i]));
    }
}

// The begin index of every leaf (and B[L] = the active count) by merging the
// sorted leaf keys K with the sorted particle keys P, the refresh of all
// leaves at the start of an update: B[i] = #{j : P[j] < K[i]}.  In the merged
// order (a leaf key before an equal particle key) K[i] sits at i + B[i].  The
// merged sequence of L + nActive entries is cut into chunks of kMergeChunk; a
// first kernel finds each cut's leaf count by a binary search of the merge
// path, and a second one takes a chunk per CTA: its particle keys into shared
// memory, each of its leaf keys a search there.  Every key is read once and
// coalesced, where lower bounds one leaf at a time read the sampled index and
// a window per leaf.
constexpr int kMergeChunk = 2048;

// Leaves among the first d entries of the merged order.
__device__ __forceinline__ u32 mergeSplit(const u64 *K, u32 L, const u64 *P, u32 nA, u64 d)
{
    u32 lo = d > nA ? u32(d - nA) : 0u, hi = d < L ? u32(d) : L;
    while (lo < hi)
    {
        const u32 mid = (lo + hi) >> 1;
        // leaf mid comes before particle d - mid - 1: more than mid leaves
        if (K[mid] <= P[d - mid - 1]) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static __global__ void mergeSplitKernel(TreeBufs tb, const u64 *P, u32 *splits)
{
    const DeviceState *st = tb.st;
    if (halted(st)) return;
    const u32 L = u32(st->numLeaves), nA = st->numActiveParticles;
    const u64 M = u64(L) + nA;
    const u64 chunks = (M + kMergeChunk - 1) / kMergeChunk;
    const u64 *K = tb.k(st->activeBuffer);
    for (u64 c = blockIdx.x * u64(blockDim.x) + threadIdx.x; c <= chunks; c += u64(gridDim.x) * blockDim.x)
        splits[c] = mergeSplit(K, L, P, nA, c * kMergeChunk < M ? c * kMergeChunk : M);
}

static __global__ void __launch_bounds__(256) mergeBeginKernel(TreeBufs tb, const u64 *P, const u32 *splits)
{
    __shared__ u64 sP[kMergeChunk];
    const DeviceState *st = tb.st;
    if (halted(st)) return;
    const int a = st->activeBuffer;
    const u32 L = u32(st->numLeaves), nA = st->numActiveParticles;
    const u64 M = u64(L) + nA;
    const u64 chunks = (M + kMergeChunk - 1) / kMergeChunk;
    const u64 *K = tb.k(a);
    u32 *B = tb.b(a);
    if (blockIdx.x == 0 && threadIdx.x == 0) B[L] = nA;
    for (u64 c = blockIdx.x; c < chunks; c += gridDim.x)
    {
        const u64 d0 = c * kMergeChunk, d1 = d0 + kMergeChunk < M ? d0 + kMergeChunk : M;
        const u32 i0 = splits[c], i1 = splits[c + 1];
        const u32 j0 = u32(d0 - i0), j1 = u32(d1 - i1);
        __syncthreads();  // the previous chunk's searches are done
        for (u32 j = j0 + threadIdx.x; j < j1; j += blockDim.x) sP[j - j0] = P[j];
        __syncthreads();
        for (u32 i = i0 + threadIdx.x; i < i1; i += blockDim.x)
        {
            const u64 k = K[i];
            u32 lo = 0, len = j1 - j0;
            while (len)
            {
                const u32 half = len >> 1;
                const bool less = sP[lo + half] < k;
                lo = less ? lo + half + 1 : lo;
                len = less ? len - half - 1 : half;
            }
            B[i] = j0 + lo;
        }
    }
}

// Near-field counts by parent cell.
//
// NF(leaf) = own x (population of the 27 periodic same-level cells around the
// leaf) (computeNFCooperative, octree_rebalance.cuh:579-634), and a complete
// sibling group may merge when parent count x (population of the 27 cells
// around the parent, one level up) <= bucket (computeGroupCanMergeKernel,
// octree_rebalance.cuh:636-700).  Both depend only on the particles, not on
// the tree, so they are computed per parent cell P at level l-1 (a "unit"):
//   * the 8 children of P have their 27-cell stencils inside the 4 x 4 x 4
//     block of level-l cells around P, and that block is partitioned by the
//     children of the 27 parent-level cells Q around P (P included) that
//     touch P (per axis: offset -1 gives the upper child, 0 both, +1 the
//     lower);
//   * a Q that is an internal node of the tree (found in the node table)
//     gives its child counts as differences of its children's begin indices;
//     any other Q is a leaf or lies inside one, and its particles are counted
//     per child within that leaf's few keys, found through the table too;
//   * each leaf of P sums its 3 x 3 x 3 sub-block, and the group flag is the
//     sum of the 27 Q populations.
// Periodic wrap at low levels makes several offsets name the same cell;
// every offset is counted, as in the per-leaf stencil.
// A warp takes 32 list entries, cuts them into units (runs of leaves with
// the same parent) and treats up to kUnitBatch units at once: phase A spreads
// the (unit, Q) pairs over the lanes and resolves those found in the node
// table; the rest are queued and phase B spreads them over the lanes for the
// counts inside leaves; phase C gives every lane its own leaf.  Lanes stay
// busy instead of following the slowest Q of one unit.
constexpr u32 kNFScanMax = 256;  // key ranges up to this length are scanned, longer ones searched
constexpr int kNFGallop = 4;     // gallop window of the fallback search: 15 keys
constexpr int kUnitBatch = 8;    // units of a warp in flight

// Leaf index of child 0 of the parent at `pStart` if all 8 children are
// leaves (a complete group), else -1.
__device__ __forceinline__ int completeGroup(const u64 *K, int L, int h, unsigned level, u64 pStart, u64 pRange)
{
    const int i0 = h - int(octDigit(K[h], level));
    if (i0 < 0 || i0 + 8 > L) return -1;
    if (K[i0] != pStart || K[i0 + 8] != pStart + pRange) return -1;
    return i0;
}

// Cell of `start` at level `pl`: grid coordinates of its origin (21-bit) and,
// for Hilbert, the curve state before each level (6 bits per level; levels
// 0-9 in st0, 10-19 in st1, 20 in st2) and the state of its children.
struct CellPath
{
    u32 x, y, z;
    u64 st0, st1, st2;
    int childState;
};

template <bool Hilbert>
__device__ __forceinline__ CellPath decodeCell(u64 start, unsigned pl, const unsigned char *sNext,
                                               const unsigned char *sDec)
{
    CellPath c{0, 0, 0, 0, 0, 0, kHilbertStart};
    if constexpr (Hilbert)
    {
        int st = kHilbertStart;
        for (unsigned k = 0; k < pl; ++k)
        {
            const u64 bitsv = u64(st) << (6 * (k < 10 ? k : (k < 20 ? k - 10 : k - 20)));
            if (k < 10) c.st0 |= bitsv;
            else if (k < 20) c.st1 |= bitsv;
            else c.st2 |= bitsv;
            const unsigned b = kOctLevels - 1 - k;
            const unsigned o = sDec[st * 8 + int((start >> (3u * b)) & 7u)];
            c.x |= ((o >> 2) & 1u) << b;
            c.y |= ((o >> 1) & 1u) << b;
            c.z |= (o & 1u) << b;
            st = sNext[st * 8 + int(o)];
        }
        c.childState = st;
    }
    else
    {
        c.x = compact3(start >> 2);
        c.y = compact3(start >> 1);
        c.z = compact3(start);
    }
    return c;
}

// Node table: internal node -> the begin indices of its 8 children in the
// sorted keys and its end (9 values; child counts and the node's count are
// their differences).  It holds every cell that has been an internal node
// of the tree since the keys were last sorted: nodeTableKernel enters the
// ancestors of new leaves before each near-field refresh, and the refresh
// only reads it.  The values depend only on the sorted keys, so an entry
// stays right while the tree changes; the table is cleared when the
// particles are sorted again and otherwise only grows.  A cell that is not
// in the table is a leaf or lies inside one: the child of its deepest entered
// ancestor that holds it has few keys, which the refresh counts.  Open
// addressing with linear probing, at most kCellProbes probes; keys are cell
// codes (never 0), 0 marks an empty slot.
constexpr int kGroupBegins = 9;
constexpr int kGroupRow = 12;  // words per slot: the key (2), the 9 values, 1 spare (48 B, 16-byte aligned)
constexpr u32 kCellProbes = 64;
struct NodeTable
{
    u32 *rows;  // [slot][kGroupRow]
    u32 slots;
};

// Cell code: the key prefix of a cell at `level` below a placeholder bit,
// unique over all levels.
__device__ __forceinline__ u64 cellCode(u64 start, unsigned level)
{
    return (start >> (3u * (kOctLevels - level))) | (u64(1) << (3u * level));
}

// Home slot of a code among `slots`: Fibonacci hashing (the high bits of one
// 64-bit product), then a multiply-shift into [0, slots).
__device__ __forceinline__ u32 codeSlot(u64 code, u32 slots)
{
    const u32 h = u32((code * 0x9E3779B97F4A7C15ull) >> 32);
    return u32((u64(h) * slots) >> 32);
}

__device__ __forceinline__ u32 nextSlot(u32 slot, u32 slots) { return slot + 1 < slots ? slot + 1 : 0u; }

// Begin indices of the cell `code` (9 values into b), or false.
__device__ __forceinline__ bool nodeBegins(const NodeTable &gt, u64 code, u32 (&b)[kGroupBegins])
{
    u32 slot = codeSlot(code, gt.slots);
    for (u32 probe = 0; probe < kCellProbes; ++probe)
    {
        // the key and the values in one 48-byte record: three 16-byte loads
        const uint4 *row = reinterpret_cast<const uint4 *>(gt.rows + size_t(slot) * kGroupRow);
        const uint4 r0 = __ldg(row), r1 = __ldg(row + 1), r2 = __ldg(row + 2);
        const u64 key = (u64(r0.y) << 32) | r0.x;
        b[0] = r0.z; b[1] = r0.w;
        b[2] = r1.x; b[3] = r1.y; b[4] = r1.z; b[5] = r1.w;
        b[6] = r2.x; b[7] = r2.y; b[8] = r2.z;
        if (key == code) return true;
        if (key == 0) return false;
        slot = nextSlot(slot, gt.slots);
    }
    return false;
}

// The row of cell `code`, entered if absent (nullptr if the probes run out;
// the table is sized so they do not).  Writers of one cell store the same
// values, so racing writers are harmless.
__device__ __forceinline__ u32 *nodeRow(const NodeTable &gt, u64 code)
{
    u32 slot = codeSlot(code, gt.slots);
    for (u32 probe = 0; probe < kCellProbes; ++probe)
    {
        u32 *row = gt.rows + size_t(slot) * kGroupRow;
        const u64 prev = atomicCAS(reinterpret_cast<unsigned long long *>(row), 0ull,
                                   static_cast<unsigned long long>(code));
        if (prev == 0ull || prev == code) return row + 2;  // the values follow the key
        slot = nextSlot(slot, gt.slots);
    }
    return nullptr;
}

// Begin indices of the 8 children of the cell [qKey, qKey + 8 * cr) (children
// at `level`, cr their range) among the keys P[lo, hi) of an enclosing cell:
// a count by digit for short ranges, lower bounds otherwise.
__device__ __forceinline__ void childBeginsWithin(const u64 *P, u32 lo, u32 hi, u64 qKey, unsigned level,
                                                  u32 (&b)[kGroupBegins])
{
    const u64 cr = octRange(level);
    const u64 qEnd = qKey + 8 * cr;
    const unsigned cShift = 3u * (kOctLevels - level);
    if (hi - lo <= kNFScanMax)
    {
        // 16-bit counters per digit in two registers (hi - lo <= kNFScanMax < 2^16)
        u32 below = 0;
        u64 lowDigits = 0, highDigits = 0;
        for (u32 t = lo; t < hi; ++t)
        {
            const u64 k = __ldg(P + t);
            if (k < qKey) ++below;
            else if (k < qEnd)
            {
                const unsigned d = unsigned(k >> cShift) & 7u;
                const u64 inc = u64(1) << (16 * (d & 3u));
                if (d < 4) lowDigits += inc;
                else highDigits += inc;
            }
        }
        b[0] = lo + below;
#pragma unroll
        for (int d = 0; d < 8; ++d)
            b[d + 1] = b[d] + u32(((d < 4 ? lowDigits : highDigits) >> (16 * (d & 3))) & 0xffffu);
        return;
    }
    const u32 n = hi - lo;
#pragma unroll
    for (int d = 0; d <= 8; ++d) b[d] = lo + lowerBound32(P + lo, n, qKey + u64(d) * cr);
}

// Enters the internal nodes above every leaf (All) or above the new leaves of
// the last pass: the child begin of each ancestor whose child the leaf
// starts (up the levels while the leaf is a first child), and the end of each
// ancestor the leaf ends (up the levels while it is a last child).  Every
// child of an internal node starts with some leaf and its last child ends
// with one, so all 9 values of every internal node are entered.  A complete
// sibling group (a parent whose 8 children are leaves, most internal nodes)
// is entered whole by its first leaf, which also walks on from the parent;
// its other leaves add nothing.
template <bool All>
static __global__ void __launch_bounds__(kRefreshThreads) nodeTableKernel(TreeBufs tb, NodeTable gt)
{
    const DeviceState *st = tb.st;
    if (halted(st)) return;
    const int a = st->activeBuffer;
    const int L = st->numLeaves;
    const u64 *K = tb.k(a);
    const u32 *B = tb.b(a);
    const int count = All ? L : st->dirtyCount;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
    {
        const int i = All ? j : tb.dirty[j];
        const u64 s = K[i];
        const unsigned lev = octLevel(K[i + 1] - s);
        if (lev < 1 || lev > kOctLevels) continue;
        unsigned first = lev, last = lev;  // levels the two walks start from
        u32 b1 = B[i + 1];
        // complete sibling group around the leaf?
        const unsigned d = octDigit(s, lev);
        const int i0 = i - int(d);
        const u64 pRange = octRange(lev - 1);
        const u64 pStart = s & ~(pRange - 1);
        if (i0 >= 0 && i0 + 8 <= L && K[i0] == pStart && K[i0 + 8] == pStart + pRange)
        {
            if (d != 0) continue;  // the first leaf enters the group
            u32 *row = nodeRow(gt, cellCode(pStart, lev - 1));
            if (row)
            {
#pragma unroll
                for (int k = 0; k < kGroupBegins; ++k) row[k] = B[i + k];
            }
            // the walks go on from the parent, which the first leaf starts and ends
            first = last = lev - 1;
            b1 = B[i + 8];
        }
        const u32 b0 = B[i];
        for (unsigned l = first; l >= 1; --l)
        {
            const unsigned dd = octDigit(s, l);
            u32 *row = nodeRow(gt, cellCode(s & ~(octRange(l - 1) - 1), l - 1));
            if (row) row[dd] = b0;
            if (dd != 0) break;
        }
        for (unsigned l = last; l >= 1; --l)
        {
            const unsigned dd = octDigit(s, l);
            if (dd != 7) break;
            u32 *row = nodeRow(gt, cellCode(s & ~(octRange(l - 1) - 1), l - 1));
            if (row) row[8] = b1;
        }
    }
}

// Begin indices of the parent-level cell Q at qKey (children at `level`)
// that is not an internal node: the child of its deepest entered ancestor
// that holds Q (Q itself, or the leaf Q lies in; or a cell that was one of
// them earlier) gives a short key range, in which Q's keys are counted.
// False if no ancestor is entered or its values are not a key range.
__device__ __forceinline__ bool beginsInside(const NodeTable &gt, const u64 *P, u32 n, u64 qKey, unsigned level,
                                             u32 (&b)[kGroupBegins])
{
    for (int l = int(level) - 2; l >= 0; --l)
    {
        u32 e[kGroupBegins];
        if (nodeBegins(gt, cellCode(qKey & ~(octRange(unsigned(l)) - 1), unsigned(l)), e))
        {
            const unsigned d = octDigit(qKey, unsigned(l) + 1);  // the child that holds Q
            u32 lo = e[0], hi = e[1];
#pragma unroll
            for (int k = 1; k < 8; ++k)
                if (unsigned(k) == d)
                {
                    lo = e[k];
                    hi = e[k + 1];
                }
            if (lo > hi || hi > n) return false;
            childBeginsWithin(P, lo, hi, qKey, level, b);
            return true;
        }
    }
    return false;
}

// Per-warp scratch of the units in flight.
// The 4 x 4 x 4 child-count blocks of a warp's units in shared memory.  The 8
// children of a unit read their 3 x 3 x 3 sub-blocks from offsets {0, 1, 4, 5,
// 16, 17, 20, 21} (plus a common offset), the same banks for every unit of a
// dense [unit][64] array; unit u starts at u * 64 + {0, 2, 8, 10}[u % 4] +
// 16 * (u / 4) instead, so the sub-block reads of 4 consecutive units (one
// warp instruction) fall in 32 distinct banks.
__host__ __device__ __forceinline__ int unitBlockBase(int u)
{
    return u * 64 + ((0xA820 >> (4 * (u & 3))) & 15) + 16 * (u >> 2);
}
constexpr int kUnitBlockWords = (kUnitBatch - 1) * 64 + 10 + 16 * ((kUnitBatch - 1) / 4) + 64;

struct UnitBlocks
{
    u32 mem[kUnitBlockWords];
    __device__ __forceinline__ u32 *operator[](int u) { return mem + unitBlockBase(u); }
};

struct UnitScratch
{
    u64 pStart[kUnitBatch], st0[kUnitBatch], st1[kUnitBatch], st2[kUnitBatch];
    u32 qtot[kUnitBatch][27];             // population of each Q
    u32 cx[kUnitBatch], cy[kUnitBatch], cz[kUnitBatch];
    u32 hintB[kUnitBatch];                // begin index of the unit's first leaf
    int childState[kUnitBatch], level[kUnitBatch], active[kUnitBatch];
    UnitBlocks block;
    u64 slowKey[kUnitBatch * 27];
    unsigned short slowItem[kUnitBatch * 27];  // unit * 27 + q
    unsigned char slowState[kUnitBatch * 27];
    int nSlow;
};

// Key and child Hilbert state of the parent-level cell at offset q around the
// parent of unit u.
// The same from the decoded path of the parent cell P (key pStart at level pl).
template <bool Hilbert>
__device__ __forceinline__ u64 neighbourCellOf(const CellPath &path, u64 pStart, unsigned pl, int q, int &qState,
                                               const unsigned char *sEnc, const unsigned char *sNext)
{
    const int dx = q % 3 - 1, dy = (q / 3) % 3 - 1, dz = q / 9 - 1;
    const u32 cube = 1u << (kOctLevels - pl);
    const u32 cx = path.x, cy = path.y, cz = path.z;
    const u32 x = (cx + u32(dx) * cube) & 0x1fffffu;
    const u32 y = (cy + u32(dy) * cube) & 0x1fffffu;
    const u32 z = (cz + u32(dz) * cube) & 0x1fffffu;
    qState = path.childState;
    const u32 diff = (x ^ cx) | (y ^ cy) | (z ^ cz);  // zero only when the wrap maps Q onto P
    if (diff == 0) return pStart;
    if constexpr (Hilbert)
    {
        // Q agrees with P on the levels above the first differing bit: keep
        // that key prefix and encode the suffix from P's state there
        const unsigned m = unsigned(__clz(diff)) - (32u - kOctLevels);
        const u64 word = m < 10 ? path.st0 : (m < 20 ? path.st1 : path.st2);
        int st = int((word >> (6 * (m < 10 ? m : (m < 20 ? m - 10 : m - 20)))) & 63u);
        u64 suffix = 0;
        for (unsigned k = m; k < pl; ++k)
        {
            const unsigned b = kOctLevels - 1 - k;
            const unsigned o = (((x >> b) & 1u) << 2) | (((y >> b) & 1u) << 1) | ((z >> b) & 1u);
            const int e = st * 8 + int(o);
            suffix = (suffix << 3) | sEnc[e];
            st = sNext[e];
        }
        qState = st;
        const unsigned keep = 3u * m;
        const u64 prefix = keep ? (pStart >> (63u - keep)) << (63u - keep) : 0ull;
        return prefix | (suffix << (3u * (kOctLevels - pl)));
    }
    else
    {
        return mortonKey(x, y, z);
    }
}

template <bool Hilbert, class Scratch>
__device__ __forceinline__ u64 neighbourCell(const Scratch &w, int u, int q, int &qState,
                                             const unsigned char *sEnc, const unsigned char *sNext)
{
    const CellPath path{w.cx[u], w.cy[u], w.cz[u], w.st0[u], w.st1[u], w.st2[u], w.childState[u]};
    return neighbourCellOf<Hilbert>(path, w.pStart[u], unsigned(w.level[u]) - 1, q, qState, sEnc, sNext);
}

// Where the children of the neighbour cell at offset q land in the unit's
// 4 x 4 x 4 block, per child state and digit: [Morton, Hilbert][q][state],
// 8 bits per digit (the block position, or 0xff for a child that does not
// touch P).  Filled once per device from the host.
__device__ u64 gDigitPos[2 * 27 * 48];

// Child counts of Q from its 9 begin indices (children in digit order) into
// the unit's block.
template <bool Hilbert>
__device__ __forceinline__ void childrenFromPacked(const u32 (&b)[kGroupBegins], int q, int qState, u32 *block)
{
    const u64 packed = gDigitPos[(Hilbert ? 27 * 48 : 0) + q * 48 + qState];
#pragma unroll
    for (int d = 0; d < 8; ++d)
    {
        const unsigned p = unsigned(packed >> (8 * d)) & 0xffu;
        if (p != 0xff) block[p] = b[d + 1] - b[d];
    }
}

// Near-field counts and group flags of the new leaves (All: of every leaf),
// after octBeginKernel and nodeTableKernel.  A run of empty leaves whose
// group is incomplete or empty needs no work (NF 0; an empty parent can
// always merge).
template <bool Hilbert, bool All>
static __global__ void __launch_bounds__(kRefreshThreads, 4)
    octNearFieldKernel(TreeBufs tb, KeyIndex idx, unsigned bucket, HilbertTables h, NodeTable gt)
{
    __shared__ unsigned char sEnc[48 * 8], sNext[48 * 8], sDec[48 * 8];
    __shared__ UnitScratch sWarp[kRefreshThreads / 32];
    DeviceState *st = tb.st;
    if (halted(st)) return;
    if constexpr (Hilbert)
    {
        for (int k = threadIdx.x; k < 48 * 8; k += blockDim.x)
        {
            sEnc[k] = h.enc[k];
            sNext[k] = h.encNext[k];
            sDec[k] = h.decOct[k];
        }
    }
    __syncthreads();
    const int a = st->activeBuffer;
    const int L = st->numLeaves;
    const u64 *K = tb.k(a);
    const u32 *B = tb.b(a);
    u32 *NF = tb.nf(a);
    u8 *Gf = tb.g(a);
    UnitScratch &w = sWarp[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned ltMask = (1u << lane) - 1u;
    const int warpsTotal = gridDim.x * (blockDim.x / 32);
    const int w0 = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int count = All ? L : st->dirtyCount;
    for (int base = w0 * 32; base < count; base += warpsTotal * 32)
    {
        const int j = base + lane;
        const bool valid = j < count;
        const int i = valid ? (All ? j : tb.dirty[j]) : 0;
        const u64 s = valid ? K[i] : 0;
        const unsigned lev = valid ? octLevel(K[i + 1] - s) : 0;
        const u32 c = valid ? B[i + 1] - B[i] : 0;
        const u64 pk = lev > 0 ? (s & ~(octRange(lev - 1) - 1)) : 0;
        const int iPrev = __shfl_up_sync(0xffffffffu, i, 1);
        const u64 pkPrev = __shfl_up_sync(0xffffffffu, pk, 1);
        const unsigned levPrev = __shfl_up_sync(0xffffffffu, lev, 1);
        const bool head = valid && (lane == 0 || i != iPrev + 1 || pk != pkPrev || lev != levPrev || lev == 0);
        const unsigned heads = __ballot_sync(0xffffffffu, head);
        const unsigned validMask = __ballot_sync(0xffffffffu, valid);
        const unsigned nonEmpty = __ballot_sync(0xffffffffu, c != 0);
        const int endLane = 32 - __clz(validMask);
        const int nUnits = __popc(heads);
        // this lane's unit (within the chunk) and, for heads, the unit's last lane + 1
        const int myUnit = valid ? __popc(heads & (ltMask | (1u << lane))) - 1 : -1;
        const unsigned later = heads & ~(ltMask | (1u << lane));
        const int runEnd = later ? __ffs(later) - 1 : endLane;
        CellPath path{0, 0, 0, 0, 0, 0, kHilbertStart};
        if (head && lev > 0) path = decodeCell<Hilbert>(pk, lev - 1, sNext, sDec);

        for (int b0 = 0; b0 < nUnits; b0 += kUnitBatch)
        {
            const int nb = min(kUnitBatch, nUnits - b0);
            // ---- set-up: the head lane of each unit of the batch
            if (head && myUnit >= b0 && myUnit < b0 + nb)
            {
                const int u = myUnit - b0;
                int act = 1;
                if (lev == 0)
                {
                    // the root leaf: all 27 periodic cells are the root itself
                    const u64 cr = c;
                    const u64 v = cr * cr * 27ull;
                    NF[i] = v > 0xffffffffull ? 0xffffffffu : u32(v);
                    act = 0;
                }
                else
                {
                    const unsigned runMask =
                        (runEnd == 32 ? 0xffffffffu : ((1u << runEnd) - 1u)) & ~((1u << lane) - 1u);
                    if ((nonEmpty & runMask) == 0)
                    {
                        // empty run: NF 0; the flag needs the Q's only if the parent holds particles
                        const u64 pRange = octRange(lev - 1);
                        const int i0 = completeGroup(K, L, i, lev, pk, pRange);
                        if (i0 < 0 || B[i0 + 8] == B[i0])
                        {
                            for (int t = 0; t < runEnd - lane; ++t) NF[i + t] = 0;
                            if (i0 >= 0) Gf[i0] = 1;
                            act = 0;
                        }
                    }
                }
                w.active[u] = act;
                w.pStart[u] = pk;
                w.level[u] = int(lev);
                w.cx[u] = path.x;
                w.cy[u] = path.y;
                w.cz[u] = path.z;
                w.st0[u] = path.st0;
                w.st1[u] = path.st1;
                w.st2[u] = path.st2;
                w.childState[u] = path.childState;
                w.hintB[u] = B[i];
            }
            if (lane == 0) w.nSlow = 0;
            __syncwarp();

            // ---- phase A: (unit, Q) pairs over the lanes; complete groups from the table
            const int items = nb * 27;
            for (int ib = 0; ib < items; ib += 32)
            {
                const int it = ib + lane;
                const int u = it / 27, q = it - (it / 27) * 27;
                bool slow = false;
                u64 qKey = 0;
                int qState = 0;
                if (it < items && w.active[u])
                {
                    qKey = neighbourCell<Hilbert>(w, u, q, qState, sEnc, sNext);
                    const unsigned level = unsigned(w.level[u]);
                    u32 gb[kGroupBegins];
                    if (nodeBegins(gt, cellCode(qKey, level - 1), gb))
                    {
                        childrenFromPacked<Hilbert>(gb, q, qState, w.block[u]);
                        const u32 total = gb[8] - gb[0];
                        w.qtot[u][q] = total;
                    }
                    else
                    {
                        slow = true;
                    }
                }
                const unsigned slowMask = __ballot_sync(0xffffffffu, slow);
                if (slow)
                {
                    const int k = w.nSlow + __popc(slowMask & ltMask);
                    w.slowKey[k] = qKey;
                    w.slowItem[k] = (unsigned short)it;
                    w.slowState[k] = (unsigned char)qState;
                }
                __syncwarp();
                if (lane == 0) w.nSlow += __popc(slowMask);
                __syncwarp();
            }

            // ---- phase B: the Q's that are not nodes, over the lanes: counted
            // inside the leaf that holds them
            const int nSlow = w.nSlow;
            for (int k = lane; k < nSlow; k += 32)
            {
                const int it = w.slowItem[k];
                const int u = it / 27, q = it - u * 27;
                const u64 qKey = w.slowKey[k];
                const unsigned level = unsigned(w.level[u]);
                const int qState = int(w.slowState[k]);
                u32 begins[kGroupBegins];
                if (!beginsInside(gt, idx.keys, u32(idx.n), qKey, level, begins))
                {
                    // no enclosing cell entered (not expected): search the keys
                    const u32 lo = idx.lowerNear<kNFGallop>(w.hintB[u], qKey);
                    const u32 hi = lowerFrom(idx, lo, qKey + octRange(level - 1));
                    childBeginsWithin(idx.keys, lo, hi, qKey, level, begins);
                }
                childrenFromPacked<Hilbert>(begins, q, qState, w.block[u]);
                w.qtot[u][q] = begins[8] - begins[0];
            }
            __syncwarp();

            // ---- phase C: every lane its own leaf; the head lane the group flag
            if (valid && myUnit >= b0 && myUnit < b0 + nb)
            {
                const int u = myUnit - b0;
                if (w.active[u])
                {
                    u32 out = 0;
                    if (c)
                    {
                        const unsigned d = octDigit(s, lev);
                        const unsigned o = Hilbert ? unsigned(sDec[w.childState[u] * 8 + int(d)]) : d;
                        const u32 *sub = w.block[u] + (o >> 2) * 16 + ((o >> 1) & 1u) * 4 + (o & 1u);
                        u64 pop = 0;
                        if (lev > 1)
                        {
                            u32 p32 = 0;
#pragma unroll
                            for (int x = 0; x < 3; ++x)
#pragma unroll
                                for (int y = 0; y < 3; ++y)
#pragma unroll
                                    for (int z = 0; z < 3; ++z) p32 += sub[x * 16 + y * 4 + z];
                            pop = p32;
                        }
                        else
                        {
                            // level 1: the periodic wrap repeats cells, the sum may exceed 2^32
                            for (int x = 0; x < 3; ++x)
                                for (int y = 0; y < 3; ++y)
                                    for (int z = 0; z < 3; ++z) pop += sub[x * 16 + y * 4 + z];
                        }
                        const u64 v = u64(c) * pop;
                        out = v > 0xffffffffull ? 0xffffffffu : u32(v);
                    }
                    NF[i] = out;
                    if (head)
                    {
                        const int i0 = completeGroup(K, L, i, lev, pk, octRange(lev - 1));
                        if (i0 >= 0)
                        {
                            u64 qsum = 0;
                            for (int q = 0; q < 27; ++q) qsum += w.qtot[u][q];
                            Gf[i0] = u64(w.qtot[u][13]) * qsum <= u64(bucket) ? 1 : 0;
                        }
                    }
                }
            }
            __syncwarp();
        }
    }
}

// N[i] = B[i+1] - B[i] on the active buffer.
static __global__ void materializeCountsKernel(TreeBufs tb)
{
    const DeviceState *st = tb.st;
    const int a = st->activeBuffer, L = st->numLeaves;
    const u32 *B = tb.b(a);
    u32 *N = tb.n(a);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L; i += gridDim.x * blockDim.x) N[i] = B[i + 1] - B[i];
}

// --------------------------------------------------------------------------
// Binary (kdtree3d_rebalance.cuh:61-125)
// --------------------------------------------------------------------------
struct BinaryOp
{
    const u64 *K;
    const u32 *B;
    unsigned bucket, maxDepth;
    __device__ __forceinline__ bool siblings(int L, int first) const  // binarySiblings, binary_node.cuh:91-98
    {
        if (first < 0 || first + 1 >= L) return false;
        const u64 r = K[first + 1] - K[first];
        return !(K[first] & r) && K[first + 2] - K[first + 1] == r;
    }
    __device__ __forceinline__ int operator()(int i, int L) const
    {
        const u32 ci = B[i + 1] - B[i];
        const bool merge = i && siblings(L, i - 1) && u64(B[i] - B[i - 1]) + ci <= bucket;
        if (merge) return 0;
        return (ci > bucket && unsigned(clz64(K[i + 1] - K[i])) < maxDepth) ? 2 : 1;
    }
};

static __global__ void __launch_bounds__(kScanThreads) binDecideScanKernel(TreeBufs tb, unsigned bucket, unsigned maxDepth)
{
    const int a = tb.st->activeBuffer;
    const BinaryOp op{tb.k(a), tb.b(a), bucket, maxDepth};
    decideScan(op, tb);
}

static __global__ void __launch_bounds__(kScatterThreads)
    binScatterKernel(TreeBufs tb, long long limit, int mode)
{
    DeviceState *st = tb.st;
    if (halted(st)) return;
    const long long total = st->proposal;
    const bool proceed = !st->needsResize && st->changed && total <= limit;
    if (proceed)
    {
        const int L = st->numLeaves;
        const int a = st->activeBuffer, b = a ^ 1;
        const int lane = threadIdx.x & 31;
        const int warpsTotal = gridDim.x * (blockDim.x / 32);
        const int w0 = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
        for (int base = w0 * 32; base < L; base += warpsTotal * 32)
        {
            const int i = base + lane;
            int nDirty = 0;
            i64 ni = 0;
            if (i < L)
            {
                const int op = opAt(tb.offs, i);
                if (op)
                {
                    ni = tb.offs[i];
                    const u64 s = tb.k(a)[i];
                    tb.k(b)[ni] = s;
                    tb.b(b)[ni] = tb.b(a)[i];
                    if (op == 2)
                    {
                        tb.k(b)[ni + 1] = s + (tb.k(a)[i + 1] - s) / 2;
                        nDirty = 1;
                    }
                }
                if (i == 0)
                {
                    tb.k(b)[total] = kMaxKey;
                    tb.b(b)[total] = st->numActiveParticles;
                }
            }
            const int d0 = warpAppend(&st->dirtyCount, nDirty);
            if (nDirty) tb.dirty[d0] = int(ni) + 1;
        }
    }
    commitIfLast(st, limit, mode, true, nullptr);
}

// Binary count refresh: B of new split points (All: every boundary).  The
// reference counts over the active prefix of P (binaryLeafCountsKernel,
// kdtree3d_rebalance.cuh:127-138); lower bounds of keys below 2^63 agree.
template <bool All>
static __global__ void binRefreshKernel(TreeBufs tb, KeyIndex idx)
{
    DeviceState *st = tb.st;
    if (halted(st)) return;
    const int a = st->activeBuffer, L = st->numLeaves;
    const u64 *K = tb.k(a);
    u32 *B = tb.b(a);
    if (All && blockIdx.x == 0 && threadIdx.x == 0) B[L] = st->numActiveParticles;
    const int count = All ? L : st->dirtyCount;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
    {
        const int i = All ? j : tb.dirty[j];
        B[i] = u32(idx.lower(K[i]));
    }
}

// Reset at the start of update() (resetRebalanceStateKernel,
// octree_rebalance.cuh:62-73): changed, converged and the active count.
// One warp (the active count by a warp-wide search).
static __global__ void resetForUpdateKernel(DeviceState *st, const u64 *P, size_t n)
{
    const unsigned active = n ? warpLowerBound(P, 0, u32(n), kMaxKey, int(threadIdx.x & 31)) : 0u;
    if (threadIdx.x != 0) return;
    st->changed = 0;
    st->converged = 0;
    st->numActiveParticles = active;
    st->dirtyCount = 0;
    st->updatePasses = 0;
}

// Per-pass reset of the flags the decision accumulates.
static __global__ void beginPassKernel(DeviceState *st)
{
    st->changed = 0;
    st->dirtyCount = 0;
}

// Sample every kSampleStride-th key for KeyIndex.
static __global__ void sampleKeysKernel(const u64 *P, size_t n, u64 *sample, size_t ns)
{
    for (size_t j = blockIdx.x * size_t(blockDim.x) + threadIdx.x; j < ns; j += size_t(gridDim.x) * blockDim.x)
        sample[j] = P[j << kSampleShift];
}

}  // namespace rb
}  // namespace aot
