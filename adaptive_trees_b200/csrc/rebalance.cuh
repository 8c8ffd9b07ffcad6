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
// aggregate.  Called by one thread.
__device__ __forceinline__ i64 lookback(u64 *status, u32 tile, i64 aggregate, int *error)
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
            if (++spins > kLookbackSpins)
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
    int nDirty = 0, op = 0;
    i64 ni = 0;
    if (i < L)
    {
        const u64 *K = tb.k(a);
        const i64 *offs = tb.offs;
        op = opAt(offs, i);
        const u64 start = K[i];
        const unsigned level = octLevel(K[i + 1] - start);
        ni = offs[i];
        u64 *Kn = tb.k(b);
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
            const u64 nr = octRange(level + splitLevels(op));
            for (int c = 0; c < op; ++c) Kn[ni + c] = start + u64(c) * nr;
            Bn[ni] = tb.b(a)[i];  // the first child starts where the parent did
            nDirty = NF ? op : op - 1;
        }
        if (i == 0)
        {
            Kn[total] = kMaxKey;
            Bn[total] = st->numActiveParticles;
        }
    }
    // work lists (warp-aggregated appends; list order is irrelevant)
    const int d0 = warpAppend(&st->dirtyCount, nDirty);
    if (nDirty)
    {
        if (op > 1)
        {
            const int c0 = NF ? 0 : 1;
            for (int c = c0; c < op; ++c) tb.dirty[d0 + c - c0] = int(ni) + c;
        }
        else
        {
            tb.dirty[d0] = int(ni);
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

// Near-field counts by parent cell.
//
// NF(leaf) = own x (population of the 27 periodic same-level cells around the
// leaf) (computeNFCooperative, octree_rebalance.cuh:579-634), and a complete
// sibling group may merge when parent count x (population of the 27 cells
// around the parent, one level up) <= bucket (computeGroupCanMergeKernel,
// octree_rebalance.cuh:636-700).  Both depend only on the particles, not on
// the tree, so they are computed per parent cell P at level l-1 (a "unit"):
//   * the 27 parent-level cells Q around P (P included) are found by two
//     lower bounds each, one lane per Q;
//   * the 8 children of P have their 27-cell stencils inside the 4 x 4 x 4
//     block of level-l cells around P, and that block is partitioned by the
//     children of the Q's that touch P (per axis: offset -1 gives the upper
//     child, 0 both, +1 the lower): each lane counts its Q's particles into
//     its block positions (a scan of a short range, or binary searches of
//     its child boundaries when the range is long);
//   * each leaf of P sums its 3 x 3 x 3 sub-block, and the group flag is the
//     sum of the 27 Q populations.
// Periodic wrap at low levels makes several offsets name the same cell;
// every offset is counted, as in the per-leaf stencil.  One warp per unit:
// 54 lower bounds serve up to 8 leaves and the group flag.
constexpr u32 kNFScanMax = 256;  // Q ranges up to this length are scanned
constexpr int kNFGallop = 4;     // gallop window of the Q searches: 15 keys from the last unit's

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

__device__ __forceinline__ CellPath shflPath(const CellPath &c, int src)
{
    CellPath r;
    r.x = __shfl_sync(0xffffffffu, c.x, src);
    r.y = __shfl_sync(0xffffffffu, c.y, src);
    r.z = __shfl_sync(0xffffffffu, c.z, src);
    r.st0 = __shfl_sync(0xffffffffu, c.st0, src);
    r.st1 = __shfl_sync(0xffffffffu, c.st1, src);
    r.st2 = __shfl_sync(0xffffffffu, c.st2, src);
    r.childState = __shfl_sync(0xffffffffu, c.childState, src);
    return r;
}

// One unit: the leaves h..h+run-1 (children of the parent P at level
// level-1, decoded in `pp`) and the group flag of P's complete group.
// sPos[q * 8 + o] is the block position of child octant o of the Q at lane q,
// or 0xff where that child does not touch P.
template <bool Hilbert>
__device__ __forceinline__ void nearFieldUnit(const KeyIndex &idx, u32 *block, const u64 *K, const u32 *B, u32 *NF,
                                              u8 *G, int L, unsigned bucket, int h, int run, unsigned level,
                                              const CellPath &pp, u32 &hint, const unsigned char *sEnc,
                                              const unsigned char *sNext, const unsigned char *sDec,
                                              const unsigned char *sPos)
{
    const int lane = threadIdx.x & 31;
    const unsigned pl = level - 1;  // parent level
    const u64 pRange = octRange(pl);
    const u64 pStart = K[h] & ~(pRange - 1);

    // lane q < 27: the parent-level cell Q at offset (q%3-1, q/3%3-1, q/9-1)
    u32 lo = 0, hi = 0;
    if (lane < 27)
    {
        const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
        const u32 cube = 1u << (kOctLevels - pl);
        const u32 x = (pp.x + u32(dx) * cube) & 0x1fffffu;
        const u32 y = (pp.y + u32(dy) * cube) & 0x1fffffu;
        const u32 z = (pp.z + u32(dz) * cube) & 0x1fffffu;
        u64 qKey = pStart;
        int qState = pp.childState;  // Hilbert state of Q's children
        const u32 diff = (x ^ pp.x) | (y ^ pp.y) | (z ^ pp.z);  // zero only when the wrap maps Q onto P
        if (diff != 0)
        {
            if constexpr (Hilbert)
            {
                // Q agrees with P on the levels above the first differing bit:
                // keep that key prefix and encode the suffix from P's state there
                const unsigned m = unsigned(__clz(diff)) - (32u - kOctLevels);
                const u64 word = m < 10 ? pp.st0 : (m < 20 ? pp.st1 : pp.st2);
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
                qKey = prefix | (suffix << (3u * (kOctLevels - pl)));
            }
            else
            {
                qKey = mortonKey(x, y, z);
            }
        }
        lo = idx.lowerNear<kNFGallop>(hint, qKey);
        hi = lowerFrom(idx, lo, qKey + pRange);
        hint = lo;

        const unsigned char *pos = sPos + lane * 8;
        const u32 n = hi - lo;
        const unsigned cShift = 3u * (kOctLevels - level);
        const u64 *P = idx.keys + lo;
        if (n <= kNFScanMax)
        {
            // count Q's particles per child octant in registers: 16-bit fields
            // (n <= kNFScanMax < 2^16) of two words; the child digit maps to its
            // octant through a 3-bit-per-digit word built once for Q's state
            u32 octOf = 0;
            if constexpr (Hilbert)
            {
#pragma unroll
                for (int d = 0; d < 8; ++d) octOf |= u32(sDec[qState * 8 + d]) << (3 * d);
            }
            u64 lowOcts = 0, highOcts = 0;
            for (u32 t = 0; t < n; ++t)
            {
                const unsigned d = unsigned(__ldg(P + t) >> cShift) & 7u;
                const unsigned o = Hilbert ? (octOf >> (3 * d)) & 7u : d;
                const u64 inc = u64(1) << (16 * (o & 3u));
                if (o < 4) lowOcts += inc;
                else highOcts += inc;
            }
#pragma unroll
            for (int o = 0; o < 8; ++o)
                if (pos[o] != 0xff) block[pos[o]] = u32(((o < 4 ? lowOcts : highOcts) >> (16 * (o & 3))) & 0xffffu);
        }
        else
        {
            const u64 cr = octRange(level);
#pragma unroll 1
            for (int o = 0; o < 8; ++o)
            {
                const unsigned p = pos[o];
                if (p == 0xff) continue;
                const unsigned dg = Hilbert ? unsigned(sEnc[qState * 8 + o]) : unsigned(o);
                const u64 cs = qKey + u64(dg) * cr;
                block[p] = lowerBound32(P, n, cs + cr) - lowerBound32(P, n, cs);
            }
        }
    }
    __syncwarp();

    // the unit's leaves: own count x population of the 3 x 3 x 3 sub-block
    // (27 distinct cells, so at most n < 2^32, except at level 1 where the
    // periodic wrap repeats cells)
    if (lane < run)
    {
        const int i = h + lane;
        const u32 c = B[i + 1] - B[i];
        u32 out = 0;
        if (c)
        {
            const unsigned d = octDigit(K[i], level);
            const unsigned o = Hilbert ? unsigned(sDec[pp.childState * 8 + int(d)]) : d;
            const u32 *sub = block + (o >> 2) * 16 + ((o >> 1) & 1u) * 4 + (o & 1u);
            u64 pop;
            if (level > 1)
            {
                u32 p32 = 0;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b)
#pragma unroll
                        for (int e = 0; e < 3; ++e) p32 += sub[a * 16 + b * 4 + e];
                pop = p32;
            }
            else
            {
                pop = 0;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        for (int e = 0; e < 3; ++e) pop += sub[a * 16 + b * 4 + e];
            }
            const u64 v = u64(c) * pop;
            out = v > 0xffffffffull ? 0xffffffffu : u32(v);
        }
        NF[i] = out;
    }

    // group flag of a complete group: parent count x population around the parent
    u64 qpop = lane < 27 ? u64(hi - lo) : 0;
    for (int off = 16; off > 0; off >>= 1) qpop += __shfl_xor_sync(0xffffffffu, qpop, off);
    const u32 pc = __shfl_sync(0xffffffffu, hi - lo, 13);
    if (lane == 0)
    {
        const int i0 = completeGroup(K, L, h, level, pStart, pRange);
        if (i0 >= 0) G[i0] = u64(pc) * qpop <= u64(bucket) ? 1 : 0;
    }
    __syncwarp();
}

// Near-field counts and group flags of the new leaves (All: of every leaf),
// after octBeginKernel.  Each warp takes 32 list entries at a time, cuts them
// into runs of consecutive leaves with the same parent, decodes the runs'
// parents lane-parallel and processes each run as one unit.  A run of empty
// leaves whose group is incomplete or empty needs no search (NF 0; an empty
// parent can always merge).
template <bool Hilbert, bool All>
static __global__ void __launch_bounds__(kRefreshThreads)
    octNearFieldKernel(TreeBufs tb, KeyIndex idx, unsigned bucket, HilbertTables h)
{
    __shared__ unsigned char sEnc[48 * 8], sNext[48 * 8], sDec[48 * 8], sPos[27 * 8];
    __shared__ u32 sBlock[kRefreshThreads / 32][64];
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
    for (int k = threadIdx.x; k < 27 * 8; k += blockDim.x)
    {
        // per axis: offset -1 touches P with its upper child, 0 with both, +1 with its lower;
        // block coordinate 2 * offset + child bit + 1
        const int q = k >> 3, o = k & 7;
        const int d[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
        const int bit[3] = {o >> 2, (o >> 1) & 1, o & 1};
        bool ok = true;
        int p = 0;
        for (int ax = 0; ax < 3; ++ax)
        {
            if ((d[ax] < 0 && bit[ax] == 0) || (d[ax] > 0 && bit[ax] == 1)) ok = false;
            p = p * 4 + (2 * d[ax] + bit[ax] + 1);
        }
        sPos[k] = ok ? (unsigned char)p : (unsigned char)0xff;
    }
    __syncthreads();
    const int a = st->activeBuffer;
    const int L = st->numLeaves;
    const u64 *K = tb.k(a);
    const u32 *B = tb.b(a);
    u32 *NF = tb.nf(a);
    u8 *Gf = tb.g(a);
    u32 *block = sBlock[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int warpsTotal = gridDim.x * (blockDim.x / 32);
    const int w0 = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int count = All ? L : st->dirtyCount;
    u32 hint = 0;
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
        unsigned heads = __ballot_sync(0xffffffffu, head);
        const unsigned validMask = __ballot_sync(0xffffffffu, valid);
        const unsigned nonEmpty = __ballot_sync(0xffffffffu, c != 0);
        const int endLane = 32 - __clz(validMask);
        // decode the parents of all runs at once (head lanes)
        CellPath path{0, 0, 0, 0, 0, 0, kHilbertStart};
        if (head && lev > 0) path = decodeCell<Hilbert>(pk, lev - 1, sNext, sDec);
        while (heads)
        {
            const int hl = __ffs(heads) - 1;
            heads &= heads - 1;
            const int next = heads ? __ffs(heads) - 1 : endLane;
            const int hIdx = __shfl_sync(0xffffffffu, i, hl);
            const unsigned lv = __shfl_sync(0xffffffffu, lev, hl);
            const int run = next - hl;
            if (lv == 0)
            {
                // the root leaf: all 27 periodic cells are the root itself
                if (lane == 0)
                {
                    const u64 cr = B[hIdx + 1] - B[hIdx];
                    const u64 v = cr * cr * 27ull;
                    NF[hIdx] = v > 0xffffffffull ? 0xffffffffu : u32(v);
                }
                continue;
            }
            const unsigned runMask = (next == 32 ? 0xffffffffu : ((1u << next) - 1u)) & ~((1u << hl) - 1u);
            if ((nonEmpty & runMask) == 0)
            {
                // empty run: NF 0; the group flag needs a search only if the parent holds particles
                const u64 pRange = octRange(lv - 1);
                const u64 pStart = __shfl_sync(0xffffffffu, s, hl) & ~(pRange - 1);
                int i0 = -1;
                if (lane == 0) i0 = completeGroup(K, L, hIdx, lv, pStart, pRange);
                i0 = __shfl_sync(0xffffffffu, i0, 0);
                const bool parentEmpty = i0 < 0 || B[i0 + 8] == B[i0];
                if (parentEmpty)
                {
                    if (lane >= hl && lane < next) NF[i] = 0;
                    if (lane == 0 && i0 >= 0) Gf[i0] = 1;
                    continue;
                }
            }
            const CellPath pp = shflPath(path, hl);
            nearFieldUnit<Hilbert>(idx, block, K, B, NF, Gf, L, bucket, hIdx, run, lv, pp, hint, sEnc, sNext, sDec,
                                   sPos);
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
static __global__ void resetForUpdateKernel(DeviceState *st, const u64 *P, size_t n)
{
    st->changed = 0;
    st->converged = 0;
    st->numActiveParticles = n ? u32(lowerBoundDev(P, n, kMaxKey)) : 0u;
    st->dirtyCount = 0;
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
