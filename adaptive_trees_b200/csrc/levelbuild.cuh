// levelbuild.cuh -- device kernels of the converged octree build.
//
// The reference builds an octree from the root by rounds of split/merge
// decisions until a round changes nothing (rebalanceBuild, octree.cu:159-180;
// calculateNodeOp, octree_rebalance.cuh:174-249).  The decision value of a
// cell -- its particle count (LeafCount) or its near-field count NF = count x
// population of the 27 periodic same-level cells around it (NFCount,
// octree_rebalance.cuh:579-634) -- depends only on the particles, and it
// never grows from a cell to its children.  So the tree the rounds converge
// to is unique: a cell is an internal node exactly when its value exceeds the
// bucket and its level is below 21.  This file builds that tree one level at
// a time, without the rounds:
//   expand    the internal cells ("units") of level l get the begin indices
//             of their 8 children in the sorted keys (and, for NFCount, a row
//             in the node table of the near-field lookups);
//   nearField NFCount: the near-field counts of the children of the level-l
//             units, one unit per parent cell as in the refresh of the
//             rounds (octNearFieldKernel);
//   classify  the children whose value exceeds the bucket become the units of
//             level l + 1 (slots taken by warp-aggregated atomics); the
//             others are leaves of the tree;
//   leafCount, place: subtree leaf counts bottom-up, then every leaf's
//             position in the cornerstone array top-down.
//
// The capacity the reference ends with depends on how many leaves each round
// proposed (resizeWithHeadroom history, octree.cu:159-180 and 453-457).  That
// history follows from the same cells: the rounds start at the root; a leaf
// whose value exceeds the bucket splits in the next round by 1-4 levels at
// once (the level jump of calculateNodeOp), and a group of 8 leaves whose
// parent does not exceed it merges.  Call a cell reached by a split "landed"
// and the levels a split spans its "region".  A landed cell arrives at round
// a; if it is an internal node it splits at once, and its region's 8^k cells
// arrive at round a + 1; every leaf f of the final tree in that region, at
// relative depth j <= k, is then represented by its 8^(k-j) descendants at
// the landing level, which merge up one level per round, so f stands for
// 8^max(0, k - (t - a - 1) - j) leaves at round t >= a + 1.  The classify
// kernel counts the final leaves per (a, k, j) and the landed internal nodes
// per round; the host sums the leaf counts of every round from them.
#pragma once

#include "rebalance.cuh"

namespace aot
{
namespace lb
{
constexpr int kThreads = 256;
constexpr u32 kLeaf = 0xffffffffu;     // child slot: the child is a leaf
constexpr int kArrivals = 32;          // arrival rounds tracked (>= kOctLevels + 2)
constexpr int kJumps = 5;              // split depth k = 1..4
constexpr int kContribBins = kArrivals * kJumps * kJumps;
constexpr int kRow = rb::kGroupRow;    // unit row: key (2 words), 9 child begins, region word

// Device control block of one build.
struct Control
{
    u32 levelStart[kOctLevels + 2];
    u32 levelCount[kOctLevels + 2];
    int overflow;       // the unit arena is too small
    int late;           // an arrival round beyond the tracked ones
    int error;          // reserved (the level build has no waits)
    int placeOverflow;  // the tree has more leaves than the cornerstone buffers hold
};

// The unit arena: units of all levels, level l at
// [levelStart[l], levelStart[l] + levelCount[l]).
struct Arena
{
    u32 *rows;       // [cap][kRow]
    u32 *val;        // [cap][8] value of each child (NF or count)
    u32 *child;      // [cap][8] unit index of an internal child, or kLeaf
    u32 *leaves;     // [cap] leaves in the unit's subtree
    u32 *offset;     // [cap] cornerstone index of the unit's first leaf
    u32 *nbr;        // NFCount: [cap][27] the cells around each unit (nbrRef)
    u32 *parent;     // NFCount: [cap] parent unit * 8 + the unit's digit in it
    u32 *usys;       // batch of trees: [cap] the tree (system) of each unit
    u32 *sysRoot;    // batch of trees: [systems] each system's root unit, or kLeaf
    Control *ctl;
    unsigned long long *contrib;  // [kArrivals][kJumps][kJumps] final leaves per (a, k, j)
    unsigned long long *landed;   // [kArrivals] internal nodes landing in round t
    u32 cap;
};

// Region word of a unit, describing the region its children belong to:
// arrival round of the region's landed cell (8 bits), that cell's level
// (5 bits) and the region's depth k (3 bits).
__host__ __device__ __forceinline__ u32 regionWord(u32 a, u32 level, u32 k) { return a | (level << 8) | (k << 16); }
__device__ __forceinline__ u32 regionArrival(u32 w) { return w & 0xffu; }
__device__ __forceinline__ u32 regionLevel(u32 w) { return (w >> 8) & 0x1fu; }
__device__ __forceinline__ u32 regionDepth(u32 w) { return (w >> 16) & 7u; }
// The same word also holds the unit's own level (bits 19-23) and the curve
// state that orders its children (bits 24-29, Hilbert).
__host__ __device__ __forceinline__ u32 withUnit(u32 region, u32 level, u32 state)
{
    return (region & 0x7ffffu) | (level << 19) | (state << 24);
}
__device__ __forceinline__ u32 unitLevelOf(u32 w) { return (w >> 19) & 0x1fu; }
__device__ __forceinline__ u32 unitStateOf(u32 w) { return (w >> 24) & 0x3fu; }

// A cell around a unit, at the unit's level: a unit index when the cell is an
// internal node, else kLeafRef | (parent unit * 8 + digit) naming the leaf
// of the tree that holds the cell (the cell itself or a coarser leaf).
constexpr u32 kLeafRef = 0x80000000u;

// Levels a leaf of value x at level m splits by (calculateNodeOp,
// octree_rebalance.cuh:188-249: 8, 64, 512 or 4096 children), given that it
// splits (x > bucket, m < 21).  LeafCount compares with 32-bit products of
// the bucket, NFCount with 64-bit ones.
__host__ __device__ __forceinline__ u32 splitDepth(bool nf, u32 x, u32 bucket, unsigned m)
{
    if (nf)
    {
        const u64 c = x, b = bucket;
        if (c > b * 262144 && m + 3 < kOctLevels) return 4;
        if (c > b * 4096 && m + 2 < kOctLevels) return 3;
        if (c > b * 64 && m + 1 < kOctLevels) return 2;
        return 1;
    }
    if (x > bucket * 512u && m + 3 < kOctLevels) return 4;
    if (x > bucket * 64u && m + 2 < kOctLevels) return 3;
    if (x > bucket * 8u && m + 1 < kOctLevels) return 2;
    return 1;
}

__device__ __forceinline__ u64 rowKey(const u32 *row) { return (u64(row[1]) << 32) | row[0]; }

// The root: a unit at level 0 when its value exceeds the bucket (NF of the
// root: 27 x count^2, clamped, octree.cu:23-38), else the whole tree is the
// root leaf, written straight to the cornerstone buffers.
// One warp: the active count by a warp-wide search, then lane 0.
static __global__ void rootKernel(Arena a, rb::TreeBufs tb, const u64 *P, size_t n, unsigned bucket, int nf)
{
    DeviceState *st = tb.st;
    const unsigned active = n ? warpLowerBound(P, 0, u32(n), kMaxKey, int(threadIdx.x & 31)) : 0u;
    if (threadIdx.x != 0) return;
    const u64 sq = u64(active) * active;
    const u32 nfRoot = sq > 0xffffffffull / 27ull ? 0xffffffffu : u32(27ull * sq);
    const u32 x = nf ? nfRoot : active;
    const int err = st->error;
    *st = DeviceState{};
    st->error = err;
    st->numActiveParticles = active;
    Control &c = *a.ctl;
    c.levelStart[0] = 0;
    if (x > bucket)
    {
        u32 *row = a.rows;
        row[0] = 0;
        row[1] = 0;
        row[2] = 0;
        row[10] = active;
        row[11] = withUnit(regionWord(0, 0, splitDepth(nf != 0, x, bucket, 0)), 0, kHilbertStart);
        c.levelCount[0] = 1;
        a.offset[0] = 0;
        if (nf)
        {
            // every cell around the root is the root (periodic wrap)
            for (int q = 0; q < 27; ++q) a.nbr[q] = 0;
            a.parent[0] = kLeaf;
        }
        st->numLeaves = 0;  // set when the tree is placed
    }
    else
    {
        c.levelCount[0] = 0;
        tb.K[0][0] = 0;
        tb.K[0][1] = kMaxKey;
        tb.B[0][0] = 0;
        tb.B[0][1] = active;
        tb.NF[0][0] = nf ? nfRoot : 0u;
        tb.N[0][0] = active;
        st->numLeaves = 1;
    }
}

// Lower bounds of the 7 inner child boundaries key + (d + 1) * cr of a unit
// whose keys are P[lo, hi), searched side by side (7 independent loads per
// step): first among the sampled keys (every 32nd key, a small array that
// stays in L2), then in the window of at most 31 keys the sample leaves.
__device__ __forceinline__ void innerBegins(const KeyIndex &idx, u32 lo, u32 hi, u64 key, u64 cr, u32 (&b)[7])
{
    const u32 jA = (lo + kSampleStride - 1) >> kSampleShift, jB = (hi + kSampleStride - 1) >> kSampleShift;
    u32 len[7];
#pragma unroll
    for (int d = 0; d < 7; ++d)
    {
        b[d] = jA;
        len[d] = jB > jA ? jB - jA : 0;
    }
    for (;;)  // first sample >= target among samples jA..jB-1
    {
        u32 live = 0;
#pragma unroll
        for (int d = 0; d < 7; ++d) live |= len[d];
        if (!live) break;
#pragma unroll
        for (int d = 0; d < 7; ++d)
        {
            if (len[d])
            {
                const u32 half = len[d] >> 1;
                const bool less = __ldg(idx.sample + b[d] + half) < key + u64(d + 1) * cr;
                b[d] = less ? b[d] + half + 1 : b[d];
                len[d] = less ? len[d] - half - 1 : half;
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 7; ++d)
    {
        // the answer lies after the last sample below the target and at or
        // before the first one at or above it
        const u32 wlo = b[d] > jA ? ((b[d] - 1) << kSampleShift) + 1 : lo;
        const u32 whi = b[d] < jB ? (b[d] << kSampleShift) : hi;
        len[d] = whi > wlo ? whi - wlo : 0;  // empty unless the keys are sorted (a failed sort stays in bounds)
        b[d] = wlo;
    }
    for (;;)
    {
        u32 live = 0;
#pragma unroll
        for (int d = 0; d < 7; ++d) live |= len[d];
        if (!live) break;
#pragma unroll
        for (int d = 0; d < 7; ++d)
        {
            if (len[d])
            {
                const u32 half = len[d] >> 1;
                const bool less = __ldg(idx.keys + b[d] + half) < key + u64(d + 1) * cr;
                b[d] = less ? b[d] + half + 1 : b[d];
                len[d] = less ? len[d] - half - 1 : half;
            }
        }
    }
}

// Levels with at most this many units expand by warps (a warp per inner
// child boundary); the chains of dependent loads of the per-thread searches
// dominate there, and the keys of a unit span most of the array.
constexpr u32 kWideUnits = 4096;
// Up to this many units, a lane per inner boundary (8 lanes per unit): more
// searches in flight where the units are too few to fill the GPU one thread
// each.
constexpr u32 kLaneUnits = 1u << 18;

// Lower bound of t among the keys P[lo, hi): first among the sampled keys in
// the range, then in the window of at most 31 keys they leave.
__device__ __forceinline__ u32 boundaryIn(const KeyIndex &idx, u32 lo, u32 hi, u64 t)
{
    const u32 jA = (lo + kSampleStride - 1) >> kSampleShift, jB = (hi + kSampleStride - 1) >> kSampleShift;
    u32 b = jA, len = jB > jA ? jB - jA : 0;
    while (len)
    {
        const u32 half = len >> 1;
        const bool less = __ldg(idx.sample + b + half) < t;
        b = less ? b + half + 1 : b;
        len = less ? len - half - 1 : half;
    }
    const u32 wlo = b > jA ? ((b - 1) << kSampleShift) + 1 : lo;
    const u32 whi = b < jB ? (b << kSampleShift) : hi;
    b = wlo;
    len = whi > wlo ? whi - wlo : 0;
    while (len)
    {
        const u32 half = len >> 1;
        const bool less = __ldg(idx.keys + b + half) < t;
        b = less ? b + half + 1 : b;
        len = less ? len - half - 1 : half;
    }
    return b;
}

// 9 child begins of the units of level l: one thread per unit (the 7 inner
// ones by innerBegins), one lane per inner boundary on levels of fewer units,
// one warp per inner boundary on levels of few units.
// `rank` and `size` number the threads taking part (a grid, or the grid of a
// persistent kernel).
__device__ __forceinline__ void expandUnits(const Arena &a, const KeyIndex &idx, int l, u32 start, u32 count, u32 rank,
                                            u32 size)
{
    const u64 cr = octRange(unsigned(l) + 1);
    if (count <= kWideUnits)
    {
        const int lane = threadIdx.x & 31;
        for (u32 w = rank >> 5; w < count * 7; w += size >> 5)
        {
            const u32 i = w / 7, d = w - i * 7;
            u32 *row = a.rows + size_t(start + i) * kRow;
            const u32 lo = row[2], hi = row[10];
            const u64 t = rowKey(row) + u64(d + 1) * cr;
            // first sampled key >= t among the samples inside [lo, hi), then
            // the window of at most 31 keys before it
            const u32 jA = (lo + kSampleStride - 1) >> kSampleShift, jB = (hi + kSampleStride - 1) >> kSampleShift;
            const u32 sIdx = warpLowerBound(idx.sample, jA, jB > jA ? jB : jA, t, lane);
            const u32 wlo = sIdx > jA ? ((sIdx - 1) << kSampleShift) + 1 : lo;
            const u32 whi = sIdx < jB ? (sIdx << kSampleShift) : hi;
            const u32 r = warpLowerBound(idx.keys, wlo, whi, t, lane);
            if (lane == 0) row[3 + d] = r;
        }
        return;
    }
    if (count <= kLaneUnits)
    {
        for (u32 e = rank; e < count * 8; e += size)
        {
            const u32 i = e >> 3, d = e & 7;
            if (d == 7) continue;
            u32 *row = a.rows + size_t(start + i) * kRow;
            row[3 + d] = boundaryIn(idx, row[2], row[10], rowKey(row) + u64(d + 1) * cr);
        }
        return;
    }
    for (u32 i = rank; i < count; i += size)
    {
        u32 *row = a.rows + size_t(start + i) * kRow;
        u32 b[7];
        innerBegins(idx, row[2], row[10], rowKey(row), cr, b);
#pragma unroll
        for (int d = 0; d < 7; ++d) row[3 + d] = b[d];
    }
}

static __global__ void __launch_bounds__(kThreads) expandKernel(Arena a, KeyIndex idx, int l)
{
    const Control &c = *a.ctl;
    if (c.overflow | c.late | c.error) return;
    expandUnits(a, idx, l, c.levelStart[l], c.levelCount[l], blockIdx.x * blockDim.x + threadIdx.x,
                gridDim.x * blockDim.x);
}

// The 27 cells around every unit of level l >= 1, from those around its
// parent U: the cell at offset (dx, dy, dz) of the unit (octant o in U) is
// child o' of the cell at offset floor((o + d) / 2) around U, o' =
// (o + d) mod 2 per axis.  That cell is a unit (the child of a unit around
// U, if internal) or lies in a leaf: a leaf child of a unit around U, or the
// leaf that already holds U's cell.
template <bool Hilbert>
static __global__ void __launch_bounds__(kThreads) nbrKernel(Arena a, int l, HilbertTables h)
{
    __shared__ unsigned char sEnc[48 * 8], sDec[48 * 8];
    const Control &c = *a.ctl;
    if (c.overflow | c.late | c.error) return;
    const u32 start = c.levelStart[l], count = c.levelCount[l];
    const size_t total = size_t(count) * 27;
    if (total <= size_t(blockIdx.x) * blockDim.x) return;
    if constexpr (Hilbert)
    {
        for (int k = threadIdx.x; k < 48 * 8; k += blockDim.x)
        {
            sEnc[k] = h.enc[k];
            sDec[k] = h.decOct[k];
        }
        __syncthreads();
    }
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x)
    {
        const u32 g = start + u32(e / 27);
        const int q = int(e - size_t(e / 27) * 27);
        const u32 pr = a.parent[g];
        const u32 U = pr >> 3, d = pr & 7u;
        const u32 stU = unitStateOf(a.rows[size_t(U) * kRow + 11]);
        const int o = Hilbert ? int(sDec[stU * 8 + d]) : int(d);
        const int tx = (o >> 2) + q % 3 - 1, ty = ((o >> 1) & 1) + (q / 3) % 3 - 1, tz = (o & 1) + q / 9 - 1;
        const int qp = ((tx + 2) / 2) + 3 * ((ty + 2) / 2) + 9 * ((tz + 2) / 2);  // offset around U
        const u32 r = a.nbr[size_t(U) * 27 + qp];
        u32 ref = r;
        if (!(r & kLeafRef))
        {
            const int oc = ((tx & 1) << 2) | ((ty & 1) << 1) | (tz & 1);
            const u32 stV = unitStateOf(a.rows[size_t(r) * kRow + 11]);
            const u32 dv = Hilbert ? u32(sEnc[stV * 8 + oc]) : u32(oc);
            const u32 ch = a.child[size_t(r) * 8 + dv];
            ref = ch != kLeaf ? ch : (kLeafRef | (r * 8 + dv));
        }
        a.nbr[size_t(g) * 27 + q] = ref;
    }
}

// Near-field counts of the children of the level-l units: per unit, the 27
// parent-level cells Q around it (nbrKernel) give the 4 x 4 x 4 block of
// child counts -- from the 9 child begins of Q when Q is a unit, counted
// within the keys of the leaf that holds Q otherwise -- and each child sums
// its 3 x 3 x 3 sub-block (octNearFieldKernel's unit, with the cells around
// it known instead of looked up).
// Per-warp scratch of the units in flight (the refresh's scratch without the
// group-flag populations, which leaves more of the SM's shared storage to L1).
struct UnitScratch
{
    u64 pStart[rb::kUnitBatch];
    int childState[rb::kUnitBatch];
    rb::UnitBlocks block;
    u32 slowRef[rb::kUnitBatch * 27];
    unsigned short slowItem[rb::kUnitBatch * 27];
    int nSlow;
};

// 5 CTAs per SM (48 registers, 29.6 KB of scratch each): 0.7 % faster builds
// at 16 Mi than 4.
template <bool Hilbert>
static __global__ void __launch_bounds__(kThreads, 5)
    nearFieldKernel(Arena a, KeyIndex idx, int l, HilbertTables h)
{
    using rb::kUnitBatch;
    __shared__ unsigned char sEnc[48 * 8], sNext[48 * 8], sDec[48 * 8];
    __shared__ UnitScratch sWarp[kThreads / 32];
    const Control &c = *a.ctl;
    if (c.overflow | c.late | c.error) return;
    const u32 start = c.levelStart[l], count = c.levelCount[l];
    if (count <= blockIdx.x * u32(kThreads / 32) * u32(rb::kUnitBatch)) return;  // no units for this CTA
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
    const unsigned m = unsigned(l) + 1;
    UnitScratch &w = sWarp[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned ltMask = (1u << lane) - 1u;
    const u32 warpsTotal = gridDim.x * (blockDim.x / 32);
    const u32 w0 = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    for (u32 base = w0 * kUnitBatch; base < count; base += warpsTotal * kUnitBatch)
    {
        const int nb = int(min(u32(kUnitBatch), count - base));
        if (lane < nb)
        {
            // the cell's path is decoded only where a neighbour lies inside a
            // coarser leaf (phase B); the children's curve state is in the row
            const u32 *row = a.rows + size_t(start + base + u32(lane)) * kRow;
            w.pStart[lane] = rowKey(row);
            w.childState[lane] = int(unitStateOf(row[11]));
        }
        if (lane == 0) w.nSlow = 0;
        __syncwarp();
        // phase A: (unit, Q) pairs over the lanes; a Q that is a unit gives
        // its children's counts from its row
        const int items = nb * 27;
        for (int ib = 0; ib < items; ib += 32)
        {
            const int it = ib + lane;
            const int u = it / 27, q = it - (it / 27) * 27;
            u32 ref = 0;
            bool slow = false;
            if (it < items)
            {
                ref = a.nbr[size_t(start + base + u32(u)) * 27 + q];
                if (ref & kLeafRef)
                {
                    slow = true;
                }
                else
                {
                    const uint4 *vr = reinterpret_cast<const uint4 *>(a.rows + size_t(ref) * kRow);
                    const uint4 r0 = vr[0], r1 = vr[1], r2 = vr[2];
                    const u32 gb[rb::kGroupBegins] = {r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z};
                    rb::childrenFromPacked<Hilbert>(gb, q, int(unitStateOf(r2.w)), w.block[u]);
                }
            }
            const unsigned slowMask = __ballot_sync(0xffffffffu, slow);
            if (slow)
            {
                const int k = w.nSlow + __popc(slowMask & ltMask);
                w.slowRef[k] = ref;
                w.slowItem[k] = (unsigned short)it;
            }
            __syncwarp();
            if (lane == 0) w.nSlow += __popc(slowMask);
            __syncwarp();
        }
        // phase B: Q in a leaf: its children counted among the leaf's keys
        const int nSlow = w.nSlow;
        for (int k = lane; k < nSlow; k += 32)
        {
            const int it = w.slowItem[k];
            const int u = it / 27, q = it - u * 27;
            const u32 lr = w.slowRef[k] & ~kLeafRef;
            const u32 P = lr >> 3, d = lr & 7u;
            const u32 *prow = a.rows + size_t(P) * kRow;
            const u32 preg = prow[11];
            u64 qKey;
            int qState;
            if (unitLevelOf(preg) + 1 == unsigned(l))
            {
                // the leaf is Q itself: child d of its parent unit
                qKey = rowKey(prow) + u64(d) * octRange(unsigned(l));
                const u32 stP = unitStateOf(preg);
                qState = Hilbert ? int(sNext[stP * 8 + sDec[stP * 8 + d]]) : kHilbertStart;
            }
            else
            {
                const rb::CellPath path = rb::decodeCell<Hilbert>(w.pStart[u], unsigned(l), sNext, sDec);
                qKey = rb::neighbourCellOf<Hilbert>(path, w.pStart[u], unsigned(l), q, qState, sEnc, sNext);
            }
            u32 begins[rb::kGroupBegins];
            rb::childBeginsWithin(idx.keys, prow[2 + d], prow[3 + d], qKey, m, begins);
            rb::childrenFromPacked<Hilbert>(begins, q, qState, w.block[u]);
        }
        __syncwarp();
        // phase C: the 8 children of each unit, two per lane
        for (int e = lane; e < nb * 8; e += 32)
        {
            const int u = e >> 3, d = e & 7;
            const u32 g = start + base + u32(u);
            const u32 *row = a.rows + size_t(g) * kRow;
            const u32 cnt = row[2 + d + 1] - row[2 + d];
            u32 out = 0;
            if (cnt)
            {
                const unsigned o = Hilbert ? unsigned(sDec[w.childState[u] * 8 + d]) : unsigned(d);
                const u32 *sub = w.block[u] + (o >> 2) * 16 + ((o >> 1) & 1u) * 4 + (o & 1u);
                u64 pop = 0;
                if (m > 1)
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
                const u64 v = u64(cnt) * pop;
                out = v > 0xffffffffull ? 0xffffffffu : u32(v);
            }
            a.val[size_t(g) * 8 + d] = out;
        }
        __syncwarp();
    }
}

// Children of the level-l units: those whose value exceeds the bucket (below
// level 21) become the units of level l + 1, the others are leaves, counted
// into the round history by (arrival, depth, relative level).  A warp takes
// the slots of its new units with one atomic add; the order of the units in
// a level is free (every later step finds them through the child and parent
// links, and the placement follows the digits).
// Forest: the history counts go to the unit's system's bins in global memory
// (sContrib / sLanded unused); otherwise to the CTA's shared bins.
template <bool NF, bool Hilbert, bool Forest>
__device__ __forceinline__ void classifyUnits(const Arena &a, int l, unsigned bucket, u32 start, u32 count,
                                              const unsigned char *sNext, const unsigned char *sDec, u32 *sContrib,
                                              u32 *sLanded, u32 rank, u32 size)
{
    Control &c = *a.ctl;
    const u32 next = start + count;
    if (rank == 0) c.levelStart[l + 1] = next;
    const unsigned m = unsigned(l) + 1;
    const u64 cr = octRange(m);
    const int lane = threadIdx.x & 31;
    for (u32 i0 = rank & ~31u; i0 < count; i0 += size)
    {
        const u32 i = i0 + u32(lane);
        const bool valid = i < count;
        const u32 g = start + (valid ? i : 0);
        const uint4 *row4 = reinterpret_cast<const uint4 *>(a.rows + size_t(g) * kRow);
        u32 b[rb::kGroupBegins], x[8];
        u32 reg = 0;
        u64 key = 0;
        unsigned highMask = 0;
        if (valid)
        {
            const uint4 r0 = row4[0], r1 = row4[1], r2 = row4[2];
            key = (u64(r0.y) << 32) | r0.x;
            b[0] = r0.z; b[1] = r0.w;
            b[2] = r1.x; b[3] = r1.y; b[4] = r1.z; b[5] = r1.w;
            b[6] = r2.x; b[7] = r2.y; b[8] = r2.z;
            reg = r2.w;
            if constexpr (NF)
            {
                const uint4 *v4 = reinterpret_cast<const uint4 *>(a.val + size_t(g) * 8);
                const uint4 v0 = v4[0], v1 = v4[1];
                x[0] = v0.x; x[1] = v0.y; x[2] = v0.z; x[3] = v0.w;
                x[4] = v1.x; x[5] = v1.y; x[6] = v1.z; x[7] = v1.w;
            }
#pragma unroll
            for (int d = 0; d < 8; ++d)
            {
                if constexpr (!NF) x[d] = b[d + 1] - b[d];
                if (x[d] > bucket && m < kOctLevels) highMask |= 1u << d;
            }
        }
        // slots of the warp's new units: one atomic add per warp
        const u32 nHigh = u32(__popc(highMask));
        u32 incl = nHigh;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const u32 t = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += t;
        }
        u32 base = 0;
        if (lane == 31 && incl) base = atomicAdd(&c.levelCount[l + 1], incl);
        base = __shfl_sync(0xffffffffu, base, 31);
        if (!valid) continue;
        const u32 aR = regionArrival(reg), lR = regionLevel(reg), kR = regionDepth(reg);
        const u32 j = m - lR;  // 1 <= j <= kR
        const u32 sys = Forest ? a.usys[g] : 0u;
        u32 rank = base + incl - nHigh;
        u32 slots[8];
#pragma unroll
        for (int d = 0; d < 8; ++d)
        {
            u32 slot = kLeaf;
            if (highMask & (1u << d))
            {
                const u32 gc = next + rank++;
                if (gc < a.cap)
                {
                    u32 creg = reg;
                    if (j == kR)
                    {
                        // a landed internal node: a leaf in round aR + 1, splitting at once
                        creg = regionWord(aR + 1, m, splitDepth(NF, x[d], bucket, m));
                        if (aR + 2 >= u32(kArrivals)) c.late = 1;
                        else if (Forest) atomicAdd(a.landed + size_t(sys) * kArrivals + aR + 1, 1ull);
                        else atomicAdd(&sLanded[aR + 1], 1u);
                    }
                    if constexpr (Forest) a.usys[gc] = sys;
                    // the child's own level and the curve state ordering its children
                    u32 cst = kHilbertStart;
                    if constexpr (Hilbert)
                    {
                        const u32 st = unitStateOf(reg);
                        cst = sNext[st * 8 + sDec[st * 8 + d]];
                    }
                    if constexpr (NF) a.parent[gc] = g * 8 + u32(d);
                    const u64 ck = key + u64(d) * cr;
                    uint4 *crow = reinterpret_cast<uint4 *>(a.rows + size_t(gc) * kRow);
                    crow[0] = make_uint4(u32(ck), u32(ck >> 32), b[d], 0u);
                    crow[2] = make_uint4(0u, 0u, b[d + 1], withUnit(creg, m, cst));
                    slot = gc;
                }
                else
                {
                    c.overflow = 1;
                }
            }
            else if constexpr (Forest)
            {
                atomicAdd(a.contrib + size_t(sys) * kContribBins + (aR * kJumps + kR) * kJumps + j, 1ull);
            }
            else
            {
                atomicAdd(&sContrib[(aR * kJumps + kR) * kJumps + j], 1u);
            }
            slots[d] = slot;
        }
        uint4 *ch4 = reinterpret_cast<uint4 *>(a.child + size_t(g) * 8);
        ch4[0] = make_uint4(slots[0], slots[1], slots[2], slots[3]);
        ch4[1] = make_uint4(slots[4], slots[5], slots[6], slots[7]);
    }
}

template <bool NF, bool Hilbert>
static __global__ void __launch_bounds__(kThreads) classifyKernel(Arena a, int l, unsigned bucket, HilbertTables h)
{
    __shared__ u32 sContrib[kContribBins];
    __shared__ u32 sLanded[kArrivals];
    __shared__ unsigned char sNext[48 * 8], sDec[48 * 8];
    Control &c = *a.ctl;
    if (c.overflow | c.late | c.error) return;
    const u32 start = c.levelStart[l], count = c.levelCount[l];
    if (blockIdx.x == 0 && threadIdx.x == 0) c.levelStart[l + 1] = start + count;
    if (count <= blockIdx.x * blockDim.x) return;
    if constexpr (Hilbert)
    {
        for (int k = threadIdx.x; k < 48 * 8; k += blockDim.x)
        {
            sNext[k] = h.encNext[k];
            sDec[k] = h.decOct[k];
        }
    }
    for (int k = threadIdx.x; k < kContribBins; k += kThreads) sContrib[k] = 0;
    if (threadIdx.x < kArrivals) sLanded[threadIdx.x] = 0;
    __syncthreads();
    classifyUnits<NF, Hilbert, false>(a, l, bucket, start, count, sNext, sDec, sContrib, sLanded,
                                      blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
    __syncthreads();
    for (int k = threadIdx.x; k < kContribBins; k += kThreads)
        if (sContrib[k]) atomicAdd(a.contrib + k, (unsigned long long)sContrib[k]);
    if (threadIdx.x < kArrivals && sLanded[threadIdx.x])
        atomicAdd(a.landed + threadIdx.x, (unsigned long long)sLanded[threadIdx.x]);
}

// Leaves below each unit of level l (the units of level l + 1 are done).
// `levels` is the number of levels the build expanded: units below them mean
// the build is incomplete, and nothing is counted.
__device__ __forceinline__ void leafCountUnits(const Arena &a, u32 start, u32 count, u32 rank, u32 size)
{
    for (u32 i = rank; i < count; i += size)
    {
        const u32 g = start + i;
        u32 s = 0;
#pragma unroll
        for (int d = 0; d < 8; ++d)
        {
            const u32 ch = a.child[size_t(g) * 8 + d];
            s += ch == kLeaf ? 1u : a.leaves[ch];
        }
        a.leaves[g] = s;
    }
}

static __global__ void leafCountKernel(Arena a, int l, int levels)
{
    const Control &c = *a.ctl;
    if (c.levelCount[levels] | c.overflow | c.late | c.error) return;
    leafCountUnits(a, c.levelStart[l], c.levelCount[l], blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// Cornerstone entries of the leaf children of the level-l units, and the
// first leaf index of their internal children.  Eight lanes per unit, one per
// child: a segmented scan of the children's leaf counts gives each child's
// position, so a warp writes the entries of four units at once.
// K, B (and NF, N, SEG where given) are the cornerstone arrays written: N the
// leaf counts, SEG each leaf's tree (system) in a batch of trees.
template <bool NF>
__device__ __forceinline__ void placeUnits(const Arena &a, u64 *K, u32 *B, u32 *NFo, u32 *N, int *SEG, int l,
                                           u32 start, u32 count, u32 capacity, u32 rank, u32 size)
{
    Control &c = *a.ctl;
    const u64 cr = octRange(unsigned(l) + 1);
    const int lane = threadIdx.x & 31, d = lane & 7;
    const size_t total = size_t(count) * 8;
    for (size_t e0 = rank & ~31u; e0 < total; e0 += size)
    {
        const size_t e = e0 + size_t(lane);
        const bool valid = e < total;
        const u32 g = start + u32(valid ? e >> 3 : 0);
        const u32 ch = valid ? a.child[size_t(g) * 8 + d] : kLeaf;
        const u32 mine = ch == kLeaf ? 1u : a.leaves[ch];
        // exclusive prefix of the leaf counts within the unit's 8 lanes
        u32 inc = mine;
#pragma unroll
        for (int off = 1; off < 8; off <<= 1)
        {
            const u32 t = __shfl_up_sync(0xffffffffu, inc, off);
            if (d >= off) inc += t;
        }
        if (!valid) continue;
        const u32 o = a.offset[g] + inc - mine;
        if (ch == kLeaf && o >= capacity)
        {
            c.placeOverflow = 1;  // the host grows the buffers and places again
        }
        else if (ch == kLeaf)
        {
            const u32 *row = a.rows + size_t(g) * kRow;
            K[o] = rowKey(row) + u64(d) * cr;
            B[o] = row[2 + d];
            if constexpr (NF) NFo[o] = a.val[size_t(g) * 8 + d];
            if (N) N[o] = row[3 + d] - row[2 + d];
            if (SEG) SEG[o] = int(a.usys[g]);
        }
        else
        {
            a.offset[ch] = o;
        }
    }
}

template <bool NF>
static __global__ void placeKernel(Arena a, u64 *K, u32 *B, u32 *NFo, u32 *N, int l, int levels, u32 capacity)
{
    const Control &c = *a.ctl;
    if (c.levelCount[levels] | c.overflow | c.late | c.error) return;
    placeUnits<NF>(a, K, B, NFo, N, nullptr, l, c.levelStart[l], c.levelCount[l], capacity,
                   blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// The finished tree: sentinel boundary and the state of a converged build
// (finishBuildStateKernel, octree.cu:40-47, after `rounds` changing rounds).
static __global__ void finishKernel(Arena a, rb::TreeBufs tb, int rounds, int levels, u32 capacity)
{
    DeviceState *st = tb.st;
    const Control &c = *a.ctl;
    if (c.levelCount[levels] | c.overflow | c.late | c.error | c.placeOverflow) return;
    const int leaves = c.levelCount[0] ? int(a.leaves[0]) : 1;
    if (u32(leaves) > capacity) return;
    tb.K[0][leaves] = kMaxKey;
    tb.B[0][leaves] = st->numActiveParticles;
    st->numLeaves = leaves;
    st->newNumLeaves = leaves;
    st->proposal = leaves;
    st->iteration = rounds;
    st->rounds = rounds + 1;
    st->changed = st->converged = st->needsResize = 0;
    st->numNodes = 0;
    st->activeBuffer = 0;
    st->overflow = 0;
    st->dirtyCount = 0;
}
}  // namespace lb
}  // namespace aot
