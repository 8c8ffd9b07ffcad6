// binlevel.cuh -- the converged binary (k-d) tree build, level by level.
//
// The reference builds a binary tree from the root by passes until a pass
// changes nothing (the build loop of kdtree3d.cu:239-249 over
// binaryDecisionKernel, kdtree3d_rebalance.cuh:28-60): a leaf splits in two
// when it holds more than `bucket` particles and its depth is below
// maxDepth, and two sibling leaves merge when together they hold at most
// `bucket`.  A leaf's count never grows from a node to its children, so no
// pair made by a split can merge afterwards, and the tree the passes end with
// is unique: a node is internal exactly when it holds more than `bucket`
// particles below maxDepth.  One level of internal nodes ("units") at a time:
//   level     per unit the lower bound of its midpoint key among its keys
//             (a warp per unit on levels of few units), then its two
//             children: those above the bucket become units of the next
//             level (warp-aggregated slots), the others are leaves;
//   leafCount subtree leaf counts, deepest level first;
//   place     every leaf's K, B and count, shallowest level first.
// Each pass of the reference splits one level, so the passes that change the
// tree number the deepest unit's level + 1, and its leaf capacity, grown by
// 25 % steps to the leaf count of every pass (commitIfLast, rebalance.cuh),
// ends at the first step of that chain at or above the final leaf count:
// the counts only grow during a build.
#pragma once

#include "levelbuild.cuh"

namespace aot
{
namespace bl
{
constexpr int kThreads = 256;
constexpr u32 kLeaf = 0xffffffffu;
constexpr int kLevels = 64;          // depths 0..63
constexpr u32 kWideUnits = 2048;     // levels of at most this many units search by warps

struct Control
{
    u32 levelStart[kLevels + 2];
    u32 levelCount[kLevels + 2];
    int overflow;       // the unit arena is too small
    int placeOverflow;  // more leaves than the leaf arrays hold
};

struct Arena
{
    uint4 *rows;    // [cap] key lo, key hi, begin, end
    u32 *mid;       // [cap] first key of the upper child
    u32 *child;     // [cap][2] unit index of an internal child, or kLeaf
    u32 *leaves;    // [cap] leaves in the unit's subtree
    u32 *offset;    // [cap] leaf index of the unit's first leaf
    Control *ctl;
    u32 cap;
};

// Key range of a node at depth d: 2^(63 - d).
__device__ __forceinline__ u64 depthRange(int d) { return u64(1) << (63 - d); }

// The root: a unit when it holds more than `bucket` particles (and may
// split), else the single root leaf, written straight to the leaf arrays.
static __global__ void rootKernel(Arena a, rb::TreeBufs tb, const u64 *P, size_t n, unsigned bucket,
                                  unsigned maxDepth)
{
    const unsigned active = n ? warpLowerBound(P, 0, u32(n), kMaxKey, int(threadIdx.x & 31)) : 0u;
    if (threadIdx.x != 0) return;
    DeviceState *st = tb.st;
    const int err = st->error;
    *st = DeviceState{};
    st->error = err;
    st->numActiveParticles = active;
    Control &c = *a.ctl;
    c.levelStart[0] = 0;
    if (active > bucket && maxDepth > 0)
    {
        a.rows[0] = make_uint4(0u, 0u, 0u, active);
        a.offset[0] = 0;
        c.levelCount[0] = 1;
    }
    else
    {
        c.levelCount[0] = 0;
        tb.K[0][0] = 0;
        tb.K[0][1] = kMaxKey;
        tb.B[0][0] = 0;
        tb.B[0][1] = active;
        tb.N[0][0] = active;
    }
}

// The units of depth l: their midpoints, then their children.
static __global__ void __launch_bounds__(kThreads) levelKernel(Arena a, KeyIndex idx, int l, unsigned bucket,
                                                               unsigned maxDepth)
{
    Control &c = *a.ctl;
    if (c.overflow) return;
    const u32 start = c.levelStart[l], count = c.levelCount[l];
    const u32 next = start + count;
    if (blockIdx.x == 0 && threadIdx.x == 0) c.levelStart[l + 1] = next;
    const u64 half = depthRange(l + 1);
    const bool deeper = unsigned(l + 1) < maxDepth;  // children at depth l + 1 may split
    const int lane = threadIdx.x & 31;
    if (count <= kWideUnits)
    {
        // a warp per unit: 33-way searches over the unit's keys
        const u32 warps = gridDim.x * (blockDim.x >> 5);
        for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += warps)
        {
            const u32 g = start + i;
            const uint4 r = a.rows[g];
            const u64 key = (u64(r.y) << 32) | r.x;
            const u32 m = warpLowerBound(idx.keys, r.z, r.w, key + half, lane);
            if (lane != 0) continue;
            a.mid[g] = m;
            const u32 cnt[2] = {m - r.z, r.w - m};
            for (int s = 0; s < 2; ++s)
            {
                u32 slot = kLeaf;
                if (cnt[s] > bucket && deeper)
                {
                    const u32 gc = next + atomicAdd(&c.levelCount[l + 1], 1u);
                    if (gc < a.cap)
                    {
                        const u64 ck = key + u64(s) * half;
                        a.rows[gc] = make_uint4(u32(ck), u32(ck >> 32), s ? m : r.z, s ? r.w : m);
                        slot = gc;
                    }
                    else
                    {
                        c.overflow = 1;
                    }
                }
                a.child[size_t(g) * 2 + s] = slot;
            }
        }
        return;
    }
    const u32 stride = gridDim.x * blockDim.x;
    for (u32 i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); i0 < count; i0 += stride)
    {
        const u32 i = i0 + u32(lane);
        const bool valid = i < count;
        const u32 g = start + (valid ? i : 0);
        uint4 r = make_uint4(0u, 0u, 0u, 0u);
        u64 key = 0;
        u32 m = 0;
        unsigned high = 0;
        if (valid)
        {
            r = a.rows[g];
            key = (u64(r.y) << 32) | r.x;
            m = lb::boundaryIn(idx, r.z, r.w, key + half);
            a.mid[g] = m;
            if (m - r.z > bucket && deeper) high |= 1u;
            if (r.w - m > bucket && deeper) high |= 2u;
        }
        // slots of the warp's new units: one atomic add per warp
        const u32 nHigh = u32(__popc(high));
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
        u32 rank = base + incl - nHigh;
        for (int s = 0; s < 2; ++s)
        {
            u32 slot = kLeaf;
            if (high & (1u << s))
            {
                const u32 gc = next + rank++;
                if (gc < a.cap)
                {
                    const u64 ck = key + u64(s) * half;
                    a.rows[gc] = make_uint4(u32(ck), u32(ck >> 32), s ? m : r.z, s ? r.w : m);
                    slot = gc;
                }
                else
                {
                    c.overflow = 1;
                }
            }
            a.child[size_t(g) * 2 + s] = slot;
        }
    }
}

// Leaves below each unit of depth l (the units of depth l + 1 are counted).
// `levels`: the depths the build expanded; units below them mean the build is
// incomplete, and nothing is counted or placed.
static __global__ void leafCountKernel(Arena a, int l, int levels)
{
    const Control &c = *a.ctl;
    if (c.levelCount[levels] | c.overflow) return;
    const u32 start = c.levelStart[l], count = c.levelCount[l];
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    {
        const u32 g = start + i;
        const u32 c0 = a.child[size_t(g) * 2], c1 = a.child[size_t(g) * 2 + 1];
        a.leaves[g] = (c0 == kLeaf ? 1u : a.leaves[c0]) + (c1 == kLeaf ? 1u : a.leaves[c1]);
    }
}

// K, B and the count of the leaf children of the depth-l units, and the
// first leaf index of their internal children.
static __global__ void placeKernel(Arena a, u64 *K, u32 *B, u32 *N, int l, int levels, u32 capacity)
{
    Control &c = *a.ctl;
    if (c.levelCount[levels] | c.overflow) return;
    const u32 start = c.levelStart[l], count = c.levelCount[l];
    const u64 half = depthRange(l + 1);
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    {
        const u32 g = start + i;
        const uint4 r = a.rows[g];
        const u64 key = (u64(r.y) << 32) | r.x;
        const u32 m = a.mid[g];
        const u32 lo[2] = {r.z, m}, hi[2] = {m, r.w};
        u32 o = a.offset[g];
        for (int s = 0; s < 2; ++s)
        {
            const u32 ch = a.child[size_t(g) * 2 + s];
            if (ch != kLeaf)
            {
                a.offset[ch] = o;
                o += a.leaves[ch];
            }
            else if (o >= capacity)
            {
                c.placeOverflow = 1;  // the host grows the leaf arrays and places again
                ++o;
            }
            else
            {
                K[o] = key + u64(s) * half;
                B[o] = lo[s];
                N[o] = hi[s] - lo[s];
                ++o;
            }
        }
    }
}

// The finished tree: its sentinel and the state the reference's passes end
// with (the last pass changes nothing: converged, one more pass counted).
static __global__ void finishKernel(Arena a, rb::TreeBufs tb, int leaves, int passes, long long logicalCap)
{
    DeviceState *st = tb.st;
    tb.K[0][leaves] = kMaxKey;
    tb.B[0][leaves] = st->numActiveParticles;
    st->numLeaves = st->newNumLeaves = leaves;
    st->numNodes = (leaves - 1) * 2 + 1;
    st->proposal = leaves;
    st->iteration = passes;
    st->rounds = passes + 1;
    st->converged = 1;
    st->changed = st->needsResize = 0;
    st->activeBuffer = 0;
    st->overflow = 0;
    st->dirtyCount = 0;
    st->logicalCap = logicalCap;
}
}  // namespace bl
}  // namespace aot
