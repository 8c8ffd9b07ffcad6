// tree_view.cuh -- traversal-free FMM view of a cornerstone tree.
//
// Produces the arrays of TreeView<LevelBits> (tree_view.cu:151-562): box SFC
// index with placeholder bit, split flag, depth, parent and first-child
// indices, per-level offsets, per-box particle ranges and the particle ->
// leaf-node map.  Nodes are numbered breadth first; inside a level all
// child-0 nodes come first (in the order of their parents), then all child-1
// nodes, and so on -- the reference's child-centric layout.
//
// Pipeline (every size read from DeviceState, grids sized by capacity, so the
// view can be captured inside the update graph):
//   classify     leaf levels + per-level leaf histogram; each boundary between
//                neighbouring leaves whose right side starts child 1 of their
//                lowest common ancestor marks exactly one internal node
//   metadata     per-level node counts and offsets by the backward recurrence
//                nodes[l] = leaves[l] + nodes[l+1] / 2^b
//   level order  one stable onesweep pass keyed by level (non-internal
//                boundaries get key 255 and sort last)
//   layout order stable onesweep sort of (1 << b*level) | reversed child path
//   nodes        internal and leaf nodes written at their final indices
//   mapping      particle -> leaf node by an upper bound over leaf begin indices
#pragma once

#include "common.cuh"

namespace aot
{
namespace tv
{
constexpr int kThreads = 256;
constexpr int kMaxLevelsOct = 21, kMaxLevelsBin = 63;

struct ViewBufs
{
    // outputs
    u64 *box;
    u8 *split, *depth;
    int *parent, *child, *levelOffset;
    u32 *pbegin, *pcount;
    u64 *pmap;
    u8 *maxDepth;
    // scratch
    u8 *leafLevel;
    int *leafToNode;
    int *leavesPerLevel, *internalPerLevel, *nodesPerLevel, *levelOffsetInternal;
    u64 *candStart;    // per boundary
    u8 *candLevel;     // per boundary
    u64 *lvKeys, *lvKeysAlt;   // level-sort keys (per boundary)
    u32 *lvVals, *lvValsAlt;   // boundary indices
    u64 *layKeys, *layKeysAlt; // layout keys (per internal)
    u32 *layVals, *layValsAlt; // level-order positions
    u64 *intStartSfc;  // internal starts in (level, SFC) order
    u8 *intLevelSfc;
    int *intMBySfc;    // layout rank inside the level, by SFC position
    u64 *intStartLay;  // internal starts in layout order
    u8 *intLevelLay;
};

template <int b>
__device__ __forceinline__ unsigned viewLevel(u64 range) { return unsigned(clz64(range)) / b; }
template <int b>
__device__ __forceinline__ u64 viewRange(unsigned level) { return kMaxKey >> (b * level); }
template <int b>
__device__ __forceinline__ int viewMaxLevel() { return b == 3 ? kMaxLevelsOct : kMaxLevelsBin; }

// Lowest common ancestor level of two distinct keys below 2^63
// (lcaLevel, tree_view.cu:94-108): levels whose node prefixes agree.
template <int b>
__device__ __forceinline__ unsigned lcaLevel(u64 x, u64 y)
{
    const unsigned common = unsigned(clz64(x ^ y));
    unsigned l = (common - 1) / b;
    const unsigned m = unsigned(viewMaxLevel<b>());
    return l < m ? l : m;
}

// Stage 1 (classifyLeavesAndInternalsKernel, tree_view.cu:151-203).
template <int b>
static __global__ void classifyKernel(const u64 *Kact0, const u64 *Kact1, DeviceState *st, int leafCap, ViewBufs v)
{
    __shared__ int sHist[64];
    if (threadIdx.x < 64) sHist[threadIdx.x] = 0;
    __syncthreads();
    const u64 *K = st->activeBuffer ? Kact1 : Kact0;
    const int L = st->numLeaves <= leafCap ? st->numLeaves : 0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0)
    {
        if (st->numLeaves > leafCap) st->needsResize = 1;
        else st->numNodes = L + (L - 1) / ((1 << b) - 1);
    }
    if (i < L)
    {
        const unsigned lev = viewLevel<b>(K[i + 1] - K[i]);
        v.leafLevel[i] = u8(lev);
        atomicAdd(&sHist[lev], 1);
    }
    if (i < leafCap - 1)
    {
        u64 key = 255;
        if (i < L - 1)
        {
            const u64 left = K[i], right = K[i + 1];
            const unsigned lca = lcaLevel<b>(left, right);
            const u64 pr = viewRange<b>(lca);
            const u64 parentStart = right & ~(pr - 1);
            const unsigned slot = unsigned((right - parentStart) / viewRange<b>(lca + 1));
            v.candStart[i] = parentStart;
            v.candLevel[i] = u8(lca);
            if (slot == 1) key = lca;
        }
        v.lvKeys[i] = key;
        v.lvVals[i] = u32(i);
    }
    __syncthreads();
    if (threadIdx.x < 64 && sHist[threadIdx.x]) atomicAdd(&v.leavesPerLevel[threadIdx.x], sHist[threadIdx.x]);
}

// Stage 2 (buildLevelMetadataKernel, tree_view.cu:211-275), one thread.
template <int b>
static __global__ void metadataKernel(DeviceState *st, int leafCap, ViewBufs v)
{
    const int L = st->numLeaves <= leafCap ? st->numLeaves : 0;
    if (L == 0) return;
    const int maxL = viewMaxLevel<b>();
    int maxLevel = 0;
    for (int l = 0; l <= maxL; ++l)
    {
        if (v.leavesPerLevel[l]) maxLevel = l;
        v.internalPerLevel[l] = 0;
        v.nodesPerLevel[l] = 0;
    }
    *v.maxDepth = u8(maxLevel);
    v.nodesPerLevel[maxLevel] = v.leavesPerLevel[maxLevel];
    for (int l = maxLevel - 1; l >= 0; --l)
    {
        v.internalPerLevel[l] = v.nodesPerLevel[l + 1] >> b;
        v.nodesPerLevel[l] = v.leavesPerLevel[l] + v.internalPerLevel[l];
    }
    v.levelOffset[0] = 0;
    for (int l = 0; l <= maxLevel; ++l) v.levelOffset[l + 1] = v.levelOffset[l] + v.nodesPerLevel[l];
    const int numNodes = v.levelOffset[maxLevel + 1];
    for (int l = maxLevel + 1; l <= maxL; ++l) v.levelOffset[l + 1] = numNodes;
    v.levelOffsetInternal[0] = 0;
    for (int l = 0; l <= maxLevel; ++l)
        v.levelOffsetInternal[l + 1] = v.levelOffsetInternal[l] + v.internalPerLevel[l];
    const int numInternal = v.levelOffsetInternal[maxLevel + 1];
    for (int l = maxLevel + 1; l <= maxL; ++l) v.levelOffsetInternal[l + 1] = numInternal;
}

// Stages 3-5: internal starts/levels in (level, SFC) order and layout keys
// (makeInternalLayoutKeysKernel, tree_view.cu:301-339).
template <int b>
static __global__ void layoutKeysKernel(const u64 *lvSortedKeys, const u32 *lvSortedVals, int intCap, ViewBufs v)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= intCap) return;
    const u64 lk = lvSortedKeys[j];
    u64 key = ~u64(0);
    if (lk != 255)
    {
        const u32 bi = lvSortedVals[j];
        const u64 start = v.candStart[bi];
        const unsigned level = v.candLevel[bi];
        v.intStartSfc[j] = start;
        v.intLevelSfc[j] = u8(level);
        // reversed child path: digit at `level` most significant
        u64 path = 0;
        for (unsigned d = level; d > 0; --d)
        {
            const u64 digit = (start >> (63 - b * d)) & ((1u << b) - 1);
            path = (path << b) | digit;
        }
        key = (u64(1) << (b * level)) | path;
    }
    v.layKeys[j] = key;
    v.layVals[j] = u32(j);
}

// materializeInternalLayoutKernel (tree_view.cu:340-358)
static __global__ void materializeKernel(const u64 *laySortedKeys, const u32 *laySortedVals, int intCap, ViewBufs v)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= intCap || laySortedKeys[j] == ~u64(0)) return;
    const u32 pos = laySortedVals[j];
    const unsigned level = v.intLevelSfc[pos];
    v.intLevelLay[j] = u8(level);
    v.intStartLay[j] = v.intStartSfc[pos];
    v.intMBySfc[pos] = j - v.levelOffsetInternal[level];
}

// finalNodeIndex (tree_view.cu:383-401)
template <int b>
__device__ __forceinline__ int finalNodeIndex(unsigned level, u64 start, const ViewBufs &v)
{
    if (level == 0) return 0;
    const u64 pr = viewRange<b>(level - 1);
    const u64 parentStart = start & ~(pr - 1);
    const int lo = v.levelOffsetInternal[level - 1], hi = v.levelOffsetInternal[level];
    if (hi <= lo) return 0;  // no internal node at the parent level: not a valid tree
    int pos = lo + int(lowerBoundDev(v.intStartSfc + lo, size_t(hi - lo), parentStart));
    if (pos >= hi) pos = hi - 1;  // keep the lookup inside the level even for an invalid tree
    const int parentM = v.intMBySfc[pos];
    const unsigned slot = unsigned((start - parentStart) / viewRange<b>(level));
    return v.levelOffset[level] + int(slot) * v.internalPerLevel[level - 1] + parentM;
}

// Stage 6 (buildInternalNodesKernel, tree_view.cu:407-482)
template <int b>
static __global__ void internalNodesKernel(DeviceState *st, int leafCap, int intCap, KeyIndex idx, int counts, ViewBufs v)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int L = st->numLeaves <= leafCap ? st->numLeaves : 0;
    const int I = L > 0 ? (L - 1) / ((1 << b) - 1) : 0;
    if (j >= I || j >= intCap) return;
    const unsigned level = v.intLevelLay[j];
    const u64 start = v.intStartLay[j];
    const u64 end = start + viewRange<b>(level);
    const int node = finalNodeIndex<b>(level, start, v);
    v.box[node] = (u64(1) << (b * level)) | (start >> (63 - b * level));
    v.depth[node] = u8(level);
    v.split[node] = 1;
    if (level == 0) v.parent[node] = -1;
    const int m = j - v.levelOffsetInternal[level];
    const int M = v.internalPerLevel[level];
    const int firstChild = v.levelOffset[level + 1] + m;
    v.child[node] = firstChild;
    for (int s = 0; s < (1 << b); ++s) v.parent[firstChild + s * M] = node;
    if (counts)
    {
        const u32 bg = u32(idx.lower(start)), en = u32(idx.lower(end));
        v.pbegin[node] = bg;
        v.pcount[node] = en - bg;
        if (level == 0) v.pcount[st->numNodes] = en - bg;
    }
}

// Stage 7 (buildLeafNodesKernel, tree_view.cu:488-538)
template <int b>
static __global__ void leafNodesKernel(const u64 *K0, const u64 *K1, const u32 *B0, const u32 *B1, DeviceState *st,
                                int leafCap, int counts, ViewBufs v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int L = st->numLeaves <= leafCap ? st->numLeaves : 0;
    if (i >= L) return;
    const u64 *K = st->activeBuffer ? K1 : K0;
    const u32 *B = st->activeBuffer ? B1 : B0;
    const unsigned level = v.leafLevel[i];
    const u64 start = K[i];
    const int node = finalNodeIndex<b>(level, start, v);
    v.box[node] = (u64(1) << (b * level)) | (start >> (63 - b * level));
    v.depth[node] = u8(level);
    v.split[node] = 0;
    v.child[node] = -1;
    v.leafToNode[i] = node;
    if (level == 0) v.parent[node] = -1;
    if (counts)
    {
        v.pbegin[node] = B[i];
        v.pcount[node] = B[i + 1] - B[i];
        if (level == 0) v.pcount[st->numNodes] = B[i + 1] - B[i];
    }
}

// Particle mapping (fillSfcParticleIndexKernel, tree_view.cu:542-562): the leaf
// holding sorted particle p is the last leaf whose begin index is <= p.
static __global__ void mappingKernel(const u32 *B0, const u32 *B1, DeviceState *st, int leafCap, size_t n, ViewBufs v)
{
    const size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (p >= n) return;
    const int L = st->numLeaves <= leafCap ? st->numLeaves : 0;
    if (L == 0) return;
    if (p >= st->numActiveParticles)
    {
        v.pmap[p] = ~u64(0);
        return;
    }
    const u32 *B = st->activeBuffer ? B1 : B0;
    // upper bound of p over B[0..L)
    size_t lo = 0, len = size_t(L);
    while (len > 0)
    {
        const size_t half = len >> 1;
        const bool le = B[lo + half] <= u32(p);
        lo = le ? lo + half + 1 : lo;
        len = le ? len - half - 1 : half;
    }
    v.pmap[p] = u64((long long)v.leafToNode[lo - 1]);
}

static __global__ void flagResizeKernel(DeviceState *st) { st->needsResize = 1; }

}  // namespace tv
}  // namespace aot
