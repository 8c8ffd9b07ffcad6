// forest_levels.cuh -- the converged build of every system of a forest in one
// persistent (cooperative) launch.
//
// Each system is built as a single tree's converged build by levels
// (levelbuild.cuh): the tree the reference's rounds converge to (rebalanceBuild,
// octree.cu:159-180, LeafCount decisions of calculateNodeOp,
// octree_rebalance.cuh:174-249) is unique -- a cell is internal exactly when
// it holds more than `bucket` particles below level 21 -- so the internal
// cells of all systems are expanded level by level together, and each
// system's round history (the leaf counts its rounds would have had, which
// decide leafCapacity) is derived from its own cells.  One kernel runs every
// phase, separated by grid barriers:
//   roots      a level-0 unit for every system with more than `bucket` active
//              particles (the others are a single root leaf);
//   levels     expand (child begins), barrier, classify (new units, history
//              bins per system), barrier -- until a level has no units;
//   leafCount  subtree leaf counts, deepest level first;
//   layout     CTA 0: each system's first entry (an exclusive scan of
//              leaves + 1 over the systems), sentinels and root leaves, the
//              per-system and forest-wide state;
//   history    per system (one CTA each): leaves after every round;
//   place      every leaf's entry, shallowest level first;
//   counts     N = differences of B.
// A barrier waits a bounded number of polls; a CTA that gives up records it
// and every CTA returns at its next barrier.  The launch is cooperative, so
// all CTAs are resident and the waits end unless a CTA has failed.
#pragma once

#include "forest.cuh"
#include "grid_barrier.cuh"
#include "levelbuild.cuh"

namespace aot
{
namespace forest
{
// The barrier and the outcome of one persistent build (zeroed before the launch).
struct LevelStatus
{
    GridBarrier bar;
    int entriesOverflow; // the leaf arrays hold fewer entries than the forest needs
    int tooManyRounds;   // a system's rounds would not converge within maxDepth
    int historyMismatch; // a system's derived history does not end at its tree
    int deepest;         // deepest level holding units
    long long entries;   // entries of all systems (leaves and sentinels)
};

struct LevelArgs
{
    lb::Arena a;
    KeyIndex idx;     // sorted keys of all systems and their sample
    Bufs f;
    LevelStatus *ls;
    u32 capacity;     // entries the leaf arrays hold
    unsigned bucket;
    int maxDepth;
    HilbertTables h;
};

template <bool Hilbert>
static __global__ void __launch_bounds__(lb::kThreads) levelBuildKernel(LevelArgs p)
{
    using namespace lb;
    __shared__ unsigned char sNext[48 * 8], sDec[48 * 8];
    __shared__ u32 sBin[kContribBins];
    __shared__ unsigned long long sVal[kContribBins];
    __shared__ int sBins, sRounds;
    __shared__ i64 sWarp[kThreads / 32];
    __shared__ i64 sCarry;
    const Arena &a = p.a;
    Control &c = *a.ctl;
    LevelStatus *ls = p.ls;
    const u32 rank = blockIdx.x * blockDim.x + threadIdx.x, size = gridDim.x * blockDim.x;
    const int S = p.f.numSystems;
    if (vload(p.f.st->error)) return;  // the sort gave up: the host reports it
    if constexpr (Hilbert)
    {
        for (int k = threadIdx.x; k < 48 * 8; k += blockDim.x)
        {
            sNext[k] = p.h.encNext[k];
            sDec[k] = p.h.decOct[k];
        }
    }
    // roots, and zeroed history bins
    for (size_t i = rank; i < size_t(S) * kContribBins; i += size) a.contrib[i] = 0;
    for (size_t i = rank; i < size_t(S) * kArrivals; i += size) a.landed[i] = 0;
    for (u32 s = rank; s < u32(S); s += size)
    {
        const u32 active = p.f.sys[s].active;
        u32 root = kLeaf;
        if (active > p.bucket)
        {
            const u32 g = atomicAdd(&c.levelCount[0], 1u);
            if (g < a.cap)
            {
                u32 *row = a.rows + size_t(g) * kRow;
                const u32 base = p.f.systems[s].base;
                row[0] = 0;
                row[1] = 0;
                row[2] = base;
                row[10] = base + active;
                row[11] = withUnit(regionWord(0, 0, splitDepth(false, active, p.bucket, 0)), 0, kHilbertStart);
                a.usys[g] = s;
                root = g;
            }
            else
            {
                c.overflow = 1;
            }
        }
        a.sysRoot[s] = root;
    }
    if (!gridBarrier(&ls->bar)) return;
    // levels: every CTA reads the same counts and flags after a barrier
    int deepest = -1;
    for (int l = 0; l < int(kOctLevels); ++l)
    {
        const u32 start = vload(c.levelStart[l]), count = vload(c.levelCount[l]);
        if (vload(c.overflow) | vload(c.late) || count == 0) break;
        deepest = l;
        expandUnits(a, p.idx, l, start, count, rank, size);
        if (!gridBarrier(&ls->bar)) return;
        classifyUnits<false, Hilbert, true>(a, l, p.bucket, start, count, sNext, sDec, nullptr, nullptr, rank, size);
        if (!gridBarrier(&ls->bar)) return;
    }
    if (vload(c.overflow) | vload(c.late)) return;
    for (int l = deepest; l >= 0; --l)
    {
        leafCountUnits(a, vload(c.levelStart[l]), vload(c.levelCount[l]), rank, size);
        if (!gridBarrier(&ls->bar)) return;
    }
    // layout (CTA 0): systems one after the other, each followed by its sentinel
    if (blockIdx.x == 0)
    {
        if (threadIdx.x == 0) sCarry = 0;
        __syncthreads();
        for (int s0 = 0; s0 < S; s0 += kThreads)
        {
            const int s = s0 + int(threadIdx.x);
            u32 root = kLeaf, leaves = 0;
            if (s < S)
            {
                root = a.sysRoot[s];
                leaves = root == kLeaf ? 1u : a.leaves[root];
            }
            i64 total;
            const i64 excl = rb::blockExclusiveScan(s < S ? i64(leaves) + 1 : 0, sWarp, total);
            const i64 first = sCarry + excl;
            if (s < S)
            {
                SysState &ss = p.f.sys[s];
                ss.start = int(first);
                ss.leaves = int(leaves);
                ss.startNew = int(first);
                ss.sentinelNew = int(first + leaves);
                ss.changed = 0;
                ss.rejected = 0;
                ss.proposal = int(leaves) + 1;
                ss.needsResize = 0;
                ss.frozen = 0;
                if (first + i64(leaves) < i64(p.capacity))
                {
                    const u32 base = p.f.systems[s].base;
                    p.f.K[0][first + leaves] = kMaxKey;
                    p.f.B[0][first + leaves] = base + ss.active;
                    p.f.SEG[0][first + leaves] = s;
                    if (root == kLeaf)
                    {
                        p.f.K[0][first] = 0;
                        p.f.B[0][first] = base;
                        p.f.SEG[0][first] = s;
                    }
                }
                if (root != kLeaf) a.offset[root] = u32(first);
            }
            __syncthreads();
            if (threadIdx.x == 0) sCarry += total;
            __syncthreads();
        }
        if (threadIdx.x == 0)
        {
            const i64 entries = sCarry;
            ls->entries = entries;
            ls->deepest = deepest;
            if (entries > i64(p.capacity)) ls->entriesOverflow = 1;
            State &st = *p.f.st;
            const int err = st.error;
            st = State{};
            st.error = err;
            st.entries = int(entries);
            st.proposal = entries;
        }
    }
    if (!gridBarrier(&ls->bar)) return;
    if (vload(ls->entriesOverflow)) return;
    // each system's leaves after every round that changes it: a final leaf at
    // (arrival a, region depth k, relative level j) stands for
    // 8^max(0, k - (t - a - 1) - j) leaves in round t, a landed internal node
    // for one; the rounds end at max(a + 1 + k - j)
    for (int s = blockIdx.x; s < S; s += gridDim.x)
    {
        if (threadIdx.x == 0)
        {
            sBins = 0;
            sRounds = 0;
        }
        __syncthreads();
        const unsigned long long *cb = a.contrib + size_t(s) * kContribBins;
        for (int k = threadIdx.x; k < kContribBins; k += kThreads)
        {
            const unsigned long long v = cb[k];
            if (!v) continue;
            const int slot = atomicAdd(&sBins, 1);
            sBin[slot] = u32(k);
            sVal[slot] = v;
            const int j = k % kJumps, kk = (k / kJumps) % kJumps, ai = k / (kJumps * kJumps);
            atomicMax(&sRounds, ai + 1 + kk - j);
        }
        __syncthreads();
        const int rounds = sRounds, nb = sBins;
        const int t = int(threadIdx.x) + 1;
        if (t <= rounds)
        {
            unsigned long long at = t < kArrivals ? a.landed[size_t(s) * kArrivals + t] : 0ull;
            for (int q = 0; q < nb; ++q)
            {
                const int k = int(sBin[q]);
                const int j = k % kJumps, kk = (k / kJumps) % kJumps, ai = k / (kJumps * kJumps);
                if (ai + 1 > t) continue;
                const int e = kk - (t - ai - 1) - j;
                at += sVal[q] << (3 * (e > 0 ? e : 0));
            }
            if (t <= p.maxDepth) p.f.history[size_t(t - 1) * S + s] = (long long)at;
            if (t == rounds && at != u64(p.f.sys[s].leaves)) ls->historyMismatch = 1;
        }
        if (threadIdx.x == 0)
        {
            p.f.sys[s].iteration = rounds;
            if (rounds > p.maxDepth) ls->tooManyRounds = 1;
        }
        __syncthreads();
    }
    // placement, shallowest level first (a unit's first entry comes from its parent)
    for (int l = 0; l <= deepest; ++l)
    {
        placeUnits<false>(a, p.f.K[0], p.f.B[0], nullptr, nullptr, p.f.SEG[0], l, vload(c.levelStart[l]),
                          vload(c.levelCount[l]), p.capacity, rank, size);
        if (!gridBarrier(&ls->bar)) return;
    }
    const i64 E = vload(ls->entries);
    for (i64 i = rank; i < E; i += size)
        p.f.N[i] = p.f.K[0][i] == kMaxKey ? 0u : p.f.B[0][i + 1] - p.f.B[0][i];
}

}  // namespace forest
}  // namespace aot
