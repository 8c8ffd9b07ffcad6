// ao_oracle.cpp -- CPU oracle for the adaptive-tree path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the host and in plain
// sequential C++, the algorithm of nrottstegge/Adaptive_Trees for
// adaptive_octree::Tree<Real, Octree|Binary>: SFC key generation, the stable
// (key, slot) order of the particle sort, the iterative octree build, the
// fixed-pass graph update with its capacity rejection, the binary k-d passes
// and the traversal-free tree views.  Only tests/, the smoke check and the
// CPU-baseline leg of bench.py may load it.  The product library never calls
// into this file.
//
// Each function names the reference file:line it follows (paths relative to
// the reference project root).  Parity of this restatement is pinned against
// the reference's golden vectors (tests/verification_data/reference_output,
// checked by tests/test_oracle_golden.py) and, on a GPU host, against the
// reference library itself (oracle/_ref).
//
// Semantics are modelled at host synchronisation points: after build(),
// doBuffersNeedResize() and the getters, the oracle holds what the reference
// would report there.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace aoo
{
using u8 = std::uint8_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;
using i64 = std::int64_t;

constexpr unsigned kOctLevels = 21;                 // maxTreeLevel<u64>, sfc_keys.cuh:33-36
constexpr unsigned kBinDepth = 63;                  // maxBinaryDepth, config.hpp:47
constexpr u64 kMaxKey = u64(1) << 63;               // maxKey, config.hpp:48
constexpr u64 kInvalidKey = ~u64(0);                // invalidParticleKey, config.hpp:43
constexpr int kInvalidNode = -1;                    // invalidNodeIndex, config.hpp:42

// ---------------------------------------------------------------------------
// Integer helpers (sfc_keys.cuh:62-142, helpers.cuh:65-107)
// ---------------------------------------------------------------------------
static inline int clz64(u64 x) { return x ? __builtin_clzll(x) : 64; }
static inline int clz32(u32 x) { return x ? __builtin_clz(x) : 32; }

// nodeRange<u64>(level), sfc_keys.cuh:92-97
static inline u64 octRange(unsigned level) { return u64(1) << (3u * (kOctLevels - level)); }
// treeLevel<u64>(range), sfc_keys.cuh:100-104
static inline unsigned octLevel(u64 range) { return unsigned(clz64(range - 1) - 1) / 3; }
// octalDigit, sfc_keys.cuh:108-112
static inline unsigned octDigit(u64 code, unsigned position)
{
    return unsigned(code >> (3u * (kOctLevels - position))) & 7u;
}
// log8ceil<unsigned> as used on the split op code (octree_rebalance.cuh:349)
static inline unsigned log8ceil32(u32 n)
{
    if (n == 0) return 0;
    const int lz = clz32(n - 1);
    return 10u - unsigned(lz - 2) / 3u;
}

// lowerBound, helpers.cuh:65-85
static inline size_t lowerBound(const u64 *a, size_t n, u64 v)
{
    return size_t(std::lower_bound(a, a + n, v) - a);
}
// upperBound, helpers.cuh:87-107
static inline size_t upperBound(const u64 *a, size_t n, u64 v)
{
    return size_t(std::upper_bound(a, a + n, v) - a);
}

// ---------------------------------------------------------------------------
// Morton / Hilbert (sfc_keys.cuh:174-347)
// ---------------------------------------------------------------------------
// 21-bit spread to every third bit (sfc_keys.cuh:174-183).
static inline u64 spread3(u64 v)
{
    u64 x = v & 0x1fffffull;
    x = (x | x << 32) & 0x001f00000000ffffull;
    x = (x | x << 16) & 0x001f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
// Inverse of spread3 (sfc_keys.cuh:186-195): gather every third bit.
static inline u64 gather3(u64 v)
{
    u64 r = 0;
    for (unsigned b = 0; b < 21; ++b) r |= ((v >> (3 * b)) & 1ull) << b;
    return r;
}
// iMorton<u64>, sfc_keys.cuh:198-215: x supplies the top bit of each triplet.
static inline u64 morton(unsigned ix, unsigned iy, unsigned iz)
{
    return (spread3(ix) << 2) | (spread3(iy) << 1) | spread3(iz);
}
struct C3 { unsigned x, y, z; };
// decodeMorton<u64>, sfc_keys.cuh:222-237
static inline C3 demorton(u64 k)
{
    return {unsigned(gather3(k >> 2)), unsigned(gather3(k >> 1)), unsigned(gather3(k))};
}
// iHilbert<u64>, sfc_keys.cuh:248-290 (the Cornerstone 3-D Hilbert curve).
static inline u64 hilbert(unsigned px, unsigned py, unsigned pz)
{
    static const unsigned order[8] = {0, 1, 3, 2, 7, 6, 4, 5};
    u64 key = 0;
    for (int level = int(kOctLevels) - 1; level >= 0; --level)
    {
        const unsigned xi = (px >> level) & 1u, yi = (py >> level) & 1u, zi = (pz >> level) & 1u;
        key = (key << 3) + order[(xi << 2) | (yi << 1) | zi];
        const unsigned ny = !yi, nz = !zi;
        if (xi & (ny | zi)) px = ~px;
        if ((xi & (yi | zi)) | (yi & nz)) py = ~py;
        if ((xi & ny & nz) | (yi & nz)) pz = ~pz;
        if (zi)
        {
            const unsigned t = px;
            px = py;
            py = pz;
            pz = t;
        }
        else if (ny)
        {
            std::swap(px, pz);
        }
    }
    return key;
}
// decodeHilbert<u64>, sfc_keys.cuh:293-331
static inline C3 dehilbert(u64 key)
{
    unsigned px = 0, py = 0, pz = 0;
    for (unsigned level = 0; level < kOctLevels; ++level)
    {
        const unsigned oct = unsigned(key >> (3 * level)) & 7u;
        const unsigned xi = oct >> 2, yi = (oct >> 1) & 1u, zi = oct & 1u;
        if (yi ^ zi)
        {
            const unsigned t = px;
            px = pz;
            pz = py;
            py = t;
        }
        else if ((!xi && !yi && !zi) || (xi && yi && zi))
        {
            std::swap(px, pz);
        }
        const unsigned mask = (1u << level) - 1;
        if (xi & (yi | zi)) px ^= mask;
        if ((xi & ((!yi) | (!zi))) | ((!xi) & yi & zi)) py ^= mask;
        if ((xi & (!yi) & (!zi)) | (yi & zi)) pz ^= mask;
        px |= xi << level;
        py |= (xi ^ yi) << level;
        pz |= (yi ^ zi) << level;
    }
    return {px, py, pz};
}
static inline u64 sfcEncode(unsigned x, unsigned y, unsigned z, bool h)
{
    return h ? hilbert(x, y, z) : morton(x, y, z);
}
static inline C3 sfcDecode(u64 k, bool h) { return h ? dehilbert(k) : demorton(k); }

// Same-level periodic neighbour (sfc_keys.cuh:376-410).
static inline int pbc(int x)
{
    const int R = 1 << kOctLevels;
    const int r = x < 0 ? x + R : x;
    return r >= R ? r - R : r;
}
static inline u64 neighbourKey(const C3 &c, unsigned cube, unsigned level, int dx, int dy, int dz, bool h)
{
    const int x = pbc(int(c.x) + dx * int(cube));
    const int y = pbc(int(c.y) + dy * int(cube));
    const int z = pbc(int(c.z) + dz * int(cube));
    return sfcEncode(unsigned(x), unsigned(y), unsigned(z), h) & ~(octRange(level) - 1);
}

// GPU float->integer conversions (cvt.rzi with saturation, NaN -> 0), which
// the reference kernels use for int(...) and KeyType(...).
static inline int satI32(double v)
{
    if (std::isnan(v)) return 0;
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return int(-2147483647 - 1);
    return int(std::trunc(v));
}
static inline u64 satU64(double v)
{
    if (std::isnan(v) || v <= 0) return 0;
    if (v >= 18446744073709551616.0) return ~u64(0);
    return u64(v);
}

// Box + quantisation (sfc_keys.cuh:420-496).  Arithmetic in Real; the
// device code contracts floor(x*mx) - xmin*mx into one fused multiply-add.
template <class T>
struct QBox
{
    T xmin, ymin, zmin, ilx, ily, ilz;
    unsigned bx, by, bz;
};
template <class T>
static QBox<T> makeQBox(const double *b)
{
    const T xmin = T(b[0]), xmax = T(b[1]), ymin = T(b[2]), ymax = T(b[3]), zmin = T(b[4]), zmax = T(b[5]);
    QBox<T> q;
    q.xmin = xmin;
    q.ymin = ymin;
    q.zmin = zmin;
    q.ilx = T(1) / (xmax - xmin);
    q.ily = T(1) / (ymax - ymin);
    q.ilz = T(1) / (zmax - zmin);
    const T lx = xmax - xmin, ly = ymax - ymin, lz = zmax - zmin;
    const T md = std::max(std::max(lx, ly), lz);
    const T bias = T(0.5849625007211563);
    q.bx = kOctLevels - unsigned(std::floor(std::log2(md / lx) + bias));
    q.by = kOctLevels - unsigned(std::floor(std::log2(md / ly) + bias));
    q.bz = kOctLevels - unsigned(std::floor(std::log2(md / lz) + bias));
    return q;
}
template <class T>
static inline int quantise(T v, T vmin, T il, unsigned bits)
{
    const T m = T(1u << bits) * il;
    const T f = std::floor(v * m);
    const T q = std::fma(-vmin, m, f);
    int i = satI32(double(q));
    return std::min(i, int(1u << bits) - 1);
}
template <class T>
static inline u64 octreeKey(T x, T y, T z, const QBox<T> &q, bool h)
{
    const T esc = std::numeric_limits<T>::max();
    if (x == esc && y == esc && z == esc) return kInvalidKey;  // config.hpp:107-113
    const unsigned ix = unsigned(quantise(x, q.xmin, q.ilx, q.bx)) & 0x1fffffu;
    const unsigned iy = unsigned(quantise(y, q.ymin, q.ily, q.by)) & 0x1fffffu;
    const unsigned iz = unsigned(quantise(z, q.zmin, q.ilz, q.bz)) & 0x1fffffu;
    return sfcEncode(ix, iy, iz, h);
}

// Binary longest-side geometry (binary_node.cuh:17-40) and key
// (binary_node.cuh:43-59, kdtree3d_rebalance.cuh:248-259).
struct Geometry { u8 axis[kBinDepth]; };
static Geometry makeGeometry(const double *b, unsigned maxDepth)
{
    if (maxDepth > kBinDepth) throw std::invalid_argument("Binary maxDepth exceeds key precision");
    long double len[3] = {(long double)b[1] - (long double)b[0], (long double)b[3] - (long double)b[2],
                          (long double)b[5] - (long double)b[4]};
    for (auto s : len)
        if (!(s > 0) || !std::isfinite(s)) throw std::invalid_argument("Tree box must have finite positive sides");
    Geometry g;
    for (unsigned d = 0; d < kBinDepth; ++d)
    {
        unsigned a = 0;
        if (len[1] > len[a]) a = 1;
        if (len[2] > len[a]) a = 2;
        g.axis[d] = u8(a);
        len[a] *= 0.5L;
    }
    return g;
}
static inline u64 fixed63(double v)
{
    // cmax(0, cmin(1, v)) with the reference's comparison order (NaN passes through).
    const double cm = (1.0 < v) ? 1.0 : v;
    const double cc = (0.0 > cm) ? 0.0 : cm;
    const u64 k = satU64(cc * 9223372036854775808.0);
    return std::min(k, kMaxKey - 1);
}
template <class T>
static inline u64 binaryKey(T x, T y, T z, const double *b, const Geometry &g)
{
    const T esc = std::numeric_limits<T>::max();
    if (x == esc && y == esc && z == esc) return kInvalidKey;
    const double vx = (double(x) - double(T(b[0]))) / (double(T(b[1])) - double(T(b[0])));
    const double vy = (double(y) - double(T(b[2]))) / (double(T(b[3])) - double(T(b[2])));
    const double vz = (double(z) - double(T(b[4]))) / (double(T(b[5])) - double(T(b[4])));
    u64 c[3] = {fixed63(vx), fixed63(vy), fixed63(vz)};
    u64 key = 0;
    for (unsigned d = 0; d < kBinDepth; ++d)
    {
        u64 &v = c[g.axis[d]];
        key = (key << 1) | ((v >> (kBinDepth - 1)) & 1u);
        v <<= 1;
    }
    return key;
}

// ---------------------------------------------------------------------------
// State and capacity bookkeeping
// ---------------------------------------------------------------------------
// RebalanceState, helpers.cuh:109-120
struct State
{
    int changed = 0, converged = 0, numLeaves = 1, newNumLeaves = 1, needsResize = 0, numNodes = 0,
        activeBuffer = 0;
    u32 numActive = 0;
};
// thrust::device_vector size/capacity, modelled for the buffers whose
// capacity feeds leafCapacity (octree.cu:453-457).
struct Cap { size_t size = 0, cap = 0; };
static void capResize(Cap &v, size_t n)  // vector_base::append growth
{
    if (n > v.cap) v.cap = std::max(v.size + std::max(v.size, n - v.size), 2 * v.cap);
    v.size = n;
}
static void capReserve(Cap &v, size_t n) { if (n > v.cap) v.cap = n; }
static void capHeadroom(Cap &v, size_t req)  // resizeWithHeadroom, helpers.cuh:122-141
{
    if (req > v.cap) v.cap = req + req / 4;
    v.size = req;
}

struct Views { bool ts = false, pc = false, pm = false; bool any() const { return ts || pc || pm; } };

// TreeView<LevelBits> (tree_view.hpp:20-115, tree_view.cu:755-1134)
struct TreeViewO
{
    unsigned b = 3;  // LevelBits
    bool scratch = false;
    size_t leafCap = 0, particleCap = 0;
    Views prepared;
    bool depthAlloc = false;
    u8 maxDepth = 0;
    size_t numNodesLogical = 0, mappingLogical = 0;
    std::vector<u64> box, pmap;
    std::vector<u8> split, depth;
    std::vector<int> parent, child, levelOffset;
    std::vector<u32> pbegin, pcount;

    unsigned maxLevel() const { return kBinDepth / b; }
    unsigned children() const { return 1u << b; }
    size_t nodesFor(size_t leaves) const { return leaves + (leaves - 1) / (children() - 1); }

    void prepare(size_t leafCapacity, size_t n, Views v)  // tree_view.cu:755-791
    {
        if (!v.any()) return;
        leafCap = std::max(leafCap, leafCapacity);
        particleCap = std::max(particleCap, n);
        prepared.ts |= v.ts;
        prepared.pc |= v.pc;
        prepared.pm |= v.pm;
        scratch = true;
        depthAlloc = true;
        const size_t nodes = nodesFor(leafCap);
        if (box.size() < nodes)
        {
            box.resize(nodes);
            split.resize(nodes);
            depth.resize(nodes);
            parent.resize(nodes);
            child.resize(nodes);
        }
        levelOffset.resize(maxLevel() + 2);
        if (prepared.pc && pbegin.size() < nodes)
        {
            pbegin.resize(nodes);
            pcount.resize(nodes + 1);
        }
        if (prepared.pm && pmap.size() < particleCap) pmap.resize(particleCap);
    }
    void syncSizes(size_t leaves, size_t active)  // tree_view.cu:793-813
    {
        if (!scratch || leaves > leafCap) return;
        numNodesLogical = nodesFor(leaves);
        if (prepared.pm) mappingLogical = active;
    }
    // Builds the view of the active tree.  Returns false if the request must
    // set needsResize instead (tree_view.cu:829-845).
    bool build(const std::vector<u64> &K, const std::vector<u32> &N, size_t L, const std::vector<u64> &P, Views v,
               State &st)
    {
        if (!v.any()) return true;
        if (!scratch || (v.pc && !prepared.pc) || (v.pm && (!prepared.pm || P.size() > particleCap)))
        {
            st.needsResize = 1;
            return false;
        }
        if (L > leafCap)
        {
            st.needsResize = 1;
            return false;
        }
        const size_t numNodes = nodesFor(L);
        st.numNodes = int(numNodes);
        // Breadth-first construction.  Nodes of level l+1 are grouped by child
        // slot, and inside a slot by the order of their parents: the
        // child-centric layout of tree_view.cu:301-401 (the same order the
        // reference test's CPU BFS checks, tree_test.cu:660-778).
        struct Node { u64 begin, end; unsigned level; int parent, first; size_t kpos; };
        std::vector<Node> nodes;
        nodes.reserve(numNodes);
        nodes.push_back({0, kMaxKey, 0, kInvalidNode, kInvalidNode, 0});
        std::vector<int> offsets(maxLevel() + 2, 0);
        size_t lb = 0, le = 1;
        unsigned maxLeafLevel = 0;
        for (unsigned lev = 0; lev <= maxLevel(); ++lev)
        {
            offsets[lev] = int(lb);
            std::vector<int> parents;
            for (size_t i = lb; i < le; ++i)
            {
                const size_t pos = size_t(std::lower_bound(K.begin(), K.begin() + L + 1, nodes[i].begin) - K.begin());
                if (pos >= L || K[pos] != nodes[i].begin) throw std::runtime_error("view: node start is not a boundary");
                nodes[i].kpos = pos;
                if (nodes[i].end != K[pos + 1])
                {
                    nodes[i].first = int(le + parents.size());
                    parents.push_back(int(i));
                }
                else
                {
                    maxLeafLevel = std::max(maxLeafLevel, lev);
                }
            }
            for (unsigned s = 0; s < children(); ++s)
                for (int p : parents)
                {
                    const u64 w = (nodes[p].end - nodes[p].begin) >> b;
                    const u64 bg = nodes[p].begin + u64(s) * w;
                    nodes.push_back({bg, bg + w, lev + 1, p, kInvalidNode, 0});
                }
            lb = le;
            le = nodes.size();
        }
        offsets[maxLevel() + 1] = int(nodes.size());
        if (nodes.size() != numNodes) throw std::runtime_error("view: node count mismatch");
        maxDepth = u8(maxLeafLevel);
        for (size_t l = 0; l < offsets.size(); ++l) levelOffset[l] = offsets[l];
        const size_t n = P.size();
        for (size_t i = 0; i < numNodes; ++i)
        {
            const Node &nd = nodes[i];
            box[i] = (u64(1) << (b * nd.level)) | (nd.begin >> (kBinDepth - b * nd.level));
            split[i] = nd.first != kInvalidNode;
            depth[i] = u8(nd.level);
            parent[i] = nd.parent;
            child[i] = nd.first;
        }
        // Leaf particle ranges: exclusive scan of N (tree_view.cu:691-703).
        std::vector<u32> leafBegin(L);
        {
            u32 acc = 0;
            for (size_t i = 0; i < L; ++i)
            {
                leafBegin[i] = acc;
                acc += N[i];
            }
        }
        if (v.pc)
        {
            for (size_t i = 0; i < numNodes; ++i)
            {
                if (nodes[i].first == kInvalidNode)  // buildLeafNodesKernel, 488-538
                {
                    pbegin[i] = leafBegin[nodes[i].kpos];
                    pcount[i] = N[nodes[i].kpos];
                }
                else  // buildInternalNodesKernel, 472-481
                {
                    const size_t bgn = lowerBound(P.data(), n, nodes[i].begin);
                    const size_t end = lowerBound(P.data(), n, nodes[i].end);
                    pbegin[i] = u32(bgn);
                    pcount[i] = u32(end - bgn);
                }
            }
            pcount[numNodes] = pcount[0];
        }
        if (v.pm)  // fillSfcParticleIndexKernel, 542-562
        {
            std::vector<int> leafToNode(L, 0);
            for (size_t i = 0; i < numNodes; ++i)
                if (nodes[i].first == kInvalidNode) leafToNode[nodes[i].kpos] = int(i);
            for (size_t p = 0; p < n; ++p)
            {
                if (P[p] >= kMaxKey)
                {
                    pmap[p] = ~u64(0);
                    continue;
                }
                const size_t leaf = upperBound(K.data(), L, P[p]) - 1;
                pmap[p] = u64(std::int64_t(leafToNode[leaf]));
            }
        }
        return true;
    }
};

// ---------------------------------------------------------------------------
// Octree model (octree.cu, octree_rebalance.cuh)
// ---------------------------------------------------------------------------
struct Tree
{
    // configuration
    int kind = 0;  // 0 octree, 1 binary
    int real = 1;  // 0 float, 1 double
    size_t n = 0;
    const void *x = nullptr, *y = nullptr, *z = nullptr;
    unsigned bucket = 64, maxDepth = 21, iterations = 2;
    bool nf = false, hil = false;
    double box[6] = {0, 1, 0, 1, 0, 1};
    Views cfgViews, preparedViews;
    Geometry geom{};
    // device-equivalent state
    std::vector<u64> P, K;
    std::vector<u32> Perm, N, NF;
    std::vector<u8> GCM;
    State st;
    size_t leafCapacity = 0;
    Cap Kc, Tc;  // K_d and tmpTree capacities (octree)
    bool built = false;
    TreeViewO view;
    // host-visible values refreshed at readbacks
    size_t hostLeaves = 1, hostActive = 0, hostNodes = 0;
    // trajectory counters (diagnostics)
    unsigned buildIterations = 0;

    size_t L() const { return K.size() - 1; }

    // --- keys + sort (octree.cu:285-307; kdtree3d.cu:161-172) ---
    template <class T>
    void keysT()
    {
        const T *px = static_cast<const T *>(x), *py = static_cast<const T *>(y), *pz = static_cast<const T *>(z);
        std::vector<u64> keys(n);
        if (kind == 0)
        {
            const QBox<T> q = makeQBox<T>(box);
            for (size_t i = 0; i < n; ++i) keys[i] = octreeKey<T>(px[i], py[i], pz[i], q, hil);
        }
        else
        {
            for (size_t i = 0; i < n; ++i) keys[i] = binaryKey<T>(px[i], py[i], pz[i], box, geom);
        }
        std::vector<std::pair<u64, u32>> kv(n);
        for (size_t i = 0; i < n; ++i) kv[i] = {keys[i], u32(i)};
        std::sort(kv.begin(), kv.end());  // lexicographic = stable LSD order
        P.resize(n);
        Perm.resize(n);
        for (size_t i = 0; i < n; ++i)
        {
            P[i] = kv[i].first;
            Perm[i] = kv[i].second;
        }
    }
    void computeKeys()
    {
        if (real == 0) keysT<float>();
        else keysT<double>();
    }
    u32 activeCount() const { return n ? u32(lowerBound(P.data(), n, kMaxKey)) : 0u; }

    // --- octree per-leaf quantities ---
    u32 leafCount(u64 a, u64 b) const  // calculateNodeCount, octree_rebalance.cuh:368-379
    {
        return u32(lowerBound(P.data(), n, b) - lowerBound(P.data(), n, a));
    }
    // computeNFCooperative, octree_rebalance.cuh:579-634
    u64 nearField(u64 start, unsigned level, u32 *own) const
    {
        const unsigned cube = 1u << (kOctLevels - level);
        const C3 c = sfcDecode(start, hil);
        const u64 range = octRange(level);
        u64 pop = 0, centre = 0;
        for (int cell = 0; cell < 27; ++cell)
        {
            const int dx = cell % 3 - 1, dy = (cell / 3) % 3 - 1, dz = cell / 9 - 1;
            const u64 key = cell == 13 ? start : neighbourKey(c, cube, level, dx, dy, dz, hil);
            const u64 cnt = u64(lowerBound(P.data(), n, key + range) - lowerBound(P.data(), n, key));
            pop += cnt;
            if (cell == 13) centre = cnt;
        }
        if (own) *own = u32(std::min<u64>(centre, 0xffffffffull));
        return centre * pop;
    }
    // siblingIndexAndLevel, octree_rebalance.cuh:26-50
    int siblingIndex(const std::vector<u64> &t, int numNodes, int i, unsigned &level) const
    {
        const u64 s = t[i];
        level = octLevel(t[i + 1] - s);
        if (level == 0) return -1;
        const int sib = int(octDigit(s, level));
        const int first = i - sib;
        if (first < 0 || first > numNodes - 8) return -1;
        return t[first + 8] == t[first] + octRange(level - 1) ? sib : -1;
    }
    // calculateNodeOp (NFCount branch), octree_rebalance.cuh:174-249
    int nodeOp(int i, int numNodes) const
    {
        unsigned level = 0;
        const int sib = siblingIndex(K, numNodes, i, level);
        if (sib >= 0)
        {
            const int first = i - sib;
            if (first + 8 <= numNodes && GCM[first]) return sib == 0 ? 1 : 0;
        }
        const u64 c = NF[i], b = bucket;
        if (c > b * 262144 && level + 3 < kOctLevels) return 4096;
        if (c > b * 4096 && level + 2 < kOctLevels) return 512;
        if (c > b * 64 && level + 1 < kOctLevels) return 64;
        if (c > b && level < kOctLevels) return 8;
        return 1;
    }
    // calculateNodeOp (LeafCount branch), octree_rebalance.cuh:188-225.  The
    // thresholds are 32-bit unsigned products (count > bucketSize * 512).
    int nodeOpLC32(int i, int numNodes) const
    {
        unsigned level = 0;
        const int sib = siblingIndex(K, numNodes, i, level);
        if (sib > 0)
        {
            const u32 *g = N.data() + i - sib;
            u64 parent = 0;
            for (int s = 0; s < 8; ++s) parent += g[s];
            if (parent <= u64(bucket)) return 0;
        }
        const u32 c = N[i];
        if (c > u32(bucket * 512u) && level + 3 < kOctLevels) return 4096;
        if (c > u32(bucket * 64u) && level + 2 < kOctLevels) return 512;
        if (c > u32(bucket * 8u) && level + 1 < kOctLevels) return 64;
        if (c > bucket && level < kOctLevels) return 8;
        return 1;
    }
    int decide(int i, int numNodes) const { return nf ? nodeOp(i, numNodes) : nodeOpLC32(i, numNodes); }

    // Group leader test used for parent-NF refresh (octree_rebalance.cuh:83-105).
    bool groupLeader(const std::vector<u64> &t, int numNodes, int first, const std::vector<u8> *dirty) const
    {
        if (first + 8 > numNodes) return false;
        if (dirty && !(*dirty)[first]) return false;
        unsigned lev = 0;
        return siblingIndex(t, numNodes, first, lev) == 0 && lev > 0;
    }
    void refreshGroup(int first)  // computeGroupCanMergeKernel body, 636-677
    {
        const unsigned lev = octLevel(K[first + 1] - K[first]);
        const u64 parentNF = nearField(K[first], lev - 1, nullptr);
        GCM[first] = parentNF <= u64(1) * u64(bucket);
    }

    // One split/merge materialisation (processNode, octree_rebalance.cuh:253-365).
    // Returns the new tree; NF-mode caches follow the reference's reuse rules.
    void scatter(const std::vector<i64> &offs, int numOld, std::vector<u8> &nfDirty, std::vector<u8> &groupDirty)
    {
        const size_t newL = size_t(offs[numOld]);
        std::vector<u64> Kn(newL + 1);
        std::vector<u32> Nn(nf ? newL : 0), NFn(nf ? newL : 0);
        std::vector<u8> Gn(nf ? newL : 0);
        if (nf)
        {
            nfDirty.assign(newL, 0);
            groupDirty.assign(newL, 0);
        }
        auto op = [&](int i) { return int(offs[i + 1] - offs[i]); };
        for (int i = 0; i < numOld; ++i)
        {
            const u64 s = K[i];
            const unsigned level = octLevel(K[i + 1] - s);
            const int code = op(i);
            const i64 ni = offs[i];
            if (code == 0) continue;
            if (code == 1)
            {
                Kn[ni] = s;
                if (nf)
                {
                    const bool leader = i + 1 < numOld && op(i + 1) == 0;
                    if (leader)
                    {
                        nfDirty[ni] = 1;
                        groupDirty[ni] = 1;
                    }
                    else
                    {
                        Nn[ni] = N[i];
                        NFn[ni] = NF[i];
                        nfDirty[ni] = 0;
                        bool reusable = false;
                        unsigned sl = 0;
                        const int sib = siblingIndex(K, numOld, i, sl);
                        if (sib == 0 && i + 8 <= numOld)
                        {
                            reusable = true;
                            for (int s2 = 0; s2 < 8; ++s2)
                                if (op(i + s2) != 1)
                                {
                                    reusable = false;
                                    break;
                                }
                        }
                        if (reusable)
                        {
                            Gn[ni] = GCM[i];
                            groupDirty[ni] = 0;
                        }
                        else
                        {
                            groupDirty[ni] = 1;
                        }
                    }
                }
                continue;
            }
            const unsigned diff = code == 8 ? 1u : log8ceil32(u32(code));
            const u64 nr = octRange(level + diff);
            for (int c = 0; c < code; ++c)
            {
                Kn[ni + c] = s + u64(c) * nr;
                if (nf)
                {
                    nfDirty[ni + c] = 1;
                    groupDirty[ni + c] = 1;
                }
            }
        }
        Kn[newL] = kMaxKey;
        K.swap(Kn);
        if (nf)
        {
            N.swap(Nn);
            NF.swap(NFn);
            GCM.swap(Gn);
        }
    }
    // Count refresh after a materialisation (dirty-only in NF mode).
    void refreshAfterScatter(const std::vector<u8> &nfDirty, const std::vector<u8> &groupDirty)
    {
        const int Ln = int(L());
        if (!nf)
        {
            N.assign(Ln, 0);
            for (int i = 0; i < Ln; ++i) N[i] = leafCount(K[i], K[i + 1]);
            return;
        }
        for (int i = 0; i < Ln; ++i)
            if (nfDirty[i])
            {
                const unsigned lev = octLevel(K[i + 1] - K[i]);
                u32 own = 0;
                const u64 v = nearField(K[i], lev, &own);
                N[i] = own;
                NF[i] = u32(std::min<u64>(v, 0xffffffffull));
            }
        for (int i = 0; i < Ln; ++i)
            if (groupLeader(K, Ln, i, &groupDirty)) refreshGroup(i);
    }
    // Full refresh at the start of update() (refreshGraphCountsGpu with no
    // dirty lists, octree_rebalance.cuh:1112-1175).
    void refreshFull()
    {
        const int Ln = int(L());
        if (!nf)
        {
            N.assign(Ln, 0);
            for (int i = 0; i < Ln; ++i) N[i] = leafCount(K[i], K[i + 1]);
            return;
        }
        N.assign(Ln, 0);
        NF.assign(Ln, 0);
        if (GCM.size() < size_t(Ln)) GCM.resize(Ln, 0);
        for (int i = 0; i < Ln; ++i)
        {
            const unsigned lev = octLevel(K[i + 1] - K[i]);
            u32 own = 0;
            const u64 v = nearField(K[i], lev, &own);
            N[i] = own;
            NF[i] = u32(std::min<u64>(v, 0xffffffffull));
        }
        for (int i = 0; i < Ln; ++i)
            if (groupLeader(K, Ln, i, nullptr)) refreshGroup(i);
    }

    void prepareGraphBuffers(size_t capacity)  // octree.cu:182-241; kdtree3d.cu:96-116
    {
        if (kind == 0)
        {
            const size_t maxLeaves = (size_t(std::numeric_limits<int>::max()) - 1) / 8 * 7 + 1;
            if (capacity > maxLeaves) throw std::length_error("adaptive_octree: buffer capacity exceeds node index range");
            const size_t leaves = Kc.size - 1;
            leafCapacity = capacity;
            capReserve(Kc, capacity + 1);
            capResize(Kc, capacity + 1);
            capReserve(Tc, capacity + 1);
            capResize(Tc, capacity + 1);
            view.prepare(capacity, n, preparedViews);
            Kc.size = leaves + 1;
            Tc.size = leaves + 1;
            view.syncSizes(leaves, hostActive);
        }
        else
        {
            const size_t maxLeaves = size_t(std::numeric_limits<int>::max()) / 2 + 1;
            if (capacity > maxLeaves) throw std::length_error("adaptive_octree: buffer capacity exceeds node index range");
            leafCapacity = capacity;
            if (built && preparedViews.any()) view.prepare(leafCapacity, n, preparedViews);
            view.syncSizes(hostLeaves, hostActive);
        }
    }

    // --- octree build: octree.cu:427-469, rebalanceBuild 159-180 ---
    void octreeBuild()
    {
        Kc.size = 2;  // K_d.resize(2)
        st = State{};
        st.numLeaves = 0;
        st.newNumLeaves = 0;  // memset 0
        computeKeys();
        const u32 active = activeCount();
        K = {0, kMaxKey};
        N = {active};
        const u64 sq = u64(active) * active;
        NF = {sq > 0xffffffffull / 27ull ? 0xffffffffu : u32(27ull * sq)};
        GCM.clear();
        // rebalanceBuild: resetRebalanceState
        st.changed = 0;
        st.converged = 0;
        st.numActive = active;
        buildIterations = 0;
        for (unsigned it = 0; it < maxDepth; ++it)
        {
            const int numOld = int(L());
            // computeNodeOpsGpu, 453-522
            std::vector<i64> offs(numOld + 1, 0);
            bool changed = false;
            for (int i = 0; i < numOld; ++i)
            {
                const int o = decide(i, numOld);
                if (o != 1) changed = true;
                offs[i] = o;
            }
            if (!changed)
            {
                st.converged = 1;
                break;
            }
            i64 acc = 0;
            for (int i = 0; i <= numOld; ++i)
            {
                const i64 v = offs[i];
                offs[i] = acc;
                acc += v;
            }
            const int newNum = int(offs[numOld]);
            ++buildIterations;
            // updateOctreeGpu, 871-985: capacity effects
            capHeadroom(Tc, size_t(newNum) + 1);
            std::vector<u8> nfDirty, groupDirty;
            scatter(offs, numOld, nfDirty, groupDirty);
            std::swap(Kc, Tc);
            refreshAfterScatter(nfDirty, groupDirty);
        }
        const size_t leaves = L();
        const size_t cap = std::max({Kc.cap - 1, Tc.size == 0 ? size_t(0) : Tc.cap - 1,
                                     leaves + (leaves + 3) / 4});
        hostLeaves = leaves;
        prepareGraphBuffers(cap);
        // finishBuildStateKernel, octree.cu:40-47
        st.numLeaves = st.newNumLeaves = int(leaves);
        st.changed = st.converged = st.needsResize = 0;
        st.numNodes = 0;
        st.activeBuffer = 0;
        built = true;
        buildViews(cfgViews);
        needsResize();
    }

    // --- octree update: octree.cu:471-481, rebalanceUpdate 243-282 ---
    void octreePass()  // updateOctreeGraphGpu, octree_rebalance.cuh:1275-1322
    {
        st.changed = 0;
        const int cap = int(leafCapacity);
        const int numOld = st.numLeaves;
        std::vector<i64> offs(size_t(cap) + 1, 0);
        for (int t = 0; t <= cap; ++t)
        {
            int d = 0;
            if (!st.converged && !st.needsResize && t < numOld)
            {
                d = decide(t, numOld);
                if (d != 1) st.changed = 1;
            }
            offs[t] = d;
        }
        i64 acc = 0;
        for (int t = 0; t <= cap; ++t)
        {
            const i64 v = offs[t];
            offs[t] = acc;
            acc += v;
        }
        // graphCheckCapacityKernel, 1211-1232
        if (st.converged) return;
        if (st.needsResize || !st.changed)
        {
            st.converged = 1;
            return;
        }
        if (offs[cap] > i64(cap))
        {
            st.needsResize = 1;
            st.converged = 1;
            return;
        }
        st.newNumLeaves = int(offs[cap]);
        std::vector<i64> o2(offs.begin(), offs.begin() + numOld + 1);
        std::vector<u8> nfDirty, groupDirty;
        scatter(o2, numOld, nfDirty, groupDirty);
        st.numLeaves = st.newNumLeaves;
        st.activeBuffer ^= 1;
        refreshAfterScatter(nfDirty, groupDirty);
    }
    void octreeUpdate()
    {
        if (!built) throw std::logic_error("adaptive_octree: call build() before update()");
        computeKeys();
        st.changed = 0;
        st.converged = 0;
        st.numActive = activeCount();
        refreshFull();
        for (unsigned i = 0; i < iterations; ++i) octreePass();
        buildViews(cfgViews);
    }

    // --- binary backend: kdtree3d.cu, kdtree3d_rebalance.cuh ---
    static bool binSiblings(const std::vector<u64> &t, int count, int first)  // binary_node.cuh:91-98
    {
        if (first < 0 || first + 1 >= count) return false;
        const u64 r = t[first + 1] - t[first];
        return !(t[first] & r) && t[first + 2] - t[first + 1] == r;
    }
    void binaryRefresh()  // refreshCounts, kdtree3d.cu:139-145
    {
        st.changed = 0;
        st.converged = 0;
        st.numActive = activeCount();
        const int Ln = st.numLeaves;
        N.assign(Ln, 0);
        for (int i = 0; i < Ln; ++i)
            N[i] = st.numActive ? u32(lowerBound(P.data(), st.numActive, K[i + 1]) - lowerBound(P.data(), st.numActive, K[i]))
                                : 0u;
    }
    void binaryPass()  // updateBinaryGraphGpu, kdtree3d_rebalance.cuh:226-245
    {
        st.changed = 0;
        const int cap = int(leafCapacity);
        const int Ln = st.numLeaves;
        std::vector<i64> offs(size_t(cap) + 1, 0);
        for (int t = 0; t <= cap; ++t)
        {
            int op = 0;
            if (!st.converged && !st.needsResize && t < Ln)
            {
                const bool merge = t && binSiblings(K, Ln, t - 1) && u64(N[t - 1]) + N[t] <= bucket;
                op = merge ? 0 : (N[t] > bucket && unsigned(clz64(K[t + 1] - K[t])) < maxDepth ? 2 : 1);
                if (op != 1) st.changed = 1;
            }
            offs[t] = op;
        }
        i64 acc = 0;
        for (int t = 0; t <= cap; ++t)
        {
            const i64 v = offs[t];
            offs[t] = acc;
            acc += v;
        }
        if (st.converged) return;
        if (st.needsResize || !st.changed)
        {
            st.converged = 1;
            return;
        }
        if (offs[cap] > i64(cap))
        {
            st.needsResize = 1;
            st.converged = 1;
            return;
        }
        st.newNumLeaves = int(offs[cap]);
        std::vector<u64> Kn(size_t(st.newNumLeaves) + 1);
        for (int t = 0; t < Ln; ++t)
        {
            const int op = int(offs[t + 1] - offs[t]);
            if (!op) continue;
            const i64 tg = offs[t];
            Kn[tg] = K[t];
            if (op == 2) Kn[tg + 1] = K[t] + (K[t + 1] - K[t]) / 2;
        }
        Kn[st.newNumLeaves] = kMaxKey;
        K.swap(Kn);
        st.numLeaves = st.newNumLeaves;
        st.numNodes = (st.numLeaves - 1) * 2 + 1;
        st.activeBuffer ^= 1;
        // binaryLeafCountsKernel (not converged here)
        N.assign(st.numLeaves, 0);
        for (int i = 0; i < st.numLeaves; ++i)
            N[i] = st.numActive ? u32(lowerBound(P.data(), st.numActive, K[i + 1]) - lowerBound(P.data(), st.numActive, K[i]))
                                : 0u;
    }
    void readState()  // kdtree3d.cu:127-137
    {
        hostActive = st.numActive;
        hostNodes = size_t(st.numNodes);
        hostLeaves = size_t(st.numLeaves);
        view.syncSizes(hostLeaves, hostActive);
    }
    void binaryGrow()  // growBuffers, kdtree3d.cu:155-159
    {
        prepareGraphBuffers(leafCapacity + (leafCapacity + 3) / 4);
        st.needsResize = 0;
    }
    void binaryBuild()  // kdtree3d.cu:227-257
    {
        built = false;
        hostLeaves = 1;
        prepareGraphBuffers(std::max<size_t>(2, leafCapacity));
        computeKeys();
        K = {0, kMaxKey};
        st = State{};
        st.numNodes = 1;
        binaryRefresh();
        buildIterations = 0;
        for (;;)
        {
            binaryPass();
            ++buildIterations;
            readState();
            if (st.needsResize)
            {
                binaryGrow();
                binaryRefresh();
            }
            else if (st.converged)
            {
                break;
            }
        }
        built = true;
        if (preparedViews.any()) view.prepare(leafCapacity, n, preparedViews);
        buildViews(cfgViews);
        if (cfgViews.any()) needsResize();
    }
    void binaryUpdate()
    {
        if (!built) throw std::logic_error("adaptive_octree: call build() before update()");
        computeKeys();
        binaryRefresh();
        for (unsigned i = 0; i < iterations; ++i) binaryPass();
        buildViews(cfgViews);
    }

    // --- shared ---
    void buildViews(Views v)
    {
        preparedViews.ts |= v.ts;
        preparedViews.pc |= v.pc;
        preparedViews.pm |= v.pm;
        view.build(K, N, size_t(st.numLeaves), P, v, st);
    }
    bool needsResize()  // octree.cu:498-537; kdtree3d.cu:284-287
    {
        if (!built) return false;
        hostActive = st.numActive;
        hostLeaves = size_t(st.numLeaves);
        hostNodes = size_t(st.numNodes);
        if (kind == 0)
        {
            Kc.size = hostLeaves + 1;
            Tc.size = hostLeaves + 1;
        }
        view.syncSizes(hostLeaves, hostActive);
        return st.needsResize != 0;
    }
    void resizeBuffers()  // octree.cu:539-551; kdtree3d.cu:289-297
    {
        if (!built) throw std::logic_error("adaptive_octree: call build() before resizeBuffers()");
        needsResize();
        prepareGraphBuffers(leafCapacity + (leafCapacity + 3) / 4);
        st.needsResize = 0;
    }
    unsigned maxAchieved() const
    {
        if (kind == 1 && !cfgViews.any())
        {
            unsigned d = 0;
            for (size_t i = 0; i + 1 < hostLeaves + 1 && i + 1 < K.size(); ++i)
                d = std::max(d, unsigned(clz64(K[i + 1] - K[i])));
            return d;
        }
        return view.depthAlloc ? view.maxDepth : 0;
    }
};

}  // namespace aoo

// ---------------------------------------------------------------------------
// C API (same shape as the product's ao_tree_* entry points, host pointers)
// ---------------------------------------------------------------------------
extern "C" {

struct aoo_config
{
    int max_depth;
    unsigned max_particles_per_leaf;
    int update_iterations;
    double box[6];
    int split_criterion;
    int sfc_kind;
    int views_tree_structure, views_particle_counts, views_particle_mapping;
};

static thread_local std::string g_err;

static int fail(int code, const char *msg)
{
    g_err = msg;
    return code;
}

#define AOO_TRY(...)                                        \
    try                                                     \
    {                                                       \
        __VA_ARGS__;                                        \
        return 0;                                           \
    }                                                       \
    catch (const std::invalid_argument &e) { return fail(1, e.what()); } \
    catch (const std::logic_error &e) { return fail(2, e.what()); }      \
    catch (const std::exception &e) { return fail(6, e.what()); }

const char *aoo_last_error(void) { return g_err.c_str(); }

int aoo_tree_create(int kind, int real_type, const void *x, const void *y, const void *z, size_t n,
                    const aoo_config *c, void **out)
{
    AOO_TRY({
        if (!out || !c) throw std::invalid_argument("null argument");
        // Tree::backendConfig, tree.hpp:108-133
        if (c->max_depth < -1 || c->update_iterations < -1)
            throw std::invalid_argument("Tree: use -1 for backend defaults");
        if (kind == 1 && c->split_criterion != 0)
            throw std::invalid_argument("Tree: Binary NFCount is not implemented yet");
        if (kind == 1 && c->sfc_kind != 0)
            throw std::invalid_argument("Tree: Binary uses longest-side keys, not Hilbert");
        // Backend constructors, octree.cu:321-416 and kdtree3d.cu:175-216
        if (n > 0 && (!x || !y || !z))
            throw std::invalid_argument("adaptive_octree: coordinate device pointers must not be null");
        if (c->max_particles_per_leaf == 0)
            throw std::invalid_argument("adaptive_octree: particle limit must be positive");
        const unsigned iters = c->update_iterations >= 0 ? unsigned(c->update_iterations) : (kind == 0 ? 2u : 6u);
        if (iters == 0) throw std::invalid_argument("adaptive_octree: updateIterations must be positive");
        const unsigned depth = c->max_depth >= 0 ? unsigned(c->max_depth) : (kind == 0 ? 21u : 63u);
        aoo::Geometry geom{};
        if (kind == 1) geom = aoo::makeGeometry(c->box, depth);
        if (n > size_t(std::numeric_limits<std::uint32_t>::max()))
            throw std::invalid_argument("adaptive_octree: particle count exceeds 32-bit permutation index range");
        auto *t = new aoo::Tree();
        t->kind = kind;
        t->real = real_type;
        t->n = n;
        t->x = x;
        t->y = y;
        t->z = z;
        t->bucket = c->max_particles_per_leaf;
        std::memcpy(t->box, c->box, sizeof(t->box));
        t->cfgViews = {c->views_tree_structure != 0, c->views_particle_counts != 0, c->views_particle_mapping != 0};
        t->preparedViews = t->cfgViews;
        t->maxDepth = depth;
        t->iterations = iters;
        t->geom = geom;
        if (kind == 0)
        {
            t->nf = c->split_criterion == 1;
            t->hil = c->sfc_kind == 1;
            t->view.b = 3;
            aoo::capResize(t->Kc, 2);
        }
        else
        {
            t->view.b = 1;
        }
        t->K = {0, aoo::kMaxKey};
        *out = t;
    })
}

int aoo_tree_destroy(void *h)
{
    delete static_cast<aoo::Tree *>(h);
    return 0;
}

int aoo_tree_set_coordinates(void *h, const void *x, const void *y, const void *z)
{
    auto *t = static_cast<aoo::Tree *>(h);
    t->x = x;
    t->y = y;
    t->z = z;
    return 0;
}

int aoo_tree_build(void *h)
{
    AOO_TRY({
        auto *t = static_cast<aoo::Tree *>(h);
        if (t->kind == 0) t->octreeBuild();
        else t->binaryBuild();
    })
}

int aoo_tree_update(void *h)
{
    AOO_TRY({
        auto *t = static_cast<aoo::Tree *>(h);
        if (t->kind == 0) t->octreeUpdate();
        else t->binaryUpdate();
    })
}

int aoo_tree_compute_views(void *h, const int *views3)
{
    AOO_TRY({
        auto *t = static_cast<aoo::Tree *>(h);
        if (!t->built) throw std::logic_error("adaptive_octree: call build() before computeViews()");
        aoo::Views v = t->cfgViews;
        if (views3) v = {views3[0] != 0, views3[1] != 0, views3[2] != 0};
        t->buildViews(v);
    })
}

int aoo_tree_needs_resize(void *h, int *out)
{
    AOO_TRY({
        auto *t = static_cast<aoo::Tree *>(h);
        *out = t->needsResize() ? 1 : 0;
    })
}

int aoo_tree_resize_buffers(void *h)
{
    AOO_TRY({ static_cast<aoo::Tree *>(h)->resizeBuffers(); })
}

// which: 0 P, 1 Perm, 2 K, 3 N, 4 NF, 5 sfcBoxIndex, 6 hasBoxSplit, 7 boxDepth,
// 8 parentIndex, 9 childIndex, 10 levelOffset, 11 particleBeginIndex,
// 12 particleCounts, 13 sfcParticleIndex.  Copies the logical contents.
int aoo_tree_copy_buffer(void *h, int which, void *dst, size_t dst_bytes, size_t *len)
{
    AOO_TRY({
        auto *t = static_cast<aoo::Tree *>(h);
        const void *src = nullptr;
        size_t count = 0, elem = 0;
        const size_t nodes = t->view.numNodesLogical;
        const bool v = t->view.scratch;
        switch (which)
        {
        case 0: src = t->P.data(); count = t->P.size(); elem = 8; break;
        case 1: src = t->Perm.data(); count = t->Perm.size(); elem = 4; break;
        case 2: src = t->K.data(); count = t->hostLeaves + 1; elem = 8; break;
        case 3: src = t->N.data(); count = t->hostLeaves; elem = 4; break;
        case 4:
            // NF_d is sized like N_d in both criteria (octree.cu:527-530); its
            // contents are only defined for NFCount (zeros here otherwise).
            if (t->kind == 1) throw std::logic_error("Tree: Binary NFCount is not implemented yet");
            if (!t->nf && t->NF.size() < t->hostLeaves) t->NF.assign(t->hostLeaves, 0u);
            src = t->NF.data(); count = t->hostLeaves; elem = 4; break;
        case 5: src = t->view.box.data(); count = v ? nodes : 0; elem = 8; break;
        case 6: src = t->view.split.data(); count = v ? nodes : 0; elem = 1; break;
        case 7: src = t->view.depth.data(); count = v ? nodes : 0; elem = 1; break;
        case 8: src = t->view.parent.data(); count = v ? nodes : 0; elem = 4; break;
        case 9: src = t->view.child.data(); count = v ? nodes : 0; elem = 4; break;
        case 10: src = t->view.levelOffset.data(); count = v ? t->view.levelOffset.size() : 0; elem = 4; break;
        case 11: src = t->view.pbegin.data(); count = (v && t->view.prepared.pc) ? nodes : 0; elem = 4; break;
        case 12: src = t->view.pcount.data(); count = (v && t->view.prepared.pc) ? nodes + 1 : 0; elem = 4; break;
        case 13: src = t->view.pmap.data(); count = (v && t->view.prepared.pm) ? t->view.mappingLogical : 0; elem = 8; break;
        default: throw std::invalid_argument("unknown buffer");
        }
        if (len) *len = count;
        if (dst)
        {
            if (dst_bytes < count * elem) throw std::invalid_argument("destination too small");
            if (count) std::memcpy(dst, src, count * elem);
        }
    })
}

// info: [0] numParticles [1] numActiveParticles [2] numNodes [3] maxAchievedDepth
// [4] numLeaves (device state) [5] leafCapacity [6] needsResize (device state)
// [7] build iterations [8] activeBuffer [9] numNodes (device state)
int aoo_tree_info(void *h, unsigned long long *out10)
{
    AOO_TRY({
        auto *t = static_cast<aoo::Tree *>(h);
        out10[0] = t->n;
        out10[1] = t->hostActive;
        out10[2] = t->kind == 0 ? t->hostNodes : t->hostNodes;
        out10[3] = t->maxAchieved();
        out10[4] = (unsigned long long)(long long)t->st.numLeaves;
        out10[5] = t->leafCapacity;
        out10[6] = t->st.needsResize;
        out10[7] = t->buildIterations;
        out10[8] = t->st.activeBuffer;
        out10[9] = (unsigned long long)(long long)t->st.numNodes;
    })
}

// Pure key functions for known-answer tests.
int aoo_octree_keys(int real_type, const void *x, const void *y, const void *z, size_t n, const double *box,
                    int hilbert, unsigned long long *keys)
{
    AOO_TRY({
        if (real_type == 0)
        {
            const auto q = aoo::makeQBox<float>(box);
            for (size_t i = 0; i < n; ++i)
                keys[i] = aoo::octreeKey<float>(static_cast<const float *>(x)[i], static_cast<const float *>(y)[i],
                                                static_cast<const float *>(z)[i], q, hilbert != 0);
        }
        else
        {
            const auto q = aoo::makeQBox<double>(box);
            for (size_t i = 0; i < n; ++i)
                keys[i] = aoo::octreeKey<double>(static_cast<const double *>(x)[i], static_cast<const double *>(y)[i],
                                                 static_cast<const double *>(z)[i], q, hilbert != 0);
        }
    })
}

int aoo_binary_keys(int real_type, const void *x, const void *y, const void *z, size_t n, const double *box,
                    unsigned max_depth, unsigned long long *keys)
{
    AOO_TRY({
        const auto g = aoo::makeGeometry(box, max_depth);
        for (size_t i = 0; i < n; ++i)
        {
            if (real_type == 0)
                keys[i] = aoo::binaryKey<float>(static_cast<const float *>(x)[i], static_cast<const float *>(y)[i],
                                                static_cast<const float *>(z)[i], box, g);
            else
                keys[i] = aoo::binaryKey<double>(static_cast<const double *>(x)[i], static_cast<const double *>(y)[i],
                                                 static_cast<const double *>(z)[i], box, g);
        }
    })
}

int aoo_sfc_encode(unsigned x, unsigned y, unsigned z, int hilbert, unsigned long long *key)
{
    *key = aoo::sfcEncode(x, y, z, hilbert != 0);
    return 0;
}

int aoo_sfc_decode(unsigned long long key, int hilbert, unsigned *xyz)
{
    const aoo::C3 c = aoo::sfcDecode(key, hilbert != 0);
    xyz[0] = c.x;
    xyz[1] = c.y;
    xyz[2] = c.z;
    return 0;
}

}  // extern "C"
