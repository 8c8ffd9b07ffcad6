// sfc.cuh -- space-filling-curve keys on the device.
//
// Morton: bit spreading by shifts and masks.  Hilbert: the 3-D curve of the
// reference (iHilbert, sfc_keys.cuh:248-290) expressed as a 48-state machine.
// Each level of the reference transforms the remaining coordinate words by
// whole-word complements and a permutation of the three axes, so the word
// seen at the next level is always one original axis, possibly complemented:
// a state is (axis permutation, complement bits), 6 x 8 = 48 states.  The
// tables below map (state, original octant) to the emitted octal digit and
// the next state; they are generated once on the host by applying the
// reference's per-level rules to every state.  Encoding a level is then one
// table lookup instead of the reference's branchy word updates.
#pragma once

#include "common.cuh"

namespace aot
{
// --------------------------------------------------------------------------
// Morton (iMorton / decodeMorton, sfc_keys.cuh:174-237)
// --------------------------------------------------------------------------
__host__ __device__ __forceinline__ u64 spread3(u64 v)
{
    u64 x = v & 0x1fffffull;
    x = (x | x << 32) & 0x001f00000000ffffull;
    x = (x | x << 16) & 0x001f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
__host__ __device__ __forceinline__ u32 compact3(u64 v)
{
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
    v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
    v = (v ^ (v >> 8)) & 0x001f0000ff0000ffull;
    v = (v ^ (v >> 16)) & 0x001f00000000ffffull;
    v = (v ^ (v >> 32)) & 0x00000000001fffffull;
    return u32(v);
}
__host__ __device__ __forceinline__ u64 mortonKey(u32 x, u32 y, u32 z)
{
    return (spread3(x) << 2) | (spread3(y) << 1) | spread3(z);
}

// --------------------------------------------------------------------------
// Hilbert state machine
// --------------------------------------------------------------------------
// Index = state * 8 + original octant (octant = x<<2 | y<<1 | z of the
// original coordinates' bits at the level).
struct HilbertTables
{
    unsigned char enc[48 * 8];      // emitted octal digit
    unsigned char encNext[48 * 8];  // next state
    unsigned char decOct[48 * 8];   // (state, digit) -> original octant
};

// Builds the tables from the reference's per-level rules (host only).
inline HilbertTables makeHilbertTables()
{
    HilbertTables t{};
    static const unsigned order[8] = {0, 1, 3, 2, 7, 6, 4, 5};  // sfc_keys.cuh:248-252
    static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    auto stateOf = [&](const int p[3], const int f[3]) {
        int pi = 0;
        for (int k = 0; k < 6; ++k)
            if (perms[k][0] == p[0] && perms[k][1] == p[1] && perms[k][2] == p[2]) pi = k;
        return pi * 8 + (f[0] << 2) + (f[1] << 1) + f[2];
    };
    for (int s = 0; s < 48; ++s)
    {
        const int *perm = perms[s / 8];
        const int flips[3] = {(s >> 2) & 1, (s >> 1) & 1, s & 1};
        for (unsigned o = 0; o < 8; ++o)
        {
            const unsigned ob[3] = {(o >> 2) & 1u, (o >> 1) & 1u, o & 1u};
            // bits the reference reads from its current words px, py, pz
            const unsigned xi = ob[perm[0]] ^ unsigned(flips[0]);
            const unsigned yi = ob[perm[1]] ^ unsigned(flips[1]);
            const unsigned zi = ob[perm[2]] ^ unsigned(flips[2]);
            const unsigned digit = order[(xi << 2) | (yi << 1) | zi];
            // word updates of one level (sfc_keys.cuh:270-286) on symbolic words
            int wp[3] = {perm[0], perm[1], perm[2]};
            int wf[3] = {flips[0], flips[1], flips[2]};
            const unsigned ny = !yi, nz = !zi;
            if (xi & (ny | zi)) wf[0] ^= 1;
            if ((xi & (yi | zi)) | (yi & nz)) wf[1] ^= 1;
            if ((xi & ny & nz) | (yi & nz)) wf[2] ^= 1;
            if (zi)
            {
                const int tp = wp[0], tf = wf[0];
                wp[0] = wp[1]; wf[0] = wf[1];
                wp[1] = wp[2]; wf[1] = wf[2];
                wp[2] = tp; wf[2] = tf;
            }
            else if (ny)
            {
                std::swap(wp[0], wp[2]);
                std::swap(wf[0], wf[2]);
            }
            const int next = stateOf(wp, wf);
            t.enc[s * 8 + o] = (unsigned char)digit;
            t.encNext[s * 8 + o] = (unsigned char)next;
            t.decOct[s * 8 + digit] = (unsigned char)o;
        }
    }
    return t;
}

// The identity state (permutation 0, no complements).
constexpr int kHilbertStart = 0;

// Encode the top `levels` levels of (x, y, z) (21-bit words) as a Hilbert
// key prefix, returned left-aligned in the 63-bit key (low bits zero).
// Tables are in shared memory (sEnc, sNext: 384 bytes each).
__host__ __device__ __forceinline__ u64 hilbertPrefix(u32 x, u32 y, u32 z, unsigned levels, const unsigned char *sEnc,
                                             const unsigned char *sNext)
{
    u64 key = 0;
    int s = kHilbertStart;
    for (unsigned i = 0; i < levels; ++i)
    {
        const unsigned b = kOctLevels - 1 - i;
        const unsigned o = (((x >> b) & 1u) << 2) | (((y >> b) & 1u) << 1) | ((z >> b) & 1u);
        const int idx = s * 8 + int(o);
        key = (key << 3) | sEnc[idx];
        s = sNext[idx];
    }
    return key << (3u * (kOctLevels - levels));
}

// Two levels per lookup: pair[state * 64 + (o1 << 3 | o2)] = the two emitted
// digits (d1 << 3 | d2) | the state after both << 6, for the original octants
// o1, o2 of two consecutive levels.  3072 entries built from enc / encNext.
constexpr int kHilbertPairEntries = 48 * 64;
__host__ __device__ __forceinline__ unsigned short hilbertPairEntry(int i, const unsigned char *enc,
                                                                   const unsigned char *encNext)
{
    const int s = i >> 6, o1 = (i >> 3) & 7, o2 = i & 7;
    const int a = s * 8 + o1;
    const int b = int(encNext[a]) * 8 + o2;
    return (unsigned short)((enc[a] << 3) | enc[b] | (encNext[b] << 6));
}

// The full 21-level Hilbert key of (x, y, z) with the pair table: the Morton
// interleave of the words puts each level's original octant (x << 2 | y << 1
// | z) in consecutive bits, so two levels are one 6-bit field.  Equal to
// hilbertPrefix(x, y, z, kOctLevels, ...).
__host__ __device__ __forceinline__ u64 hilbertKeyPairs(u32 x, u32 y, u32 z, const unsigned short *sPair)
{
    const u64 m = mortonKey(x, y, z);
    u64 key = 0;
    unsigned s = kHilbertStart;
#pragma unroll
    for (int i = 0; i < int(kOctLevels) / 2; ++i)  // levels 2i and 2i + 1 from the top
    {
        const unsigned v = sPair[s * 64 + (unsigned(m >> (3 * (kOctLevels - 2 - 2 * i))) & 63u)];
        key = (key << 6) | (v & 63u);
        s = v >> 6;
    }
    // the last level alone: the first digit of the entry with o2 = 0
    const unsigned v = sPair[s * 64 + ((unsigned(m) & 7u) << 3)];
    return (key << 3) | ((v >> 3) & 7u);
}

// Decode the top `levels` levels of a Hilbert key to the cell's corner in
// 21-bit integer coordinates (bits below the level are zero).
__host__ __device__ __forceinline__ void hilbertCorner(u64 key, unsigned levels, const unsigned char *sDec,
                                              const unsigned char *sNext, u32 &x, u32 &y, u32 &z)
{
    int s = kHilbertStart;
    x = y = z = 0;
    for (unsigned i = 0; i < levels; ++i)
    {
        const unsigned b = kOctLevels - 1 - i;
        const unsigned d = unsigned(key >> (3u * b)) & 7u;
        const unsigned o = sDec[s * 8 + int(d)];
        x |= ((o >> 2) & 1u) << b;
        y |= ((o >> 1) & 1u) << b;
        z |= (o & 1u) << b;
        s = sNext[s * 8 + int(o)];
    }
}

// --------------------------------------------------------------------------
// Float -> grid quantisation (sfc3D, sfc_keys.cuh:467-496)
// --------------------------------------------------------------------------
template <class T>
struct QuantBox
{
    T xmin, ymin, zmin, ilx, ily, ilz;
    unsigned bx, by, bz;  // bits per axis (21 minus the axis' shortening)
};

// floor(v*m) - vmin*m with the subtraction fused (as nvcc contracts it in the
// reference kernel), truncated with saturation and clamped to the top cell.
__device__ __forceinline__ u32 quantise(float v, float vmin, float il, unsigned bits)
{
    const float m = __fmul_rn(float(1u << bits), il);
    const float f = floorf(__fmul_rn(v, m));
    const float q = __fmaf_rn(-vmin, m, f);
    int i = __float2int_rz(q);
    const int top = int(1u << bits) - 1;
    i = i < top ? i : top;
    return u32(i) & 0x1fffffu;
}
__device__ __forceinline__ u32 quantise(double v, double vmin, double il, unsigned bits)
{
    const double m = __dmul_rn(double(1u << bits), il);
    const double f = floor(__dmul_rn(v, m));
    const double q = __fma_rn(-vmin, m, f);
    int i = __double2int_rz(q);
    const int top = int(1u << bits) - 1;
    i = i < top ? i : top;
    return u32(i) & 0x1fffffu;
}

template <class T>
__device__ __forceinline__ bool isEscaped(T x, T y, T z);
template <>
__device__ __forceinline__ bool isEscaped<float>(float x, float y, float z)
{
    const float e = 3.402823466e+38f;
    return x == e && y == e && z == e;
}
template <>
__device__ __forceinline__ bool isEscaped<double>(double x, double y, double z)
{
    const double e = 1.7976931348623157e+308;
    return x == e && y == e && z == e;
}

// --------------------------------------------------------------------------
// Binary longest-side keys (binaryEncode, binary_node.cuh:43-59)
// --------------------------------------------------------------------------
struct BinaryGeometry
{
    unsigned char axis[kBinDepth];
    int mortonOrder;  // 1 if axis[d] == d % 3 for every depth (cubic boxes)
    double xmin, xmax, ymin, ymax, zmin, zmax;  // box in double, converted from Real
};

// 63-bit fixed point of a normalised coordinate: clamp to [0, 1] keeping the
// reference's comparison order (NaN passes through), scale by 2^63, truncate
// with saturation, and keep it below 2^63.
__device__ __forceinline__ u64 fixed63(double v)
{
    const double c1 = (1.0 < v) ? 1.0 : v;
    const double c0 = (0.0 > c1) ? 0.0 : c1;
    const u64 k = __double2ull_rz(__dmul_rn(c0, 9223372036854775808.0));
    return k < kMaxKey - 1 ? k : kMaxKey - 1;
}

template <class T>
__device__ __forceinline__ u64 binaryKey(T x, T y, T z, const BinaryGeometry &g)
{
    if (isEscaped<T>(x, y, z)) return kInvalidKey;
    const double vx = __ddiv_rn(__dsub_rn(double(x), g.xmin), __dsub_rn(g.xmax, g.xmin));
    const double vy = __ddiv_rn(__dsub_rn(double(y), g.ymin), __dsub_rn(g.ymax, g.ymin));
    const double vz = __ddiv_rn(__dsub_rn(double(z), g.zmin), __dsub_rn(g.zmax, g.zmin));
    u64 c[3] = {fixed63(vx), fixed63(vy), fixed63(vz)};
    if (g.mortonOrder)
    {
        // x,y,z round robin: each axis supplies its top 21 fixed-point bits
        return mortonKey(u32(c[0] >> 42), u32(c[1] >> 42), u32(c[2] >> 42));
    }
    u64 key = 0;
#pragma unroll 9
    for (unsigned d = 0; d < kBinDepth; ++d)
    {
        const unsigned a = g.axis[d];
        const u64 v = a == 0 ? c[0] : (a == 1 ? c[1] : c[2]);
        key = (key << 1) | ((v >> (kBinDepth - 1)) & 1u);
        if (a == 0) c[0] <<= 1;
        else if (a == 1) c[1] <<= 1;
        else c[2] <<= 1;
    }
    return key;
}

}  // namespace aot
