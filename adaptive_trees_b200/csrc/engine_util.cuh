// engine_util.cuh -- host helpers shared by the engines (definitions in engine.cu).
#pragma once

#include <algorithm>
#include <cmath>

#include "engine.hpp"
#include "sfc.cuh"

namespace aot
{
// Counts one kernel launch of the engine (reported as kernel_launches).
void noteLaunch();
// SM count of the current device.
int smCount();
// Blocks of `threads` threads covering n items (at least 1).
unsigned gridFor(size_t n, unsigned threads);
// Hilbert encode/decode tables (generated once).
const HilbertTables &hilbertTables();

// Box<T> (sfc_keys.cuh:420-465): inverse lengths and per-axis bits in T.
template <class T>
QuantBox<T> makeQuantBox(const double *b)
{
    const T xmin = T(b[0]), xmax = T(b[1]), ymin = T(b[2]), ymax = T(b[3]), zmin = T(b[4]), zmax = T(b[5]);
    QuantBox<T> q;
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
}  // namespace aot
