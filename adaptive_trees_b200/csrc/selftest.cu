// selftest.cu -- checks that the engine's bounded device waits end.
//
// Every decoupled look-back of the engine (the radix sort's per-digit
// prefixes, the rebalance decide+scan) polls earlier tiles for a bounded
// number of rounds; when that runs out the kernel records kErrLookback in its
// error word and finishes, so the host sees an error status instead of a hung
// GPU.  These probes build the one situation in which the limit is reached --
// tile 0 is never processed, so nothing ever publishes its status word -- and
// let the waits of the later tiles run out under a small limit:
//   which 0: one onesweep pass (8-bit digits, 10 keys per thread) over 4
//            tiles of zero keys, launched with 3 CTAs and the tile counter
//            starting at 1, so the CTAs take tiles 1..3;
//   which 1: the decide+scan look-back of tiles 1..3 over a zeroed status
//            array.
// Every index stays inside its buffer (a tile that gave up writes its keys at
// the prefix it has, below the prefix of the full input), and every wait is
// bounded by `spinLimit`, so the probes neither fault nor hang.
#include <stdexcept>
#include <string>

#include "engine_util.cuh"
#include "radix_sort.cuh"
#include "rebalance.cuh"

namespace aot
{
namespace
{
constexpr int kProbeItems = 10;
constexpr int kProbeTile = sort::kThreads * kProbeItems;
constexpr int kProbeTiles = 4;

__global__ void __launch_bounds__(sort::kThreads, 1)
    sortWaitProbeKernel(const u64 *keysIn, u64 *keysOut, u32 *valsOut, size_t n, const u32 *bins, u32 *tileCounter,
                        u64 *status, int *error, unsigned spinLimit)
{
    sort::onesweepTile<8, kProbeItems>(sort::ContiguousTiles<kProbeTile>{n, bins}, keysIn, nullptr, keysOut,
                                       valsOut, 0, tileCounter, status, error, 8, spinLimit);
}

__global__ void scanWaitProbeKernel(u64 *status, int *error, unsigned spinLimit, i64 *prefix)
{
    if (threadIdx.x == 0) prefix[blockIdx.x] = rb::lookback(status, blockIdx.x + 1, 1, error, spinLimit);
}

// Device allocations of the probe, freed on every exit path.
struct ProbeMem
{
    void *p = nullptr;
    explicit ProbeMem(size_t bytes) { AOT_CHECK(cudaMalloc(&p, bytes)); }
    ~ProbeMem() { cudaFree(p); }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

struct ProbeStream
{
    cudaStream_t s = nullptr;
    ProbeStream() { AOT_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~ProbeStream() { cudaStreamDestroy(s); }
};
}  // namespace

int TreeEngine::boundedWaitProbe(int which, unsigned spinLimit)
{
    if (which != 0 && which != 1) throw std::invalid_argument("ao_selftest_bounded_wait: which must be 0 or 1");
    if (spinLimit == 0 || spinLimit > (1u << 16))
        throw std::invalid_argument("ao_selftest_bounded_wait: spin_limit must be in [1, 65536]");
    ProbeStream ps;
    const cudaStream_t s = ps.s;
    ProbeMem err(sizeof(int));
    AOT_CHECK(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    if (which == 0)
    {
        const size_t n = size_t(kProbeTiles) * kProbeTile;
        ProbeMem keysIn(n * sizeof(u64)), keysOut(n * sizeof(u64)), valsOut(n * sizeof(u32));
        ProbeMem bins(sort::kRadix * sizeof(u32)), counter(sizeof(u32));
        ProbeMem status(size_t(kProbeTiles) * sort::kRadix * sizeof(u64));
        AOT_CHECK(cudaMemsetAsync(keysIn.p, 0, n * sizeof(u64), s));
        AOT_CHECK(cudaMemsetAsync(bins.p, 0, sort::kRadix * sizeof(u32), s));  // every key has digit 0
        AOT_CHECK(cudaMemsetAsync(status.p, 0, size_t(kProbeTiles) * sort::kRadix * sizeof(u64), s));
        const u32 firstTile = 1;  // tile 0 is never taken, so it never publishes
        AOT_CHECK(cudaMemcpyAsync(counter.p, &firstTile, sizeof(u32), cudaMemcpyHostToDevice, s));
        const int smem = int(sizeof(sort::SharedPass<8, kProbeItems>));
        AOT_CHECK(cudaFuncSetAttribute(sortWaitProbeKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        sortWaitProbeKernel<<<kProbeTiles - 1, sort::kThreads, smem, s>>>(
            keysIn.as<u64>(), keysOut.as<u64>(), valsOut.as<u32>(), n, bins.as<u32>(), counter.as<u32>(),
            status.as<u64>(), err.as<int>(), spinLimit);
        AOT_LAUNCH_CHECK();
        AOT_CHECK(cudaStreamSynchronize(s));
    }
    else
    {
        ProbeMem status(size_t(kProbeTiles) * sizeof(u64)), prefix(size_t(kProbeTiles) * sizeof(i64));
        AOT_CHECK(cudaMemsetAsync(status.p, 0, size_t(kProbeTiles) * sizeof(u64), s));
        scanWaitProbeKernel<<<kProbeTiles - 1, 32, 0, s>>>(status.as<u64>(), err.as<int>(), spinLimit,
                                                           prefix.as<i64>());
        AOT_LAUNCH_CHECK();
        AOT_CHECK(cudaStreamSynchronize(s));
    }
    int error = 0;
    AOT_CHECK(cudaMemcpy(&error, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    return error;
}
}  // namespace aot
