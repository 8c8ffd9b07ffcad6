// Allocation-free pair sort: ao_sort_pairs with its scratch in a fixed device
// array of this file instead of caller-provided memory.
//
// Who needs it: callers that cannot allocate device memory where they sort --
// a serving process that reserves its whole device budget at start-up and
// must not grow it afterwards, or a plain C / FFI host that has no device
// allocator of its own to hand a scratch buffer to ao_sort_pairs.
//
// Limits and rules:
//  * at most kNoAllocMaxItems (1,048,576) items per call; larger n is rejected
//    with std::invalid_argument before any CUDA call;
//  * the array is one per device: calls that overlap in time on the same
//    device (from other streams or threads) share it and race, corrupting
//    each other's results.  Serialise them (one stream, or host-side order);
//  * the first call on a device does the set-up: it loads every kernel the
//    sort can launch on that device (so that no later call loads code).
//    Every call looks up the array's address on the current device, which is
//    cheap once the module is loaded and stays right if the device's context
//    is torn down and created again.  Make the first call before any stream
//    capture;
//  * what must start at zero -- the sort's digit counters, pass counters,
//    error word and decoupled look-back status words -- is cleared by the sort
//    itself on the caller's stream (cudaMemsetAsync) before its kernels run,
//    so whatever an earlier call left in the array is harmless.  The
//    key/value ping-pong halves need no clearing;
//  * the look-back waits of the sort are bounded; sortPairsNoAllocFailed
//    (ao_sort_pairs_noalloc_check) reads whether one gave up in the last call
//    of n items, which means its output is not sorted.
// Nothing here calls cudaMalloc/cudaFree or a routine that allocates.
#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>

#include "engine.hpp"

namespace aot
{
namespace
{
// Scratch layout of the pair sort for kNoAllocMaxItems items: alternate keys
// (8 B/item), alternate values (4 B/item), counters (error word and 3 pad
// words, 2 x 8 passes x 256 digits, 8 tile counters), look-back status
// (8 passes x tiles of kSortTileItems items x 256 digits x 8 B), each part
// rounded up to 256 bytes.  The call checks the sort's own size query against
// this before using the array.
constexpr size_t kNoAllocMaxItems = size_t(1) << 20;
constexpr size_t up256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kNoAllocTiles = (kNoAllocMaxItems + kSortTileItems - 1) / kSortTileItems;
constexpr size_t kNoAllocScratchBytes =
    up256(up256(up256(up256(kNoAllocMaxItems * 8) + kNoAllocMaxItems * 4) + (4 + 2 * 8 * 256 + 8) * 4) +
          size_t(8) * kNoAllocTiles * 256 * 8);  // 19,316,992 bytes

static __device__ __align__(256) unsigned char g_noAllocScratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
bool g_preloaded[kMaxDevices] = {};

// Address of g_noAllocScratch on the current device, looked up with that
// device current; the first call on a device also loads the sort's kernels.
void *noAllocScratch()
{
    int dev = 0;
    AOT_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        throw std::runtime_error("ao_sort_pairs_noalloc: device ordinal " + std::to_string(dev) +
                                 " is beyond the supported " + std::to_string(kMaxDevices));
    {
        std::lock_guard<std::mutex> lock(g_setupMutex);
        if (!g_preloaded[dev])
        {
            TreeEngine::sortPairsPreload();
            g_preloaded[dev] = true;
        }
    }
    void *p = nullptr;
    AOT_CHECK(cudaGetSymbolAddress(&p, g_noAllocScratch));
    return p;
}
}  // namespace

size_t sortPairsNoAllocMaxItems() { return kNoAllocMaxItems; }

void sortPairsNoAlloc(const unsigned long long *keysIn, unsigned long long *keysOut, const unsigned *valsIn,
                      unsigned *valsOut, size_t n, int beginBit, int endBit, cudaStream_t s)
{
    if (n > kNoAllocMaxItems)
        throw std::invalid_argument("ao_sort_pairs_noalloc: n = " + std::to_string(n) +
                                    " exceeds the fixed scratch limit of " + std::to_string(kNoAllocMaxItems) +
                                    " items; use ao_sort_pairs with caller scratch");
    // always the default sort configuration, whose scratch the array is sized for
    size_t need = 0;
    TreeEngine::sortPairsWith(0, nullptr, &need, keysIn, keysOut, valsIn, valsOut, n, beginBit, endBit, s);
    if (need > kNoAllocScratchBytes)
        throw std::logic_error("ao_sort_pairs_noalloc: the sort needs " + std::to_string(need) +
                               " scratch bytes, more than the fixed " + std::to_string(kNoAllocScratchBytes));
    size_t have = kNoAllocScratchBytes;
    TreeEngine::sortPairsWith(0, noAllocScratch(), &have, keysIn, keysOut, valsIn, valsOut, n, beginBit, endBit, s);
}

bool sortPairsNoAllocFailed(size_t n, cudaStream_t s)
{
    if (n > kNoAllocMaxItems)
        throw std::invalid_argument("ao_sort_pairs_noalloc_check: n = " + std::to_string(n) +
                                    " exceeds the fixed scratch limit of " + std::to_string(kNoAllocMaxItems));
    if (n == 0) return false;  // an empty sort launches nothing
    return TreeEngine::sortPairsFailed(noAllocScratch(), n, s);
}
}  // namespace aot
