// ref_compat.h -- forced-include shim for compiling the reference's own
// sources with this image's CCCL (2.8).  The reference was written for CCCL
// 3.x, whose thrust::device_vector::resize(n, thrust::no_init) leaves new
// elements uninitialised; CCCL 2.8 has no such overload, so thrust::no_init is
// declared here as a value that converts to T{} and resize(n, no_init)
// value-initialises the new elements.  No reference source file is changed.
// TEST INFRASTRUCTURE ONLY (oracle/_ref).
#pragma once
#include <thrust/version.h>
namespace thrust
{
struct no_init_t
{
    template <class T>
    operator T() const
    {
        return T{};
    }
};
inline constexpr no_init_t no_init{};
}  // namespace thrust
