// launch_util.cuh -- host-side helpers shared by the launchers.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace mayo {

__host__ __device__ constexpr size_t pad16(size_t x) { return (x + 15) / 16 * 16; }

// Opt `kernel` into `bytes` of dynamic shared memory on the current device.  The attribute is
// per kernel and per device; setting it is a cheap host call that is not a stream operation.
template <class K>
inline bool set_smem_attr(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return true;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess;
}

}  // namespace mayo
