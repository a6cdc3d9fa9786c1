// Drop-in utility macros and allocator aliases of the rtspatial C++ API
// (the reference's utils/util.h names: DEV_HOST, DEV_HOST_INLINE,
// DEV_INLINE, pinned_vector, device_uvector), backed by the CUDA toolkit's
// Thrust.  No OptiX.
#ifndef RTSPATIAL_B200_UTILS_UTIL_H
#define RTSPATIAL_B200_UTILS_UTIL_H

#include <cuda_runtime.h>
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>
#include <thrust/mr/allocator.h>
#include <thrust/system/cuda/memory_resource.h>

#define DEV_HOST __device__ __host__
#define DEV_HOST_INLINE __device__ __host__ __forceinline__
#define DEV_INLINE __device__ __forceinline__

namespace rtspatial {

// Host vector in page-locked memory the device can address directly.
template <typename T>
using pinned_vector = thrust::host_vector<
    T, thrust::mr::stateless_resource_allocator<
           T, thrust::system::cuda::universal_host_pinned_memory_resource>>;

template <typename T>
using device_uvector = thrust::device_vector<T>;

}  // namespace rtspatial
#endif
