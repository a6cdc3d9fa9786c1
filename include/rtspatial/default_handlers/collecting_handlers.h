// Collecting handlers: every pair is appended as (geom_id, query_id) to the
// rtspatial::dev::Queue<thrust::pair<uint32_t, uint32_t>> the Query's `arg`
// points to, in device memory (the reference's
// include/rtspatial/default_handlers/collecting_handlers.h, same names and
// signatures).  The queue never stores past its capacity; its size keeps
// counting, so size() > capacity() afterwards reports the capacity needed.
// RTSPATIAL_BUILTIN_HANDLER lets the library run its own warp-buffered
// collector (one atomic per flush) instead of a call per pair, with the same
// pairs.
#ifndef RTSPATIAL_DEFAULT_HANDLERS_COLLECTING_HANDLERS_H
#define RTSPATIAL_DEFAULT_HANDLERS_COLLECTING_HANDLERS_H

#include <thrust/pair.h>

#include <cstdint>

#include "rtspatial/utils/queue.h"

#define RTSPATIAL_BUILTIN_HANDLER 1 /* RTS_HANDLER_COLLECT */

extern "C" __forceinline__ __device__ void rtspatial_handle_point_contains(uint32_t geom_id,
                                                                           uint32_t query_id,
                                                                           void* arg) {
  auto* queue = static_cast<rtspatial::dev::Queue<thrust::pair<uint32_t, uint32_t>>*>(arg);
  queue->Append(thrust::make_pair(geom_id, query_id));
}

extern "C" __forceinline__ __device__ void rtspatial_handle_envelope_contains(uint32_t geom_id,
                                                                              uint32_t query_id,
                                                                              void* arg) {
  auto* queue = static_cast<rtspatial::dev::Queue<thrust::pair<uint32_t, uint32_t>>*>(arg);
  queue->Append(thrust::make_pair(geom_id, query_id));
}

extern "C" __forceinline__ __device__ void rtspatial_handle_envelope_intersects(uint32_t geom_id,
                                                                                uint32_t query_id,
                                                                                void* arg) {
  auto* queue = static_cast<rtspatial::dev::Queue<thrust::pair<uint32_t, uint32_t>>*>(arg);
  queue->Append(thrust::make_pair(geom_id, query_id));
}

extern "C" __forceinline__ __device__ void rtspatial_handle_line_intersects(uint32_t geom_id,
                                                                             uint32_t query_id,
                                                                             void* arg) {}

#endif
