// Counting handlers: every pair adds one to the unsigned long long the
// Query's `arg` points to (the reference's
// include/rtspatial/default_handlers/counting_handlers.h, same names and
// signatures).  Compile a handler module with this header, or build with
// RTSPATIAL_COUNTING_HANDLERS, to count; RTSPATIAL_BUILTIN_HANDLER lets the
// library run its own warp-aggregated counter (one atomic per warp) instead
// of a call per pair, with the same result.
#ifndef RTSPATIAL_DEFAULT_HANDLERS_COUNTING_HANDLERS_H
#define RTSPATIAL_DEFAULT_HANDLERS_COUNTING_HANDLERS_H

#include <cstdint>

#define RTSPATIAL_BUILTIN_HANDLER 0 /* RTS_HANDLER_COUNT */

extern "C" __forceinline__ __device__ void rtspatial_handle_point_contains(uint32_t geom_id,
                                                                           uint32_t query_id,
                                                                           void* arg) {
  atomicAdd(static_cast<unsigned long long*>(arg), 1ull);
}

extern "C" __forceinline__ __device__ void rtspatial_handle_envelope_contains(uint32_t geom_id,
                                                                              uint32_t query_id,
                                                                              void* arg) {
  atomicAdd(static_cast<unsigned long long*>(arg), 1ull);
}

extern "C" __forceinline__ __device__ void rtspatial_handle_envelope_intersects(uint32_t geom_id,
                                                                                uint32_t query_id,
                                                                                void* arg) {
  atomicAdd(static_cast<unsigned long long*>(arg), 1ull);
}

extern "C" __forceinline__ __device__ void rtspatial_handle_line_intersects(uint32_t geom_id,
                                                                             uint32_t query_id,
                                                                             void* arg) {
  atomicAdd(static_cast<unsigned long long*>(arg), 1ull);
}

#endif
