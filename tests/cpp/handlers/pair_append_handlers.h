// A handler header as a user of the reference writes one: every predicate's
// handler appends (geom_id, query_id) to a queue with one atomic per pair and
// counts its own calls, so a test can see that each predicate reaches its own
// handler.  It sets no RTSPATIAL_BUILTIN_HANDLER, so a module built from it
// calls these functions per pair.  <optix.h> is included the way the
// reference's handler headers include it (nothing from it is used).
#include <optix.h>

#include <cstdint>

struct PairSink {
  uint32_t* pairs;               // (geom_id, query_id) words
  unsigned long long capacity;   // pairs
  unsigned long long* size;      // pairs appended (may exceed capacity)
  unsigned long long* calls;     // calls per handler: point, contains, intersects, line
};

__device__ __forceinline__ void pair_sink_append(void* arg, int which, uint32_t g, uint32_t q) {
  PairSink* s = static_cast<PairSink*>(arg);
  atomicAdd(s->calls + which, 1ull);
  const unsigned long long at = atomicAdd(s->size, 1ull);
  if (at < s->capacity) {
    s->pairs[2 * at] = g;
    s->pairs[2 * at + 1] = q;
  }
}

extern "C" __device__ void rtspatial_handle_point_contains(uint32_t geom_id, uint32_t query_id,
                                                           void* arg) {
  pair_sink_append(arg, 0, geom_id, query_id);
}

extern "C" __device__ void rtspatial_handle_envelope_contains(uint32_t geom_id,
                                                              uint32_t query_id, void* arg) {
  pair_sink_append(arg, 1, geom_id, query_id);
}

extern "C" __device__ void rtspatial_handle_envelope_intersects(uint32_t geom_id,
                                                                uint32_t query_id, void* arg) {
  pair_sink_append(arg, 2, geom_id, query_id);
}

extern "C" __device__ void rtspatial_handle_line_intersects(uint32_t geom_id, uint32_t query_id,
                                                            void* arg) {
  pair_sink_append(arg, 3, geom_id, query_id);
}
