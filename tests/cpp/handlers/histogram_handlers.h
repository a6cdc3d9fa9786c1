// A custom handler that is neither counting nor collecting: per query, the
// number of matching boxes and the sum of their geom ids (arg = Histogram* in
// device memory), for the C++ drop-in test of user handlers.
#include <cstdint>

struct Histogram {
  unsigned int* count;        // per query
  unsigned long long* idsum;  // per query
};

__device__ __forceinline__ void histogram_add(void* arg, uint32_t geom_id, uint32_t query_id) {
  Histogram* h = static_cast<Histogram*>(arg);
  atomicAdd(h->count + query_id, 1u);
  atomicAdd(h->idsum + query_id, static_cast<unsigned long long>(geom_id));
}

extern "C" __device__ void rtspatial_handle_point_contains(uint32_t geom_id, uint32_t query_id,
                                                           void* arg) {
  histogram_add(arg, geom_id, query_id);
}

extern "C" __device__ void rtspatial_handle_envelope_contains(uint32_t geom_id,
                                                              uint32_t query_id, void* arg) {
  histogram_add(arg, geom_id, query_id);
}

extern "C" __device__ void rtspatial_handle_envelope_intersects(uint32_t geom_id,
                                                                uint32_t query_id, void* arg) {
  histogram_add(arg, geom_id, query_id);
}

extern "C" __device__ void rtspatial_handle_line_intersects(uint32_t, uint32_t, void*) {}
