// Source of a handler module: the query kernels with the caller's per-pair
// device handlers, the counterpart of the reference's query shaders
// (src/shaders/*.cu) compiled with a handler header.
//
// Compile it with the handler header force-included, the way the reference's
// RTSPATIAL_COMPILE_SHADERS does (CMakeLists.txt:73-104):
//
//   nvcc -cubin -gencode arch=compute_100a,code=sm_100a -std=c++17 -O3
//        -fmad=false --expt-relaxed-constexpr
//        -I <this library>/include -I <this library>/rtspatial_b200/csrc
//        -I <handler dir> -include <handler header>
//        rts_handler_module.cu -o rtspatial_handlers.cubin
//
// (cmake/rtspatial_shaders.cmake and rtspatial_b200.handlers do exactly this.)
// The header defines, as the reference's default handlers do,
//
//   extern "C" __device__ void rtspatial_handle_point_contains(uint32_t geom_id,
//                                                              uint32_t query_id, void* arg);
//   extern "C" __device__ void rtspatial_handle_envelope_contains(...);
//   extern "C" __device__ void rtspatial_handle_envelope_intersects(...);
//   extern "C" __device__ void rtspatial_handle_line_intersects(...);
//
// and each is called once per (geom_id, query_id) pair of its predicate, with
// the `arg` the Query call received.  The line handler is never called: line
// queries report nothing, as in the reference.  A header that sets
// RTSPATIAL_BUILTIN_HANDLER (the shipped counting and collecting headers do)
// tells the library that its own warp-aggregated handler of the same
// behaviour may run instead of the per-pair calls.
//
// -fmad=false: the range-intersects predicate depends on separately rounded
// products, as in the library itself.
#include <cstdint>

#include "rts_handler_kernel.cuh"

#ifndef RTSPATIAL_BUILTIN_HANDLER
#define RTSPATIAL_BUILTIN_HANDLER -1
#endif

namespace {

struct UserHandlers {
  template <int PRED>
  static __device__ __forceinline__ void call(uint32_t geom_id, uint32_t query_id, void* arg) {
    if constexpr (PRED == rts::kPoint || PRED == rts::kPoint64) {
      rtspatial_handle_point_contains(geom_id, query_id, arg);
    } else if constexpr (PRED == rts::kContains || PRED == rts::kContains64) {
      rtspatial_handle_envelope_contains(geom_id, query_id, arg);
    } else {
      rtspatial_handle_envelope_intersects(geom_id, query_id, arg);
    }
  }
};

}  // namespace

#define RTS_HANDLER_KERNEL(W, MINB)                                                             \
  extern "C" __global__ void __launch_bounds__(rts::kHandlerModuleThreads, MINB)               \
      rts_handler_query_v1_w##W(                                                                \
          const __grid_constant__ rts::Forest F, const __grid_constant__ rts::BatchDesc b0,     \
          const rts::BatchDesc* __restrict__ descs, uint32_t nb, uint32_t total_chunks,         \
          uint32_t chunk, uint32_t* __restrict__ work, const uint32_t* __restrict__ only,       \
          const uint32_t* __restrict__ only_any, const __grid_constant__ rts::MergedOrder M,    \
          const uint32_t* __restrict__ chunk_order) {                                          \
    (void)M;                                                                                    \
    rts::handler_query<UserHandlers, W>(F, b0, descs, nb, total_chunks, chunk, work, only,     \
                                        only_any, chunk_order);                                 \
  }

static_assert(rts::kHandlerModuleAbi == 1, "kernel names carry the module ABI version");
RTS_HANDLER_KERNEL(4, 2)
RTS_HANDLER_KERNEL(8, 2)
RTS_HANDLER_KERNEL(16, 2)
RTS_HANDLER_KERNEL(32, 1)

// Read by the library after loading the module.
extern "C" __device__ const int rts_module_abi_version = rts::kHandlerModuleAbi;
extern "C" __device__ const int rts_module_builtin_handler = RTSPATIAL_BUILTIN_HANDLER;
