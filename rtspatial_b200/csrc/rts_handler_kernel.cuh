// Query kernel of a handler module: the thread scheme with the caller's own
// per-pair device handlers.
//
// The reference compiles its query shaders with the user's handler header
// force-included (CMakeLists.txt:73-104, `-include ${CALLBACK_HEADER}` at
// :98) and calls rtspatial_handle_{point_contains, envelope_contains,
// envelope_intersects}(geom_id, query_id, arg) once per result
// (src/shaders/shaders_contains_point_query_2d.cu:14-25 and the other
// shaders).  A handler module does the same on this library's traversal: its
// source (shaders/rts_handler_module.cu) is compiled by the caller's build
// with the handler header included, into a cubin that the library loads
// (rts_load_handler_module) and launches in place of its own kernel for
// batches with handler RTS_HANDLER_MODULE.
//
// The kernel takes exactly the arguments of the library's query kernels (same
// persistent work queue, batches, visiting order), so the library's launch
// path drives it unchanged.  kHandlerModuleAbi names that contract: the
// module's kernels carry it in their names, and a library built against
// other descriptor layouts does not find them.
#pragma once

#include "rts_traverse.cuh"

namespace rts {

constexpr int kHandlerModuleAbi = 1;
constexpr int kHandlerModuleThreads = 256;

// H::call<PRED>(geom_id, query_id, arg): the module's adaptor to the
// rtspatial_handle_* functions.  One non-inlined function per predicate, so
// each is register-allocated for itself.
template <class H, int W, int PRED>
__device__ __noinline__ void handler_body(const Forest& F, const BatchDesc& B, uint32_t cb,
                                          uint32_t ce, const uint32_t* only) {
  const MergedOrder M{};
  run_chunk_thread<PRED, kUser, W, false, H>(F, B, cb, ce, nullptr, nullptr, only, M);
}

template <class H, int W>
__device__ __forceinline__ void handler_query(const Forest& F_in, const BatchDesc& b0,
                                              const BatchDesc* __restrict__ descs, uint32_t nb,
                                              uint32_t total_chunks, uint32_t chunk,
                                              uint32_t* __restrict__ work,
                                              const uint32_t* __restrict__ only,
                                              const uint32_t* __restrict__ only_any,
                                              const uint32_t* __restrict__ chunk_order) {
  if (only_any && *only_any == 0) return;
  __shared__ Forest F;
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&F_in);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&F);
    for (uint32_t i = threadIdx.x; i < sizeof(Forest) / 4; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const uint32_t lane = lane_id();
  for (;;) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(work, 1u);
    c = __shfl_sync(kFull, c, 0);
    if (c >= total_chunks) break;
    if (chunk_order) c = __ldg(chunk_order + c);  // c < total_chunks: a permutation
    BatchDesc B;
    if (nb == 1) {
      B = b0;
    } else {
      uint32_t lo = 0, hi = nb - 1;  // largest b with chunk_begin <= c
      while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&descs[mid].chunk_begin) <= c) lo = mid; else hi = mid - 1;
      }
      B = descs[lo];
    }
    const uint32_t cb = (c - B.chunk_begin) * chunk;
    const uint32_t ce = min(cb + chunk, B.n);
    switch (B.pred) {
      case kPoint: handler_body<H, W, kPoint>(F, B, cb, ce, only); break;
      case kContains: handler_body<H, W, kContains>(F, B, cb, ce, only); break;
      case kIntersects: handler_body<H, W, kIntersects>(F, B, cb, ce, only); break;
      case kPoint64: handler_body<H, W, kPoint64>(F, B, cb, ce, only); break;
      case kContains64: handler_body<H, W, kContains64>(F, B, cb, ce, only); break;
      case kIntersects64: handler_body<H, W, kIntersects64>(F, B, cb, ce, only); break;
      default: break;
    }
  }
}

}  // namespace rts
