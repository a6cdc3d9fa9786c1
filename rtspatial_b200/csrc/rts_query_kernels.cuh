// Query kernels: one persistent launch runs any number of batches (reference
// Query calls) through a device work queue of fixed-size query chunks.
//
// A warp takes the next chunk index with one atomicAdd, finds its batch by
// binary search over the batches' first-chunk indices, and runs the chunk
// with the traversal scheme the kernel was compiled for (thread, team or
// packet; node width W).  Predicate and handler are per batch, so one launch
// can mix point-contains, range-contains and range-intersects batches, each
// writing to its own counter or queue with its own 0-based query ids.
//
// Each rts_query_occ<MINB>.cu instantiates the kernels for one occupancy
// (MINB resident blocks per SM), so that they compile in parallel.
#pragma once

#include "rts_internal.h"

namespace rts {

template <int W, bool TEAM, bool ROUTED, int PRED, int MODE>
__device__ __forceinline__ void run_chunk(const Forest& F, const BatchDesc& B, uint32_t cb,
                                          uint32_t ce, DevPair* wbuf, uint32_t* wbat,
                                          const uint32_t* only, const MergedOrder& M) {
  if constexpr (TEAM) {
    run_chunk_team<PRED, MODE, W>(F, B, cb, ce, wbuf, wbat, only);
  } else {
    run_chunk_thread<PRED, MODE, W, ROUTED>(F, B, cb, ce, wbuf, wbat, only, M);
  }
}

// Every predicate / handler body is its own function, not inlined: a
// function is register-allocated once, for its own needs (twelve bodies in one
// function were allocated for their union and spilled), and for the tightest
// budget among the kernels that call it, so the bodies are instantiated per
// MINB.  A body is called once per chunk of queries.
template <int W, bool TEAM, bool ROUTED, int MINB, int PRED, int MODE>
__device__ __noinline__ void chunk_body(const Forest& F, const BatchDesc& B, uint32_t cb,
                                        uint32_t ce, DevPair* wbuf, uint32_t* wbat,
                                        const uint32_t* only, const MergedOrder& M) {
  run_chunk<W, TEAM, ROUTED, PRED, MODE>(F, B, cb, ce, wbuf, wbat, only, M);
}

template <int W, bool TEAM, bool ROUTED, int MINB>
__device__ __forceinline__ void dispatch_chunk(const Forest& F, const BatchDesc& B, uint32_t cb,
                                               uint32_t ce, DevPair* wbuf, uint32_t* wbat,
                                               const uint32_t* only, const MergedOrder& M) {
#define RTS_RUN(P, H) chunk_body<W, TEAM, ROUTED, MINB, P, H>(F, B, cb, ce, wbuf, wbat, only, M)
  switch (B.pred * 2 + B.mode) {
    case kPoint * 2 + kCount: RTS_RUN(kPoint, kCount); break;
    case kPoint * 2 + kCollect: RTS_RUN(kPoint, kCollect); break;
    case kContains * 2 + kCount: RTS_RUN(kContains, kCount); break;
    case kContains * 2 + kCollect: RTS_RUN(kContains, kCollect); break;
    case kIntersects * 2 + kCount: RTS_RUN(kIntersects, kCount); break;
    case kIntersects * 2 + kCollect: RTS_RUN(kIntersects, kCollect); break;
    default:
      if constexpr (!TEAM) {  // double indexes (the team scheme is float only)
        switch (B.pred * 2 + B.mode) {
          case kPoint64 * 2 + kCount: RTS_RUN(kPoint64, kCount); break;
          case kPoint64 * 2 + kCollect: RTS_RUN(kPoint64, kCollect); break;
          case kContains64 * 2 + kCount: RTS_RUN(kContains64, kCount); break;
          case kContains64 * 2 + kCollect: RTS_RUN(kContains64, kCollect); break;
          case kIntersects64 * 2 + kCount: RTS_RUN(kIntersects64, kCount); break;
          case kIntersects64 * 2 + kCollect: RTS_RUN(kIntersects64, kCollect); break;
          default: break;
        }
      }
      break;
  }
#undef RTS_RUN
}

constexpr int kQueryThreads = 256;

// ROUTED: a merged launch (results routed per query); thread scheme only.
template <int W, bool TEAM, int MINB, bool ROUTED>
__global__ void __launch_bounds__(kQueryThreads, MINB)
    k_query(const __grid_constant__ Forest F_in, const __grid_constant__ BatchDesc b0,
            const BatchDesc* __restrict__ descs, uint32_t nb, uint32_t total_chunks,
            uint32_t chunk, uint32_t* __restrict__ work, const uint32_t* __restrict__ only,
            const uint32_t* __restrict__ only_any, const __grid_constant__ MergedOrder M,
            const uint32_t* __restrict__ chunk_order) {
  if (only_any && *only_any == 0) return;
  __shared__ Forest F;
  __shared__ DevPair wbufs[kQueryThreads / 32][kWarpOutCap];
  extern __shared__ __align__(16) unsigned char qdyn[];  // merged launch: batch tables
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
    uint32_t* wbat =
        ROUTED ? reinterpret_cast<uint32_t*>(qdyn) + (threadIdx.x / 32) * kWarpBatWords : nullptr;
    dispatch_chunk<W, TEAM, ROUTED, MINB>(F, B, cb, ce, wbufs[threadIdx.x / 32], wbat, only, M);
  }
}

template <int W, bool ROUTED, int MINB, int PRED, int MODE>  // per body, as chunk_body
__device__ __noinline__ void packet_body(const Forest& F, const BatchDesc& B, uint32_t cb,
                                         uint32_t ce, DevPair* wbuf, uint32_t* wbat, void* praw,
                                         const MergedOrder& M) {
  run_chunk_packet<PRED, MODE, W, ROUTED>(F, B, cb, ce, wbuf, wbat, praw, M);
}

template <int W, bool ROUTED, int MINB>
__device__ __forceinline__ void dispatch_packet(const Forest& F, const BatchDesc& B, uint32_t cb,
                                                uint32_t ce, DevPair* wbuf, uint32_t* wbat,
                                                void* praw, const MergedOrder& M) {
#define RTS_RUN(P, H) packet_body<W, ROUTED, MINB, P, H>(F, B, cb, ce, wbuf, wbat, praw, M)
  switch (B.pred * 2 + B.mode) {
    case kPoint * 2 + kCount: RTS_RUN(kPoint, kCount); break;
    case kPoint * 2 + kCollect: RTS_RUN(kPoint, kCollect); break;
    case kContains * 2 + kCount: RTS_RUN(kContains, kCount); break;
    case kContains * 2 + kCollect: RTS_RUN(kContains, kCollect); break;
    case kIntersects * 2 + kCount: RTS_RUN(kIntersects, kCount); break;
    case kIntersects * 2 + kCollect: RTS_RUN(kIntersects, kCollect); break;
    case kPoint64 * 2 + kCount: RTS_RUN(kPoint64, kCount); break;
    case kPoint64 * 2 + kCollect: RTS_RUN(kPoint64, kCollect); break;
    case kContains64 * 2 + kCount: RTS_RUN(kContains64, kCount); break;
    case kContains64 * 2 + kCollect: RTS_RUN(kContains64, kCollect); break;
    case kIntersects64 * 2 + kCount: RTS_RUN(kIntersects64, kCount); break;
    case kIntersects64 * 2 + kCollect: RTS_RUN(kIntersects64, kCollect); break;
    default: break;
  }
#undef RTS_RUN
}

template <int W>
constexpr size_t packet_stride() {
  return (packet_smem_bytes<W>() + 15) / 16 * 16;
}

// Packet scheme: same work distribution as k_query; each warp walks its
// chunk 32 queries at a time.  (No query filter: the frontier's fallback uses
// the other schemes.)
template <int W, int MINB, bool ROUTED>
__global__ void __launch_bounds__(kQueryThreads, MINB)
    k_query_packet(const __grid_constant__ Forest F_in, const __grid_constant__ BatchDesc b0,
                   const BatchDesc* __restrict__ descs, uint32_t nb, uint32_t total_chunks,
                   uint32_t chunk, uint32_t* __restrict__ work, const uint32_t* __restrict__,
                   const uint32_t* __restrict__, const __grid_constant__ MergedOrder M,
                   const uint32_t* __restrict__ chunk_order) {
  __shared__ Forest F;
  __shared__ DevPair wbufs[kQueryThreads / 32][kWarpOutCap];
  // packet_stride<W>() per warp, then (merged launch) the warps' batch tables
  extern __shared__ __align__(16) unsigned char qdyn[];
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&F_in);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&F);
    for (uint32_t i = threadIdx.x; i < sizeof(Forest) / 4; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const uint32_t lane = lane_id();
  const uint32_t wid = threadIdx.x / 32;
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
    unsigned char* praw = qdyn + wid * packet_stride<W>();
    uint32_t* wbat = ROUTED ? reinterpret_cast<uint32_t*>(
                                  qdyn + (kQueryThreads / 32) * packet_stride<W>()) +
                                  wid * kWarpBatWords
                            : nullptr;
    dispatch_packet<W, ROUTED, MINB>(F, B, cb, ce, wbufs[wid], wbat, praw, M);
  }
}

// Staged scheme (run_chunk_staged): per warp, one StageWarp<W> area at the
// start of the dynamic shared memory, then (merged launch) the warps' batch
// tables.  Returns false when a copy wait gave up (the kernel then stops).
template <int W, bool ROUTED, int PRED, int MODE>  // per body, as chunk_body
__device__ __noinline__ bool staged_body(const Forest& F, const BatchDesc& B, uint32_t cb,
                                         uint32_t ce, DevPair* wbuf, uint32_t* wbat,
                                         const uint32_t* only, const MergedOrder& M,
                                         StageWarp<W>& S) {
  return run_chunk_staged<PRED, MODE, W, ROUTED>(F, B, cb, ce, wbuf, wbat, only, M, S);
}

template <int W, bool ROUTED>
__device__ __forceinline__ bool dispatch_staged(const Forest& F, const BatchDesc& B, uint32_t cb,
                                                uint32_t ce, DevPair* wbuf, uint32_t* wbat,
                                                const uint32_t* only, const MergedOrder& M,
                                                StageWarp<W>& S) {
#define RTS_RUN(P, H) return staged_body<W, ROUTED, P, H>(F, B, cb, ce, wbuf, wbat, only, M, S)
  switch (B.pred * 2 + B.mode) {
    case kPoint * 2 + kCount: RTS_RUN(kPoint, kCount);
    case kPoint * 2 + kCollect: RTS_RUN(kPoint, kCollect);
    case kContains * 2 + kCount: RTS_RUN(kContains, kCount);
    case kContains * 2 + kCollect: RTS_RUN(kContains, kCollect);
    case kIntersects * 2 + kCount: RTS_RUN(kIntersects, kCount);
    case kIntersects * 2 + kCollect: RTS_RUN(kIntersects, kCollect);
    case kPoint64 * 2 + kCount: RTS_RUN(kPoint64, kCount);
    case kPoint64 * 2 + kCollect: RTS_RUN(kPoint64, kCollect);
    case kContains64 * 2 + kCount: RTS_RUN(kContains64, kCount);
    case kContains64 * 2 + kCollect: RTS_RUN(kContains64, kCollect);
    case kIntersects64 * 2 + kCount: RTS_RUN(kIntersects64, kCount);
    case kIntersects64 * 2 + kCollect: RTS_RUN(kIntersects64, kCollect);
    default: return true;
  }
#undef RTS_RUN
}

template <int W>
constexpr size_t staged_stride() {
  return (sizeof(StageWarp<W>) + 15) / 16 * 16;
}

// Resident CTAs per SM the staged kernels' registers are capped for: what
// their shared memory (one StageWarp<W> per warp) lets fit on an SM.
template <int W>
constexpr int staged_min_blocks() {
  return W >= 16 ? 2 : (W >= 8 ? 3 : 4);
}

template <int W, bool ROUTED>
__global__ void __launch_bounds__(kQueryThreads, staged_min_blocks<W>())
    k_query_staged(const __grid_constant__ Forest F_in, const __grid_constant__ BatchDesc b0,
                   const BatchDesc* __restrict__ descs, uint32_t nb, uint32_t total_chunks,
                   uint32_t chunk, uint32_t* __restrict__ work, const uint32_t* __restrict__ only,
                   const uint32_t* __restrict__ only_any, const __grid_constant__ MergedOrder M,
                   const uint32_t* __restrict__ chunk_order) {
  if (only_any && *only_any == 0) return;
  __shared__ Forest F;
  __shared__ DevPair wbufs[kQueryThreads / 32][kWarpOutCap];
  extern __shared__ __align__(16) unsigned char qdyn[];
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&F_in);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&F);
    for (uint32_t i = threadIdx.x; i < sizeof(Forest) / 4; i += blockDim.x) dst[i] = src[i];
  }
  const uint32_t lane = lane_id();
  const uint32_t wid = threadIdx.x / 32;
  StageWarp<W>& S = *reinterpret_cast<StageWarp<W>*>(qdyn + wid * staged_stride<W>());
  if (lane == 0) {
    mbar_init(smem_u32(&S.bar), 32);
    S.phase = 0;
    mbar_init_fence();
  }
  __syncthreads();
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
    uint32_t* wbat = ROUTED ? reinterpret_cast<uint32_t*>(
                                  qdyn + (kQueryThreads / 32) * staged_stride<W>()) +
                                  wid * kWarpBatWords
                            : nullptr;
    if (!dispatch_staged<W, ROUTED>(F, B, cb, ce, wbufs[wid], wbat, only, M, S)) break;
  }
}

using QueryKernel = void (*)(const Forest, const BatchDesc, const BatchDesc*, uint32_t, uint32_t,
                             uint32_t, uint32_t*, const uint32_t*, const uint32_t*,
                             const MergedOrder, const uint32_t*);

template <int MINB, bool ROUTED>
QueryKernel pick_kernel_occ(const LaunchPlan& p) {
  if (p.packet) {
    switch (p.width) {
      case 4: return k_query_packet<4, MINB, ROUTED>;
      case 8: return k_query_packet<8, MINB, ROUTED>;
      case 16: return k_query_packet<16, MINB, ROUTED>;
      case 32: return k_query_packet<32, MINB, ROUTED>;
    }
  } else if (p.team) {
    if constexpr (!ROUTED) {
      switch (p.width) {
        case 4: return k_query<4, true, MINB, false>;
        case 8: return k_query<8, true, MINB, false>;
        case 16: return k_query<16, true, MINB, false>;
        case 32: return k_query<32, true, MINB, false>;
      }
    }
  } else {
    switch (p.width) {
      case 4: return k_query<4, false, MINB, ROUTED>;
      case 8: return k_query<8, false, MINB, ROUTED>;
      case 16: return k_query<16, false, MINB, ROUTED>;
      case 32: return k_query<32, false, MINB, ROUTED>;
    }
  }
  return nullptr;
}


}  // namespace rts
