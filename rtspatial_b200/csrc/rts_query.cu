// Query kernels: one persistent launch runs any number of batches (reference
// Query calls) through a device work queue of fixed-size query chunks.
//
// A warp takes the next chunk index with one atomicAdd, finds its batch by
// binary search over the batches' first-chunk indices, and runs the chunk
// with the traversal scheme the kernel was compiled for (thread or team, node
// width W).  Predicate and handler are per batch, so one launch can mix
// point-contains, range-contains and range-intersects batches, each writing
// to its own counter or queue with its own 0-based query ids.
#include "rts_internal.h"

namespace rts {

template <int W, bool TEAM, int PRED, int MODE>
__device__ __forceinline__ void run_chunk(const Forest& F, const BatchDesc& B, uint32_t cb,
                                          uint32_t ce, DevPair* wbuf, const uint32_t* only) {
  if constexpr (TEAM) {
    run_chunk_team<PRED, MODE, W>(F, B, cb, ce, wbuf, only);
  } else {
    run_chunk_thread<PRED, MODE, W>(F, B, cb, ce, wbuf, only);
  }
}

template <int W, bool TEAM>
__device__ __noinline__ void dispatch_chunk(const Forest& F, const BatchDesc& B, uint32_t cb,
                                            uint32_t ce, DevPair* wbuf, const uint32_t* only) {
  switch (B.pred * 2 + B.mode) {
    case kPoint * 2 + kCount: run_chunk<W, TEAM, kPoint, kCount>(F, B, cb, ce, wbuf, only); break;
    case kPoint * 2 + kCollect: run_chunk<W, TEAM, kPoint, kCollect>(F, B, cb, ce, wbuf, only); break;
    case kContains * 2 + kCount: run_chunk<W, TEAM, kContains, kCount>(F, B, cb, ce, wbuf, only); break;
    case kContains * 2 + kCollect:
      run_chunk<W, TEAM, kContains, kCollect>(F, B, cb, ce, wbuf, only);
      break;
    case kIntersects * 2 + kCount:
      run_chunk<W, TEAM, kIntersects, kCount>(F, B, cb, ce, wbuf, only);
      break;
    case kIntersects * 2 + kCollect:
      run_chunk<W, TEAM, kIntersects, kCollect>(F, B, cb, ce, wbuf, only);
      break;
    default: break;
  }
}

constexpr int kQueryThreads = 256;

template <int W, bool TEAM, int MINB>
__global__ void __launch_bounds__(kQueryThreads, MINB)
    k_query(const __grid_constant__ Forest F_in, const __grid_constant__ BatchDesc b0,
            const BatchDesc* __restrict__ descs, uint32_t nb, uint32_t total_chunks,
            uint32_t chunk, uint32_t* __restrict__ work, const uint32_t* __restrict__ only,
            const uint32_t* __restrict__ only_any) {
  if (only_any && *only_any == 0) return;
  __shared__ Forest F;
  __shared__ DevPair wbufs[kQueryThreads / 32][kWarpOutCap];
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
    dispatch_chunk<W, TEAM>(F, B, cb, ce, wbufs[threadIdx.x / 32], only);
  }
}

using QueryKernel = void (*)(const Forest, const BatchDesc, const BatchDesc*, uint32_t, uint32_t,
                             uint32_t, uint32_t*, const uint32_t*, const uint32_t*);

template <int MINB>
static QueryKernel pick_kernel_occ(const LaunchPlan& p) {
  if (p.team) {
    switch (p.width) {
      case 4: return k_query<4, true, MINB>;
      case 8: return k_query<8, true, MINB>;
      case 16: return k_query<16, true, MINB>;
      case 32: return k_query<32, true, MINB>;
    }
  } else {
    switch (p.width) {
      case 4: return k_query<4, false, MINB>;
      case 8: return k_query<8, false, MINB>;
      case 16: return k_query<16, false, MINB>;
      case 32: return k_query<32, false, MINB>;
    }
  }
  return nullptr;
}

static QueryKernel pick_kernel(const LaunchPlan& p) {
  return p.high_occupancy ? pick_kernel_occ<4>(p) : pick_kernel_occ<1>(p);
}

static int g_num_sms = 0;

int device_sm_count() {
  if (g_num_sms == 0) {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    g_num_sms = n > 0 ? n : 1;
  }
  return g_num_sms;
}

int query_grid_size(const LaunchPlan& plan, uint32_t total_chunks) {
  QueryKernel k = pick_kernel(plan);
  if (!k) return 0;
  device_sm_count();
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kQueryThreads, 0);
  if (per_sm <= 0) per_sm = 1;
  const uint32_t warps_per_block = kQueryThreads / 32;
  uint64_t want = (static_cast<uint64_t>(total_chunks) + warps_per_block - 1) / warps_per_block;
  uint64_t cap = static_cast<uint64_t>(g_num_sms) * per_sm;
  return static_cast<int>(want < cap ? want : cap);
}

int launch_queries(const Forest& F, const LaunchPlan& plan, const BatchDesc* hb,
                   const BatchDesc* db, uint32_t nb, uint32_t total_chunks,
                   uint32_t* work_counter, cudaStream_t s, const uint32_t* only,
                   const uint32_t* only_any) {
  if (total_chunks == 0) return RTS_OK;
  QueryKernel k = pick_kernel(plan);
  if (!k) return fail(RTS_ERR_INVALID_ARGUMENT, "unsupported node width / traversal");
  int grid = query_grid_size(plan, total_chunks);
  RTS_CUDA_TRY(cudaMemsetAsync(work_counter, 0, sizeof(uint32_t), s));
  k<<<grid, kQueryThreads, 0, s>>>(F, hb[0], db, nb, total_chunks, plan.chunk, work_counter, only,
                                   only_any);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

}  // namespace rts
