// Query launcher: picks the kernel of a launch plan (compiled per occupancy
// in rts_query_occ<MINB>.cu), sizes its persistent grid and launches it.
#include <algorithm>
#include <mutex>
#include <set>
#include <utility>

#include "rts_query_kernels.cuh"

namespace rts {

// One per rts_query_occ<MINB>.cu.
QueryKernel query_kernel_occ1(const LaunchPlan& p, bool routed);
QueryKernel query_kernel_occ2(const LaunchPlan& p, bool routed);
QueryKernel query_kernel_occ3(const LaunchPlan& p, bool routed);
QueryKernel query_kernel_occ4(const LaunchPlan& p, bool routed);

// rts_query_staged.cu
QueryKernel query_kernel_staged(const LaunchPlan& p, bool routed);
size_t staged_smem_bytes(int width);

static QueryKernel pick_kernel(const LaunchPlan& p, bool routed) {
  if (p.staged) return query_kernel_staged(p, routed);
  switch (p.min_blocks) {
    case 4: return query_kernel_occ4(p, routed);
    case 3: return query_kernel_occ3(p, routed);
    case 2: return query_kernel_occ2(p, routed);
    default: return query_kernel_occ1(p, routed);
  }
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

// Dynamic shared memory of the chosen kernel: the staged scheme's per-warp
// group slots, the packet scheme's per-warp query tables, and the per-warp
// batch tables of a merged launch.
static size_t dyn_smem_bytes(const LaunchPlan& p, bool merged) {
  size_t per = 0;
  if (p.staged) {
    return staged_smem_bytes(p.width) +
           (merged ? kWarpBatWords * sizeof(uint32_t) * (kQueryThreads / 32) : 0);
  }
  if (p.packet) {
    switch (p.width) {
      case 4: per = packet_stride<4>(); break;
      case 8: per = packet_stride<8>(); break;
      case 16: per = packet_stride<16>(); break;
      case 32: per = packet_stride<32>(); break;
    }
  }
  if (merged) per += kWarpBatWords * sizeof(uint32_t);
  return per * (kQueryThreads / 32);
}

// Once per kernel and device: raises the kernel's dynamic shared-memory limit
// (to its largest use) and asks for a shared-memory carve-out no larger than
// its resident CTAs use.  L1 and shared memory share one array per SM; the
// query kernels are register-limited to fewer CTAs than their shared memory
// would allow, and the unused carve-out serves better as L1 (the kernels
// spill through it and re-read the upper tree levels from it).
static int prepare_kernel(QueryKernel k, size_t dyn) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  RTS_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(dev, reinterpret_cast<const void*>(k));
  if (done.count(key)) return RTS_OK;
  if (dyn)
    RTS_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(dyn)));
  int blocks = 0, smem_sm = 0, reserved = 0;
  cudaFuncAttributes fa{};
  RTS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, kQueryThreads, dyn));
  RTS_CUDA_TRY(cudaFuncGetAttributes(&fa, k));
  RTS_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  RTS_CUDA_TRY(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
  if (blocks > 0 && smem_sm > 0) {
    const size_t need = static_cast<size_t>(blocks) * (fa.sharedSizeBytes + dyn + reserved);
    const int pct = static_cast<int>(std::min<size_t>(100, (need * 100 + smem_sm - 1) / smem_sm + 1));
    RTS_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
  }
  done.insert(key);
  return RTS_OK;
}

int prepare_query_kernel(const LaunchPlan& plan) {
  if (plan.user_kernel) return RTS_OK;
  QueryKernel k = pick_kernel(plan, plan.merged);
  return k ? prepare_kernel(k, dyn_smem_bytes(plan, plan.merged)) : RTS_OK;
}

int query_grid_size(const LaunchPlan& plan, uint32_t total_chunks, bool merged) {
  QueryKernel k = pick_kernel(plan, merged);
  if (!k) return 0;
  device_sm_count();
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kQueryThreads,
                                                dyn_smem_bytes(plan, merged));
  if (per_sm <= 0) per_sm = 1;
  const uint32_t warps_per_block = kQueryThreads / 32;
  uint64_t want = (static_cast<uint64_t>(total_chunks) + warps_per_block - 1) / warps_per_block;
  uint64_t cap = static_cast<uint64_t>(g_num_sms) * per_sm;
  return static_cast<int>(want < cap ? want : cap);
}

int launch_queries(const Forest& F, const LaunchPlan& plan, const BatchDesc* hb,
                   const BatchDesc* db, uint32_t nb, uint32_t total_chunks,
                   uint32_t* work_counter, cudaStream_t s, const uint32_t* only,
                   const uint32_t* only_any, const MergedOrder* merged,
                   const uint32_t* chunk_order) {
  if (total_chunks == 0) return RTS_OK;
  if (plan.user_kernel) {  // the caller's handler module: its kernel, same arguments
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, plan.user_kernel, kQueryThreads,
                                                      0) != cudaSuccess ||
        per_sm <= 0) {
      cudaGetLastError();
      per_sm = 1;
    }
    const uint64_t want = (static_cast<uint64_t>(total_chunks) + kQueryThreads / 32 - 1) /
                          (kQueryThreads / 32);
    const uint64_t cap = static_cast<uint64_t>(device_sm_count()) * per_sm;
    const unsigned grid = static_cast<unsigned>(want < cap ? want : cap);
    RTS_CUDA_TRY(cudaMemsetAsync(work_counter, 0, sizeof(uint32_t), s));
    Forest F_arg = F;
    BatchDesc b0 = hb[0];
    const BatchDesc* d_arg = db;
    uint32_t nb_arg = nb, tc_arg = total_chunks, chunk_arg = plan.chunk;
    uint32_t* work_arg = work_counter;
    const uint32_t* only_arg = only;
    const uint32_t* only_any_arg = only_any;
    MergedOrder M{nullptr, nullptr, nullptr, nullptr};
    const uint32_t* order_arg = chunk_order;
    void* args[] = {&F_arg, &b0, &d_arg, &nb_arg, &tc_arg, &chunk_arg, &work_arg,
                    &only_arg, &only_any_arg, &M, &order_arg};
    RTS_CUDA_TRY(cudaLaunchKernel(plan.user_kernel, dim3(grid), dim3(kQueryThreads), args, 0, s));
    return RTS_OK;
  }
  LaunchPlan use = plan;
  if (only) use.packet = false;  // the packet scheme takes no query filter
  if (use.staged && use.width > 16) use.staged = false;  // slots hold at most 16 boxes
  QueryKernel k = pick_kernel(use, merged != nullptr);
  if (!k) return fail(RTS_ERR_INVALID_ARGUMENT, "unsupported node width / traversal");
  const size_t dyn = dyn_smem_bytes(use, merged != nullptr);
  int rc = prepare_kernel(k, dyn);
  if (rc) return rc;
  int grid = query_grid_size(use, total_chunks, merged != nullptr);
  RTS_CUDA_TRY(cudaMemsetAsync(work_counter, 0, sizeof(uint32_t), s));
  const MergedOrder M = merged ? *merged : MergedOrder{nullptr, nullptr, nullptr, nullptr};
  k<<<grid, kQueryThreads, dyn, s>>>(F, hb[0], db, nb, total_chunks, plan.chunk, work_counter,
                                     only, only_any, M, chunk_order);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

}  // namespace rts
