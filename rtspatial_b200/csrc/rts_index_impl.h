// Internal definition of the index object behind the C-ABI, shared by the
// index calls (rts_index.cu), prepared launches (rts_plan.cu) and the serving
// engine (rts_server.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "rts_internal.h"

namespace rts {

// Pinned staging for small host->device copies that must not block the host:
// a ring of slots, each reused only after the copy that last read it is done.
struct Staging {
  static constexpr int kSlots = 4;
  void* host[kSlots] = {};
  DevBuf dev[kSlots];
  size_t host_bytes[kSlots] = {};
  cudaEvent_t done[kSlots] = {};
  int next = 0;

  // Copies `bytes` from src to a device buffer; returns its device address.
  int put(const void* src, size_t bytes, cudaStream_t s, void** dev_out) {
    int k = next;
    next = (next + 1) % kSlots;
    if (done[k]) RTS_CUDA_TRY(cudaEventSynchronize(done[k]));
    else RTS_CUDA_TRY(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming));
    if (host_bytes[k] < bytes) {
      if (host[k]) cudaFreeHost(host[k]);
      host[k] = nullptr;
      size_t cap = std::max<size_t>(bytes, 4096);
      RTS_CUDA_TRY(cudaMallocHost(&host[k], cap));
      host_bytes[k] = cap;
    }
    int rc = buf_reserve(dev[k], bytes, s, false, 0);
    if (rc) return rc;
    std::memcpy(host[k], src, bytes);
    RTS_CUDA_TRY(cudaMemcpyAsync(dev[k].ptr, host[k], bytes, cudaMemcpyHostToDevice, s));
    RTS_CUDA_TRY(cudaEventRecord(done[k], s));
    *dev_out = dev[k].ptr;
    return RTS_OK;
  }
  void release() {
    for (int k = 0; k < kSlots; ++k) {
      if (done[k]) {
        cudaEventSynchronize(done[k]);
        cudaEventDestroy(done[k]);
        done[k] = nullptr;
      }
      if (host[k]) cudaFreeHost(host[k]);
      host[k] = nullptr;
      host_bytes[k] = 0;
      buf_free(dev[k], 0);
    }
  }
};

// Scratch of one query launch in flight: work counter and the buffers of the
// query visiting-order sort.  Launches that may run concurrently need their
// own QueryScratch.
struct QueryScratch {
  DevBuf work, keys_a, keys_b, vals, order, sort_temp;
  // merged launch: queries in sorted order, their batch and reported id
  DevBuf m_queries, m_batch, m_ident, m_routes;
  // unmerged sorted launch: chunk keys and the chunk visiting order
  DevBuf ck_keys_a, ck_keys_b, ck_vals, ck_order;
  // frontier traversal
  DevBuf fr_qbuf, fr_qaux, fr_qbatch, fr_vis, fr_a, fr_b, fr_counts, fr_spill, fr_any;
  FrontierBufs fb;
  void release(cudaStream_t s) {
    DevBuf* all[] = {&work, &keys_a, &keys_b, &vals, &order, &sort_temp, &m_queries, &m_batch,
                     &m_ident, &m_routes, &ck_keys_a, &ck_keys_b, &ck_vals, &ck_order, &fr_qbuf, &fr_qaux, &fr_qbatch, &fr_vis, &fr_a, &fr_b,
                     &fr_counts, &fr_spill, &fr_any};
    for (DevBuf* b : all) buf_free(*b, s);
  }
};

constexpr uint64_t kSlotAlign = 32;

}  // namespace rts

struct rts_index {
  rts_config cfg{};
  int W = 8;
  uint64_t n_ids = 0;
  uint64_t slot_end = 0;        // slots in use (each sub-tree padded to 32)
  uint64_t updated_since_build = 0;
  uint64_t version = 0;         // bumped when buffers or sub-trees change
  rts::DevBuf leaves, leaf_ids, pos;
  rts::DevBuf status;           // device status word: kErr* bits set by query kernels
  // handler module (rts_load_handler_module): its kernels per node width 4, 8,
  // 16, 32, and the built-in handler it stands for (-1: the user's functions)
  cudaLibrary_t hmod = nullptr;
  cudaKernel_t hkern[4] = {};
  int hmod_builtin = -1;
  rts::DevBuf leaves64;         // double index: the double envelopes, slot by slot
  // a full re-sort gathers into these and swaps them with leaves / leaf_ids /
  // leaves64 (reserved with them once the index is mutated; see ensure_slots)
  rts::DevBuf spare_leaves, spare_ids, spare_leaves64;
  // node buffer the next full re-sort builds its tree in (the previous
  // largest sub-tree's buffer, or reserved for the id capacity)
  rts::DevBuf spare_nodes;
  rts::DevBuf rounded;          // double index: scratch of an insert's float rounding
  // scratch of the update split: slot bitmaps, moved ids / envelopes, count
  rts::DevBuf upd_bits, upd_ids, upd_boxes, upd_boxes64, upd_count;
  std::vector<rts::HostTree> trees;
  // scratch of the build path
  rts::DevBuf keys_a, keys_b, vals_a, vals_b, sort_temp, bounds, slots_tmp;
  // scratch of this index's own query calls
  rts::QueryScratch qs;
  rts::Staging staging;
  rts::Forest forest{};
  bool forest_dirty = true;
  // refit-vs-rebuild tuner state
  cudaEvent_t ev_rebuild0 = nullptr, ev_rebuild1 = nullptr;
  bool rebuild_timed = false;       // events recorded around the last re-sort
  double rebuild_ms = 0;            // duration of the last re-sort
  double t0_ms = 0;                 // query time reported right after a re-sort
  uint64_t updated_at_report = 0;   // updated_since_build at the previous report
  double upd_per_report = 0;        // EMA of the updated fraction between reports
  double slope = 0;                 // EMA of a in t = t0 * (1 + a * f)
};

namespace rts {

inline uint64_t round_up(uint64_t a, uint64_t b) { return (a + b - 1) / b * b; }
inline bool is_f64(const rts_index* ix) { return ix->cfg.coord_bits == 64; }
// The double envelopes of a double index, slot by slot (nullptr otherwise).
inline DBox* leaves64_of(rts_index* ix) {
  return is_f64(ix) ? static_cast<DBox*>(ix->leaves64.ptr) : nullptr;
}

int refresh_forest(rts_index* ix);
bool group_loads_streaming(const rts_index* ix, bool collecting);
// Re-sorts every box of the index into one tree at the index's node width.
int rebuild_all(rts_index* ix, cudaStream_t s);
LaunchPlan plan_for(const rts_index* ix, int pred, uint64_t total_queries);
uint64_t sum_queries(const rts_batch* batches, uint32_t n);
// kIntersects when every batch is a range-intersects batch, else kContains
// (the predicate plan_for picks the default traversal scheme by).
int launch_pred(const rts_batch* batches, uint32_t n);
bool want_sort(const rts_index* ix, uint64_t total);
// Reserves the capacity an index's first updates would allocate (rts_index.cu).
int reserve_for_updates(rts_index* ix, cudaStream_t s);
int check_handler(int handler, void* arg);
// The kernel-side handler (kCount, kCollect or kUser) of a public handler kind.
int resolve_handler(const rts_index* ix, int handler, int* mode);
// Whether a sorted launch of these batches runs merged: more than one batch,
// all of one predicate and handler, the thread or packet scheme, and either
// the counting handler or the packet scheme.
bool merge_batches(const LaunchPlan& plan, const BatchDesc* descs, uint32_t nd);
// Reserves the sort (and, when plan.merged, the merged-query) scratch and
// assigns each batch its slice of the launch's visiting order.  Call before
// the descriptors are staged.
int plan_order(QueryScratch& qs, const LaunchPlan& plan, BatchDesc* descs, uint32_t nd,
               uint64_t total, uint64_t chunks, cudaStream_t s);
int fill_order(rts_index* ix, QueryScratch& qs, const LaunchPlan& plan, const BatchDesc* host,
               const BatchDesc* dev, uint32_t nd, uint64_t total, uint64_t chunks, cudaStream_t s);
int make_descs(const rts_index* ix, const rts_batch* batches, uint32_t n_batches,
               const LaunchPlan& plan, std::vector<BatchDesc>& out, uint64_t& chunks);
// The launch of batches with the caller's handler module (mode kUser): every
// batch must use it; the plan then runs the module's thread-scheme kernel at
// the index's node width, batch by batch.  No-op for built-in handlers.
int handler_plan(const rts_index* ix, const BatchDesc* descs, uint32_t nd, LaunchPlan& plan);
// Sizes the frontier buffers of `qs` for `total` queries (no-op when large
// enough); fills qs.fb.
int reserve_frontier(rts_index* ix, QueryScratch& qs, uint64_t total, cudaStream_t s);
// One query launch by the plan's traversal: breadth-first plus its
// depth-first fallback when the plan asks for it and every batch shares one
// predicate and handler, depth-first otherwise.  descs: host copies; dd:
// device copy (required when nd > 1).
int run_launch(rts_index* ix, QueryScratch& qs, const LaunchPlan& plan, const BatchDesc* descs,
               const BatchDesc* dd, uint32_t nd, uint64_t total, uint64_t chunks, cudaStream_t s);

}  // namespace rts
