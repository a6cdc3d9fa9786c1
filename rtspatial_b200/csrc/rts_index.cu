// C-ABI implementation: the index manager behind rtspatial::SpatialIndex.
//
// State per index: the leaf slots (boxes + ids, grouped per sub-tree), the
// id -> slot map, and one W-wide implicit tree per sub-tree.  Insert builds a
// sub-tree for the new batch (the reference builds one GAS per batch and an
// IAS over all of them, spatial_index.cuh:142-196); after max_trees sub-trees,
// or for a batch larger than rebuild_fraction of the index, all boxes are
// re-sorted into a single tree; at the sub-tree limit, sub-trees that are
// small beside the largest are merged into one instead (merge_small_trees).
// Delete collapses boxes in place (node boxes stay conservative, no refit
// needed).  Update writes an envelope in place
// when it stays inside its leaf group's hull; otherwise the slot is emptied
// (a NaN box) and the envelope moves, with its id, into a new sub-tree.  All
// boxes are re-sorted once the updates since the last rebuild exceed
// rebuild_update_fraction of the index.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "rts_handler_kernel.cuh"
#include "rts_index_impl.h"

namespace rts {

static thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return (e == cudaErrorMemoryAllocation) ? RTS_ERR_OUT_OF_MEMORY : RTS_ERR_CUDA;
}

// Levels storable by the traversal's mask stack at each width.
static uint32_t max_levels_for(int W) {
  switch (W) {
    case 4: return MaskStack<4>::kLevels;
    case 8: return MaskStack<8>::kLevels;
    case 16: return MaskStack<16>::kLevels;
    case 32: return MaskStack<32>::kLevels;
  }
  return 0;
}

}  // namespace rts

using namespace rts;

namespace rts {

// Capacity a growing slot or id array asks for: exactly `need` the first
// time (an index built once stays tight), then at least twice the current
// capacity below 4 GB and a quarter more above.  With the re-sort buffers
// reserved alongside (reserve_for_resort), an index under rounds of updates
// and inserts allocates only when its ids or slots pass a capacity, not on
// every merge or re-sort: device allocations were measured on B200 to stall
// the host for tens to hundreds of ms at random (the driver maps memory under
// a lock the GPU's other processes share).
static size_t grown_bytes(const DevBuf& b, size_t need) {
  if (need <= b.bytes || b.bytes == 0) return need;
  const size_t cap = b.bytes < (4ull << 30) ? 2 * b.bytes : b.bytes + b.bytes / 4;
  return std::max(need, cap);
}

int ensure_sort_scratch(rts_index* ix, uint64_t n, cudaStream_t s) {
  size_t b = std::max<uint64_t>(n, 1) * sizeof(uint32_t);
  int rc;
  if ((rc = buf_reserve(ix->keys_a, b, s, false, 0))) return rc;
  if ((rc = buf_reserve(ix->keys_b, b, s, false, 0))) return rc;
  if ((rc = buf_reserve(ix->vals_a, b, s, false, 0))) return rc;
  if ((rc = buf_reserve(ix->vals_b, b, s, false, 0))) return rc;
  return buf_reserve(ix->bounds, 4 * sizeof(uint32_t), s, false, 0);
}

// Everything a full re-sort, a merge or an update split of an index within
// its current capacities uses: spare slot arrays as large as the slot arrays,
// and sort keys, values, sort temp and the slot list for as many ids as the
// id map holds.  Called when a slot or id array of a non-empty index grows.
static int reserve_for_resort(rts_index* ix, cudaStream_t s) {
  int rc;
  if ((rc = buf_reserve(ix->spare_leaves, ix->leaves.bytes, s, false, 0)) ||
      (rc = buf_reserve(ix->spare_ids, ix->leaf_ids.bytes, s, false, 0)) ||
      (is_f64(ix) && (rc = buf_reserve(ix->spare_leaves64, ix->leaves64.bytes, s, false, 0))))
    return rc;
  const uint64_t ids = ix->pos.bytes / sizeof(uint32_t);
  const uint64_t slots = ix->leaf_ids.bytes / sizeof(uint32_t);
  HostTree full;
  plan_levels(ids, ix->W, full);
  if ((rc = buf_reserve(ix->spare_nodes, full.node_entries * sizeof(float4), s, false, 0)))
    return rc;
  if ((rc = ensure_sort_scratch(ix, ids, s)) || (rc = reserve_sort_temp(ids, ix->sort_temp, s)) ||
      (rc = buf_reserve(ix->slots_tmp, std::max<uint64_t>(ids, 1) * sizeof(uint32_t), s, false, 0)) ||
      (rc = buf_reserve(ix->upd_bits, 2 * ((slots + 31) / 32) * sizeof(uint32_t), s, false, 0)))
    return rc;
  return RTS_OK;
}

int ensure_slots(rts_index* ix, uint64_t slots, cudaStream_t s) {
  uint64_t need = slots + kSlotAlign;
  int rc;
  if (!ix->status.ptr) {  // the device status word the query kernels report into
    if ((rc = buf_reserve(ix->status, sizeof(uint32_t), s, false, 0))) return rc;
    RTS_CUDA_TRY(cudaMemsetAsync(ix->status.ptr, 0, sizeof(uint32_t), s));
    ix->forest_dirty = true;
  }
  const bool grow = need * sizeof(uint32_t) > ix->leaf_ids.bytes;
  const uint64_t cap = grown_bytes(ix->leaf_ids, need * sizeof(uint32_t)) / sizeof(uint32_t);
  rc = buf_reserve(ix->leaves, cap * sizeof(float4), s, true, ix->slot_end * sizeof(float4));
  if (rc) return rc;
  if (is_f64(ix) &&
      (rc = buf_reserve(ix->leaves64, cap * sizeof(DBox), s, true, ix->slot_end * sizeof(DBox))))
    return rc;
  if ((rc = buf_reserve(ix->leaf_ids, cap * sizeof(uint32_t), s, true,
                        ix->slot_end * sizeof(uint32_t))))
    return rc;
  return grow && !ix->trees.empty() ? reserve_for_resort(ix, s) : RTS_OK;
}

int ensure_ids(rts_index* ix, uint64_t ids, cudaStream_t s);

// For an index about to take updates (a serving engine over it): the
// capacity its first mutations would allocate on their way, twice the used
// slots and ids and the re-sort buffers, reserved now.
int reserve_for_updates(rts_index* ix, cudaStream_t s) {
  if (ix->trees.empty()) return RTS_OK;
  int rc;
  const uint64_t slots_cap = ix->leaf_ids.bytes / sizeof(uint32_t);
  const uint64_t ids_cap = ix->pos.bytes / sizeof(uint32_t);
  if (slots_cap < 2 * ix->slot_end && (rc = ensure_slots(ix, slots_cap, s))) return rc;
  if (ids_cap < 2 * ix->n_ids && (rc = ensure_ids(ix, ids_cap + 1, s))) return rc;
  return reserve_for_resort(ix, s);
}

int ensure_ids(rts_index* ix, uint64_t ids, cudaStream_t s) {
  const size_t need = std::max<uint64_t>(ids, 1) * sizeof(uint32_t);
  const bool grow = need > ix->pos.bytes;
  int rc = buf_reserve(ix->pos, grown_bytes(ix->pos, need), s, true, ix->n_ids * sizeof(uint32_t));
  if (rc) return rc;
  return grow && !ix->trees.empty() ? reserve_for_resort(ix, s) : RTS_OK;
}

float4* leaves_of(rts_index* ix) { return static_cast<float4*>(ix->leaves.ptr); }
uint32_t* ids_of(rts_index* ix) { return static_cast<uint32_t*>(ix->leaf_ids.ptr); }
uint32_t* pos_of(rts_index* ix) { return static_cast<uint32_t*>(ix->pos.ptr); }


// Allocates the node buffer of `t` and packs its levels from its leaves.
int build_tree_levels(rts_index* ix, HostTree& t, cudaStream_t s) {
  plan_levels(t.n, ix->W, t);
  if (t.top > max_levels_for(ix->W))
    return fail(RTS_ERR_CAPACITY, "sub-tree too deep for node width " + std::to_string(ix->W));
  int rc = buf_reserve(t.nodes, t.node_entries * sizeof(float4), s, false, 0);
  if (rc) return rc;
  return launch_pack_tree(leaves_of(ix) + t.slot_base, t, ix->W, s);
}

// Sorts `n` boxes (src[idx[i]] or src[i]) along the curve, writes them and
// their ids to slots [slot_base, slot_base + n), and records pos[].
// src64 / dst64: a double index's double envelopes, moved with their slots.
int sort_into_slots(rts_index* ix, const float4* src, const uint32_t* src_ids, const uint32_t* idx,
                    uint64_t n, uint64_t id_begin, uint64_t slot_base, float4* dst_leaves,
                    uint32_t* dst_ids, cudaStream_t s, const DBox* src64 = nullptr,
                    DBox* dst64 = nullptr, bool live_only = false) {
  int rc = ensure_sort_scratch(ix, n, s);
  if (rc) return rc;
  auto* bounds = static_cast<uint32_t*>(ix->bounds.ptr);
  auto* ka = static_cast<uint32_t*>(ix->keys_a.ptr);
  auto* kb = static_cast<uint32_t*>(ix->keys_b.ptr);
  auto* va = static_cast<uint32_t*>(ix->vals_a.ptr);
  auto* vb = static_cast<uint32_t*>(ix->vals_b.ptr);
  if ((rc = launch_center_bounds(src, idx, n, bounds, s))) return rc;
  if ((rc = launch_curve_keys(src, idx, n, bounds, ix->cfg.curve, ka, va, s))) return rc;
  if ((rc = sort_pairs(ka, kb, va, vb, n, ix->sort_temp, s))) return rc;
  if ((rc = launch_gather(src, src_ids, vb, n, id_begin, slot_base, dst_leaves, dst_ids,
                          pos_of(ix), s, src64, dst64, live_only)))
    return rc;
  return launch_fill_pad(dst_leaves, dst_ids, slot_base + n, slot_base + round_up(n, kSlotAlign), s,
                         dst64);
}

int rebuild_all_impl(rts_index* ix, cudaStream_t s);

// Re-sorts every box of the index into one tree.
int rebuild_all(rts_index* ix, cudaStream_t s) {
  const uint64_t N = ix->n_ids;
  int rc;
  if (N == 0) return RTS_OK;
  if (!ix->ev_rebuild0) {
    RTS_CUDA_TRY(cudaEventCreate(&ix->ev_rebuild0));
    RTS_CUDA_TRY(cudaEventCreate(&ix->ev_rebuild1));
  }
  RTS_CUDA_TRY(cudaEventRecord(ix->ev_rebuild0, s));
  rc = rebuild_all_impl(ix, s);
  if (rc) return rc;
  RTS_CUDA_TRY(cudaEventRecord(ix->ev_rebuild1, s));
  ix->rebuild_timed = true;
  ix->t0_ms = 0;
  ix->updated_at_report = 0;
  return RTS_OK;
}

int rebuild_all_impl(rts_index* ix, cudaStream_t s) {
  const uint64_t N = ix->n_ids;
  int rc;
  // slots_tmp[id] = the current slot of each id (pos); slots emptied by
  // moved updates are not listed and drop out.
  if ((rc = buf_reserve(ix->slots_tmp, N * sizeof(uint32_t), s, false, 0))) return rc;
  auto* slots = static_cast<uint32_t*>(ix->slots_tmp.ptr);
  RTS_CUDA_TRY(cudaMemcpyAsync(slots, pos_of(ix), N * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  // The boxes are gathered into the spare slot arrays, which then become the
  // index's (the old ones are read by the gather and kept as the next spare).
  const uint64_t slots_needed = round_up(N, kSlotAlign);
  const uint64_t cap = std::max<uint64_t>(ix->leaf_ids.bytes / sizeof(uint32_t), slots_needed + kSlotAlign);
  if ((rc = buf_reserve(ix->spare_leaves, cap * sizeof(float4), s, false, 0)) ||
      (rc = buf_reserve(ix->spare_ids, cap * sizeof(uint32_t), s, false, 0)) ||
      (is_f64(ix) && (rc = buf_reserve(ix->spare_leaves64, cap * sizeof(DBox), s, false, 0))))
    return rc;
  rc = sort_into_slots(ix, leaves_of(ix), ids_of(ix), slots, N, 0, 0,
                       static_cast<float4*>(ix->spare_leaves.ptr),
                       static_cast<uint32_t*>(ix->spare_ids.ptr), s, leaves64_of(ix),
                       is_f64(ix) ? static_cast<DBox*>(ix->spare_leaves64.ptr) : nullptr);
  if (rc) return rc;
  std::swap(ix->leaves, ix->spare_leaves);
  std::swap(ix->leaf_ids, ix->spare_ids);
  if (is_f64(ix)) std::swap(ix->leaves64, ix->spare_leaves64);
  // The new tree is built in the spare node buffer; the largest old one
  // becomes the spare, the others are freed.
  HostTree t;
  t.nodes = ix->spare_nodes;
  ix->spare_nodes = DevBuf{};
  size_t big = 0;
  for (size_t i = 1; i < ix->trees.size(); ++i)
    if (ix->trees[i].nodes.bytes > ix->trees[big].nodes.bytes) big = i;
  for (size_t i = 0; i < ix->trees.size(); ++i) {
    if (i == big) {
      ix->spare_nodes = ix->trees[i].nodes;
      ix->trees[i].nodes = DevBuf{};
    } else {
      buf_free(ix->trees[i].nodes, s);
    }
  }
  ix->trees.clear();
  t.id_begin = 0;
  t.n = N;
  t.slot_base = 0;
  ix->slot_end = slots_needed;
  if ((rc = build_tree_levels(ix, t, s))) return rc;
  ix->trees.push_back(t);
  ix->updated_since_build = 0;
  ix->forest_dirty = true;
  ix->version++;
  return RTS_OK;
}

// Sub-tree limit reached: when every sub-tree but the largest together hold
// at most an eighth as many slots as it, they are merged into one new sub-tree
// behind the used slots and the largest stays as it is (the cost follows the
// small trees, not the index).  Their slots are gathered whole: slots
// emptied by moved updates come along as NaN boxes, which answer nothing, and
// pos[] moves only for ids whose envelope a slot still holds.  The old slots
// stay unused until the next full re-sort.  Beyond an eighth, queries would
// walk a second large tree, and a full re-sort is due instead; so is it when
// the merged slots would not fit in the slot arrays (the re-sort compacts the
// slots, where a merge would grow the arrays: an allocation on the update
// path).
static bool small_trees_mergeable(const rts_index* ix) {
  const auto& tr = ix->trees;
  if (tr.size() < 3 || ix->cfg.max_trees < 2) return false;
  size_t big = 0;
  for (size_t i = 1; i < tr.size(); ++i)
    if (tr[i].n > tr[big].n) big = i;
  if (big + 1 == tr.size()) return false;  // the newest tree (no levels yet) is the largest
  uint64_t m = 0;
  for (size_t i = 0; i < tr.size(); ++i)
    if (i != big) m += tr[i].n;
  const uint64_t end = ix->slot_end + round_up(m, kSlotAlign);
  const uint64_t room = ix->leaf_ids.bytes / sizeof(uint32_t);
  return 8 * m <= tr[big].n && end <= 2 * ix->n_ids + (1u << 20) && end + kSlotAlign <= room &&
         end < 0xffffffffull - kSlotAlign;
}

static int merge_small_trees(rts_index* ix, cudaStream_t s) {
  auto& tr = ix->trees;
  size_t big = 0;
  for (size_t i = 1; i < tr.size(); ++i)
    if (tr[i].n > tr[big].n) big = i;
  uint64_t m = 0;
  for (size_t i = 0; i < tr.size(); ++i)
    if (i != big) m += tr[i].n;
  const uint64_t base = ix->slot_end;
  const uint64_t end = base + round_up(m, kSlotAlign);
  int rc;
  if ((rc = ensure_slots(ix, end, s))) return rc;
  if ((rc = buf_reserve(ix->slots_tmp, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s, false, 0)))
    return rc;
  auto* slots = static_cast<uint32_t*>(ix->slots_tmp.ptr);
  uint64_t off = 0;
  for (size_t i = 0; i < tr.size(); ++i) {
    if (i == big) continue;
    if ((rc = launch_iota(slots + off, tr[i].slot_base, tr[i].n, s))) return rc;
    off += tr[i].n;
  }
  if ((rc = sort_into_slots(ix, leaves_of(ix), ids_of(ix), slots, m, 0, base, leaves_of(ix),
                            ids_of(ix), s, leaves64_of(ix), leaves64_of(ix), true)))
    return rc;
  HostTree keep = tr[big];
  for (size_t i = 0; i < tr.size(); ++i)
    if (i != big) buf_free(tr[i].nodes, s);
  tr.clear();
  tr.push_back(keep);
  HostTree t;
  t.id_begin = 0;  // ids of several batches: read from leaf_ids
  t.n = m;
  t.slot_base = base;
  ix->slot_end = end;
  ix->forest_dirty = true;
  ix->version++;
  if ((rc = build_tree_levels(ix, t, s))) return rc;
  tr.push_back(t);
  return RTS_OK;
}

// Whether the thread scheme's group loads bypass L1 allocation: as asked, or
// (auto) for collecting launches once the stored envelopes pass 64 MB.  A
// collecting launch stages its pairs through registers that spill to local
// memory, and L1 is better spent on those spills than on groups of a large
// index that are rarely reused; a counting launch spills less.  Measured on
// B200: streaming took config 2 (collecting, 10M boxes, 160 MB) from 1.56 to
// 1.37 ms, but config 1 (1M boxes, 16 MB, a tree hot in L1) from 0.061 to
// 0.075 ms and config 4's counting rounds (20M boxes) from 1.80 to 2.22 ms.
bool group_loads_streaming(const rts_index* ix, bool collecting) {
  if (ix->cfg.group_loads == RTS_LOADS_STREAMING) return true;
  if (ix->cfg.group_loads == RTS_LOADS_CACHED) return false;
  return collecting && ix->slot_end * sizeof(float4) > (64ull << 20);
}

int refresh_forest(rts_index* ix) {
  if (!ix->forest_dirty) return RTS_OK;
  // The thread scheme reads a W-group as W / 2 32-byte loads: the buffers the
  // groups live in must start on a 32-byte boundary (device allocations start
  // on 256-byte ones; this only guards that assumption).
  const auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 31u) == 0; };
  bool ok = aligned(ix->leaves.ptr);
  for (const auto& t : ix->trees) ok = ok && aligned(t.nodes.ptr);
  if (!ok) return fail(RTS_ERR_CUDA, "index buffer not 32-byte aligned");
  Forest& F = ix->forest;
  std::memset(&F, 0, sizeof(F));
  F.n_trees = static_cast<uint32_t>(ix->trees.size());
  F.width = static_cast<uint32_t>(ix->W);
  F.ids_base = ids_of(ix);
  F.err = static_cast<uint32_t*>(ix->status.ptr);
  F.stream_collect = group_loads_streaming(ix, true) ? 1u : 0u;
  F.stream_count = group_loads_streaming(ix, false) ? 1u : 0u;
  for (size_t i = 0; i < ix->trees.size(); ++i) {
    const HostTree& h = ix->trees[i];
    TreeDesc& d = F.tree[i];
    d.leaves = leaves_of(ix) + h.slot_base;
    d.leaves64 = is_f64(ix) ? leaves64_of(ix) + h.slot_base : nullptr;
    d.ids = ids_of(ix) + h.slot_base;
    d.nodes = static_cast<const float4*>(h.nodes.ptr);
    d.n = static_cast<uint32_t>(h.n);
    d.top = h.top;
    for (int L = 0; L < kMaxLevels; ++L) {
      d.level_off[L] = h.level_off[L];
      d.level_cnt[L] = h.level_cnt[L];
    }
  }
  ix->forest_dirty = false;
  return RTS_OK;
}

LaunchPlan plan_for(const rts_index* ix, int pred, uint64_t total) {
  LaunchPlan p;
  p.width = ix->W;
  int trav = ix->cfg.traversal;
  // Default scheme, from B200 measurements: range-intersects walks its
  // (sorted) queries in packets, the other predicates a query per lane.
  if (trav == RTS_TRAVERSAL_AUTO)
    trav = (pred == kIntersects || pred == kIntersects64) ? RTS_TRAVERSAL_PACKET
                                                          : RTS_TRAVERSAL_THREAD;
  // Double indexes run the thread or packet scheme only.
  if (is_f64(ix) && (trav == RTS_TRAVERSAL_TEAM || trav == RTS_TRAVERSAL_FRONTIER))
    trav = RTS_TRAVERSAL_THREAD;
  if (trav == RTS_TRAVERSAL_STAGED && ix->W > 16) trav = RTS_TRAVERSAL_THREAD;
  p.frontier = (trav == RTS_TRAVERSAL_FRONTIER);
  p.team = (trav == RTS_TRAVERSAL_TEAM);
  p.packet = (trav == RTS_TRAVERSAL_PACKET);
  p.staged = (trav == RTS_TRAVERSAL_STAGED);
  // Work items: the configured chunk, shrunk for small launches so that every
  // resident warp (about 32 per SM) still gets a few chunks.
  uint32_t chunk = ix->cfg.chunk ? ix->cfg.chunk : 128u;
  const uint64_t warps = static_cast<uint64_t>(device_sm_count()) * 32;
  const uint64_t fair = ((total + 4 * warps - 1) / (4 * warps) + 31) / 32 * 32;
  p.chunk = static_cast<uint32_t>(std::max<uint64_t>(32, std::min<uint64_t>(chunk, fair)));
  int occ = ix->cfg.query_occupancy;
  if (occ == 0) occ = p.packet ? 4 : (p.team ? 1 : 2);  // library default per scheme
  p.min_blocks = occ >= 4 ? 4 : (occ == 3 ? 3 : (occ == 2 ? 2 : 1));
  return p;
}

bool want_sort(const rts_index* ix, uint64_t total) {
  if (ix->cfg.sort_queries == 0) return false;
  if (ix->cfg.sort_queries == 1) return true;
  return total >= 8192;  // auto: small launches are latency-bound, skip the sort
}

bool merge_batches(const LaunchPlan& plan, const BatchDesc* descs, uint32_t nd) {
  if (nd < 2 || plan.frontier || plan.team || plan.user_kernel) return false;
  for (uint32_t i = 1; i < nd; ++i)
    if (descs[i].pred != descs[0].pred || descs[i].mode != descs[0].mode) return false;
  // Measured on B200: routing pays for counting and for the packet scheme
  // (which needs spatially coherent packets); the thread scheme collects
  // faster batch by batch.
  return descs[0].mode == kCount || plan.packet;
}

int plan_order(QueryScratch& qs, const LaunchPlan& plan, BatchDesc* descs, uint32_t nd,
               uint64_t total, uint64_t chunks, cudaStream_t s) {
  int rc;
  if ((rc = buf_reserve(qs.keys_a, total * 8, s, false, 0))) return rc;
  if ((rc = buf_reserve(qs.keys_b, total * 8, s, false, 0))) return rc;
  if ((rc = buf_reserve(qs.vals, total * 4, s, false, 0))) return rc;
  if ((rc = buf_reserve(qs.order, total * 4, s, false, 0))) return rc;
  if (plan.merged) {
    if ((rc = buf_reserve(qs.m_queries, total * sizeof(DBox), s, false, 0))) return rc;
    if ((rc = buf_reserve(qs.m_batch, total * 4, s, false, 0))) return rc;
    if ((rc = buf_reserve(qs.m_ident, total * 4, s, false, 0))) return rc;
    if ((rc = buf_reserve(qs.m_routes, nd * sizeof(DevQueue), s, false, 0))) return rc;
  }
  if (plan.chunk_order) {
    const uint64_t b = std::max<uint64_t>(chunks, 1) * 4;
    if ((rc = buf_reserve(qs.ck_keys_a, b, s, false, 0)) ||
        (rc = buf_reserve(qs.ck_keys_b, b, s, false, 0)) ||
        (rc = buf_reserve(qs.ck_vals, b, s, false, 0)) ||
        (rc = buf_reserve(qs.ck_order, b, s, false, 0)))
      return rc;
    size_t need = 0;
    if ((rc = chunk_order_temp_bytes(static_cast<uint32_t>(chunks), &need)) ||
        (rc = buf_reserve(qs.sort_temp, need, s, false, 0)))
      return rc;
  }
  uint64_t q = 0;
  for (uint32_t i = 0; i < nd; ++i) {
    descs[i].qbase = static_cast<uint32_t>(q);
    descs[i].order = plan.merged ? nullptr : static_cast<const uint32_t*>(qs.order.ptr) + q;
    q += descs[i].n;
  }
  return RTS_OK;
}

// Fills the visiting order planned by plan_order (descriptors already on the
// device when nd > 1).
int fill_order(rts_index* ix, QueryScratch& qs, const LaunchPlan& plan, const BatchDesc* host,
               const BatchDesc* dev, uint32_t nd, uint64_t total, uint64_t chunks, cudaStream_t s) {
  int rc = launch_query_order(dev, host[0], nd, total,
                            static_cast<const float4*>(ix->trees[0].nodes.ptr), ix->cfg.curve,
                            static_cast<unsigned long long*>(qs.keys_a.ptr),
                            static_cast<unsigned long long*>(qs.keys_b.ptr),
                            static_cast<uint32_t*>(qs.vals.ptr),
                            static_cast<uint32_t*>(qs.order.ptr), qs.sort_temp, s, plan.merged,
                            qs.m_queries.ptr, static_cast<uint32_t*>(qs.m_batch.ptr),
                            static_cast<uint32_t*>(qs.m_ident.ptr),
                            host[0].mode == kCollect ? static_cast<DevQueue*>(qs.m_routes.ptr)
                                                     : nullptr);
  if (rc || !plan.chunk_order) return rc;
  return launch_chunk_order(dev, nd, static_cast<uint32_t>(chunks), plan.chunk, total,
                            static_cast<const unsigned long long*>(qs.keys_b.ptr),
                            static_cast<uint32_t*>(qs.ck_keys_a.ptr),
                            static_cast<uint32_t*>(qs.ck_keys_b.ptr),
                            static_cast<uint32_t*>(qs.ck_vals.ptr),
                            static_cast<uint32_t*>(qs.ck_order.ptr), qs.sort_temp, s);
}

// Validates one public batch description against the index and, when the
// batch is not empty, fills its launch descriptor (chunk_begin and qbase from
// the running totals, which it advances).  *keep = false for an empty batch.
int batch_desc(const rts_index* ix, const rts_batch& b, const LaunchPlan& plan, uint64_t& chunks,
               uint64_t& qsum, BatchDesc& d, bool* keep) {
  *keep = false;
  int rc, mode;
  if ((rc = check_handler(b.handler, b.arg))) return rc;
  if ((rc = resolve_handler(ix, b.handler, &mode))) return rc;
  int pred;
  const bool f64 = b.query_kind == RTS_QUERY_POINTS_F64 || b.query_kind == RTS_QUERY_ENVELOPES_F64;
  if (b.query_kind == RTS_QUERY_POINTS || b.query_kind == RTS_QUERY_POINTS_F64) {
    if (b.predicate != RTS_PREDICATE_CONTAINS)
      return fail(RTS_ERR_INVALID_ARGUMENT, "points support only the contains predicate");
    pred = f64 ? kPoint64 : kPoint;
  } else if (b.query_kind == RTS_QUERY_ENVELOPES || b.query_kind == RTS_QUERY_ENVELOPES_F64) {
    if (b.predicate == RTS_PREDICATE_CONTAINS) pred = f64 ? kContains64 : kContains;
    else if (b.predicate == RTS_PREDICATE_INTERSECTS) pred = f64 ? kIntersects64 : kIntersects;
    else return fail(RTS_ERR_INVALID_ARGUMENT, "unknown predicate");
  } else {
    return fail(RTS_ERR_INVALID_ARGUMENT, "unknown query kind");
  }
  if (f64 != is_f64(ix))
    return fail(RTS_ERR_INVALID_ARGUMENT, f64 ? "double queries on a float index"
                                              : "float queries on a double index (use the _F64 kinds)");
  if (b.n == 0) return RTS_OK;
  if (!b.queries) return fail(RTS_ERR_INVALID_ARGUMENT, "batch queries is null");
  if (b.n > 0xffffffffull) return fail(RTS_ERR_CAPACITY, "more than 2^32-1 queries in a batch");
  d = BatchDesc{};
  d.queries = b.queries;
  d.arg = b.arg;
  d.n = static_cast<uint32_t>(b.n);
  d.pred = pred;
  d.mode = mode;
  d.chunk_begin = static_cast<uint32_t>(chunks);
  d.order = nullptr;
  d.qbase = static_cast<uint32_t>(qsum);
  qsum += b.n;
  if (qsum > 0xffffffffull) return fail(RTS_ERR_CAPACITY, "more than 2^32-1 queries in a launch");
  chunks += (b.n + plan.chunk - 1) / plan.chunk;
  if (chunks > 0xffffffffull) return fail(RTS_ERR_CAPACITY, "too many work items in one launch");
  *keep = true;
  return RTS_OK;
}

// Turns public batch descriptions into launch descriptors (validating them);
// empty batches are dropped.  chunks = work items of the launch.
int make_descs(const rts_index* ix, const rts_batch* batches, uint32_t n_batches,
               const LaunchPlan& plan, std::vector<BatchDesc>& out, uint64_t& chunks) {
  out.clear();
  out.reserve(n_batches);
  chunks = 0;
  uint64_t qsum = 0;
  for (uint32_t i = 0; i < n_batches; ++i) {
    BatchDesc d;
    bool keep = false;
    if (int rc = batch_desc(ix, batches[i], plan, chunks, qsum, d, &keep)) return rc;
    if (keep) out.push_back(d);
  }
  return RTS_OK;
}

int reserve_frontier(rts_index* ix, QueryScratch& qs, uint64_t total, cudaStream_t s) {
  const double f = ix->cfg.frontier_factor > 0 ? ix->cfg.frontier_factor : 16.0;
  uint64_t cap = static_cast<uint64_t>(f * static_cast<double>(total)) + 4096;
  cap = std::min<uint64_t>(cap, 0x7fffffffull / 2);
  int rc;
  if ((rc = buf_reserve(qs.fr_qbuf, total * 16, s, false, 0)) ||
      (rc = buf_reserve(qs.fr_qaux, total * 16, s, false, 0)) ||
      (rc = buf_reserve(qs.fr_qbatch, total * 4, s, false, 0)) ||
      (rc = buf_reserve(qs.fr_vis, total * 4, s, false, 0)) ||
      (rc = buf_reserve(qs.fr_a, cap * 8, s, false, 0)) ||
      (rc = buf_reserve(qs.fr_b, cap * 8, s, false, 0)) ||
      (rc = buf_reserve(qs.fr_counts, kMaxLevels * sizeof(uint32_t), s, false, 0)) ||
      (rc = buf_reserve(qs.fr_spill, ((total + 31) / 32) * 4 + 4, s, false, 0)) ||
      (rc = buf_reserve(qs.fr_any, 4, s, false, 0)))
    return rc;
  FrontierBufs& fb = qs.fb;
  fb.qbuf = qs.fr_qbuf.ptr;
  fb.qaux = qs.fr_qaux.ptr;
  fb.qbatch = static_cast<uint32_t*>(qs.fr_qbatch.ptr);
  fb.vis = static_cast<uint32_t*>(qs.fr_vis.ptr);
  fb.fa = qs.fr_a.ptr;
  fb.fb = qs.fr_b.ptr;
  fb.cap = static_cast<uint32_t>(std::min<uint64_t>(qs.fr_a.bytes, qs.fr_b.bytes) / 8);
  fb.counts = static_cast<uint32_t*>(qs.fr_counts.ptr);
  fb.counts_cap = qs.fr_counts.bytes / 4;
  fb.spill = static_cast<uint32_t*>(qs.fr_spill.ptr);
  fb.any_spill = static_cast<uint32_t*>(qs.fr_any.ptr);
  return RTS_OK;
}

int run_launch(rts_index* ix, QueryScratch& qs, const LaunchPlan& plan, const BatchDesc* descs,
               const BatchDesc* dd, uint32_t nd, uint64_t total, uint64_t chunks, cudaStream_t s) {
  bool uniform = plan.frontier && nd > 0;
  for (uint32_t i = 1; i < nd && uniform; ++i)
    uniform = descs[i].pred == descs[0].pred && descs[i].mode == descs[0].mode;
  auto* work = static_cast<uint32_t*>(qs.work.ptr);
  if (plan.merged) {
    // One batch: the sorted copy of every query; results routed per query.
    BatchDesc v{};
    v.queries = static_cast<const float*>(qs.m_queries.ptr);
    v.n = static_cast<uint32_t>(total);
    v.pred = descs[0].pred;
    v.mode = descs[0].mode;
    const MergedOrder mo{dd, static_cast<const uint32_t*>(qs.m_batch.ptr),
                         static_cast<const uint32_t*>(qs.m_ident.ptr),
                         static_cast<const DevQueue*>(qs.m_routes.ptr)};
    const uint64_t mchunks = (total + plan.chunk - 1) / plan.chunk;
    return launch_queries(ix->forest, plan, &v, nullptr, 1, static_cast<uint32_t>(mchunks), work,
                          s, nullptr, nullptr, &mo);
  }
  if (!uniform)
    return launch_queries(ix->forest, plan, descs, dd, nd, static_cast<uint32_t>(chunks), work, s,
                          nullptr, nullptr, nullptr,
                          plan.chunk_order ? static_cast<const uint32_t*>(qs.ck_order.ptr)
                                           : nullptr);
  int rc = reserve_frontier(ix, qs, total, s);
  if (rc) return rc;
  if ((rc = launch_frontier(ix->forest, descs[0].pred, descs[0].mode, descs, dd, nd,
                            static_cast<uint32_t>(total), qs.fb, s)))
    return rc;
  LaunchPlan fallback = plan;
  fallback.frontier = false;
  return launch_queries(ix->forest, fallback, descs, dd, nd, static_cast<uint32_t>(chunks), work, s,
                        qs.fb.spill, qs.fb.any_spill);
}

int launch_pred(const rts_batch* batches, uint32_t n) {
  bool isect = n > 0;
  for (uint32_t i = 0; i < n && isect; ++i)
    isect = (batches[i].query_kind == RTS_QUERY_ENVELOPES ||
             batches[i].query_kind == RTS_QUERY_ENVELOPES_F64) &&
            batches[i].predicate == RTS_PREDICATE_INTERSECTS;
  return isect ? kIntersects : kContains;
}

uint64_t sum_queries(const rts_batch* batches, uint32_t n) {
  uint64_t t = 0;
  for (uint32_t i = 0; i < n; ++i) t += batches[i].n;
  return t;
}

int check_handler(int handler, void* arg) {
  if (handler != RTS_HANDLER_COUNT && handler != RTS_HANDLER_COLLECT &&
      handler != RTS_HANDLER_MODULE)
    return fail(RTS_ERR_INVALID_ARGUMENT, "unknown handler");
  if (!arg) return fail(RTS_ERR_INVALID_ARGUMENT, "handler argument is null");
  return RTS_OK;
}

// The kernel-side handler of a public handler kind: a loaded module built
// from a shipped handler header stands for the built-in handler of the same
// behaviour; any other module is called per pair (kUser).
int resolve_handler(const rts_index* ix, int handler, int* mode) {
  if (handler != RTS_HANDLER_MODULE) {
    *mode = handler;
    return RTS_OK;
  }
  if (!ix->hmod)
    return fail(RTS_ERR_INVALID_ARGUMENT,
                "RTS_HANDLER_MODULE without a loaded handler module (rts_load_handler_module)");
  *mode = ix->hmod_builtin >= 0 ? ix->hmod_builtin : kUser;
  return RTS_OK;
}

int handler_plan(const rts_index* ix, const BatchDesc* descs, uint32_t nd, LaunchPlan& plan) {
  uint32_t user = 0;
  for (uint32_t i = 0; i < nd; ++i) user += descs[i].mode == kUser;
  if (user == 0) return RTS_OK;
  if (user != nd)
    return fail(RTS_ERR_INVALID_ARGUMENT,
                "batches with the handler module and with built-in handlers in one launch");
  const int slot = ix->W == 4 ? 0 : ix->W == 8 ? 1 : ix->W == 16 ? 2 : 3;
  plan.user_kernel = reinterpret_cast<const void*>(ix->hkern[slot]);
  plan.team = plan.packet = plan.frontier = plan.staged = false;
  plan.merged = false;
  return RTS_OK;
}

int query_one(rts_index* ix, int pred, const float* q, uint64_t n, int handler, void* arg,
              cudaStream_t s) {
  int rc = check_handler(handler, arg);
  if (rc) return rc;
  int mode;
  if ((rc = resolve_handler(ix, handler, &mode))) return rc;
  if (n == 0 || ix->n_ids == 0) return RTS_OK;  // spatial_index.cuh:354-356
  if (!q) return fail(RTS_ERR_INVALID_ARGUMENT, "queries is null");
  if (n > 0xffffffffull) return fail(RTS_ERR_CAPACITY, "more than 2^32-1 queries in one call");
  if ((rc = refresh_forest(ix))) return rc;
  if ((rc = buf_reserve(ix->qs.work, sizeof(uint32_t), s, false, 0))) return rc;
  BatchDesc b{};
  b.queries = q;
  b.arg = arg;
  b.n = static_cast<uint32_t>(n);
  b.pred = pred;
  b.mode = mode;
  b.chunk_begin = 0;
  b.order = nullptr;
  b.qbase = 0;
  LaunchPlan plan = plan_for(ix, pred, n);
  if ((rc = handler_plan(ix, &b, 1, plan))) return rc;
  if (want_sort(ix, n)) {
    const uint64_t chunks = (n + plan.chunk - 1) / plan.chunk;
    if ((rc = plan_order(ix->qs, plan, &b, 1, n, chunks, s))) return rc;
    if ((rc = fill_order(ix, ix->qs, plan, &b, nullptr, 1, n, chunks, s))) return rc;
  }
  uint64_t chunks = (n + plan.chunk - 1) / plan.chunk;
  return run_launch(ix, ix->qs, plan, &b, nullptr, 1, n, chunks, s);
}

}  // namespace rts

extern "C" {

int rts_config_default(rts_config* c) {
  if (!c) return fail(RTS_ERR_INVALID_ARGUMENT, "cfg is null");
  std::memset(c, 0, sizeof(*c));
  // rtspatial::Config defaults (spatial_index.cuh:22-37).
  c->max_geometries = 1000ull * 1000 * 10;
  c->max_queries = 1000ull * 1000;
  c->preallocate = 0;
  c->prefer_fast_build_geom = 0;
  c->prefer_fast_build_query = 0;
  c->compact = 0;
  c->geom_sample_rate = 0.2f;
  c->query_sample_rate = 0.2f;
  c->intersect_cost_weight = 0.95f;
  c->max_geom_samples = 10000;
  c->max_query_samples = 1000;
  c->max_parallelism = 512;
  // This library's structure defaults.
  c->node_width = 16;
  c->traversal = RTS_TRAVERSAL_AUTO;
  c->curve = RTS_CURVE_HILBERT;
  c->max_trees = 4;
  c->rebuild_fraction = 0.25f;
  c->sort_queries = 2;
  c->query_occupancy = 0;
  c->rebuild_update_fraction = 0.25f;
  c->chunk = 0;
  c->coord_bits = 32;
  return RTS_OK;
}

int rts_create(const rts_config* cfg, rts_index** out) {
  if (!out) return fail(RTS_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  rts_config c;
  if (cfg) c = *cfg; else rts_config_default(&c);
  if (c.node_width != 4 && c.node_width != 8 && c.node_width != 16 && c.node_width != 32)
    return fail(RTS_ERR_INVALID_ARGUMENT, "node_width must be 4, 8, 16 or 32");
  if (c.traversal < 0 || c.traversal > RTS_TRAVERSAL_STAGED)
    return fail(RTS_ERR_INVALID_ARGUMENT, "bad traversal");
  if (c.curve != RTS_CURVE_MORTON && c.curve != RTS_CURVE_HILBERT)
    return fail(RTS_ERR_INVALID_ARGUMENT, "bad curve");
  if (c.max_trees < 1 || c.max_trees > kMaxTrees)
    return fail(RTS_ERR_INVALID_ARGUMENT, "max_trees must be in 1..16");
  if (c.group_loads < RTS_LOADS_AUTO || c.group_loads > RTS_LOADS_STREAMING)
    return fail(RTS_ERR_INVALID_ARGUMENT, "bad group_loads");
  if (c.coord_bits == 0) c.coord_bits = 32;
  if (c.coord_bits != 32 && c.coord_bits != 64)
    return fail(RTS_ERR_INVALID_ARGUMENT, "coord_bits must be 32 or 64");
  auto* ix = new (std::nothrow) rts_index();
  if (!ix) return fail(RTS_ERR_OUT_OF_MEMORY, "host allocation failed");
  ix->cfg = c;
  ix->W = c.node_width;
  if (c.preallocate && c.max_geometries) {
    int rc = ensure_slots(ix, round_up(c.max_geometries, kSlotAlign) + kSlotAlign * kMaxTrees, 0);
    if (!rc) rc = ensure_ids(ix, c.max_geometries, 0);
    if (rc) {
      rts_destroy(ix);
      return rc;
    }
  }
  *out = ix;
  return RTS_OK;
}

int rts_destroy(rts_index* ix) {
  if (!ix) return RTS_OK;
  cudaStream_t s = 0;
  bool touched = false;
  for (auto& t : ix->trees) {
    touched |= t.nodes.ptr != nullptr;
    buf_free(t.nodes, s);
  }
  DevBuf* all[] = {&ix->leaves, &ix->leaf_ids, &ix->pos, &ix->keys_a, &ix->keys_b, &ix->vals_a,
                   &ix->vals_b, &ix->sort_temp, &ix->bounds, &ix->slots_tmp, &ix->leaves64,
                   &ix->spare_leaves, &ix->spare_ids, &ix->spare_leaves64, &ix->spare_nodes,
                   &ix->rounded, &ix->upd_bits, &ix->upd_ids, &ix->upd_boxes,
                   &ix->upd_boxes64, &ix->upd_count, &ix->status};
  for (DevBuf* b : all) {
    touched |= b->ptr != nullptr;
    buf_free(*b, s);
  }
  if (ix->ev_rebuild0) cudaEventDestroy(ix->ev_rebuild0);
  if (ix->ev_rebuild1) cudaEventDestroy(ix->ev_rebuild1);
  if (ix->hmod) {
    cudaDeviceSynchronize();  // no launch of its kernels may still run
    cudaLibraryUnload(ix->hmod);
  }
  touched |= ix->qs.work.ptr != nullptr;
  ix->qs.release(s);
  ix->staging.release();
  if (touched) {
    cudaStreamSynchronize(s);  // frees are stream-ordered
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) rts_trim_memory(dev);
  }
  delete ix;
  return RTS_OK;
}

int rts_clear(rts_index* ix, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (auto& t : ix->trees) buf_free(t.nodes, s);
  ix->trees.clear();
  ix->n_ids = 0;
  ix->slot_end = 0;
  ix->updated_since_build = 0;
  ix->forest_dirty = true;
  ix->version++;
  return RTS_OK;
}

}  // extern "C"

namespace rts {

// A new sub-tree of n envelopes given as floats (src) and, for a double
// index, as doubles (src64; src is then their float rounding).  ids == nullptr:
// an Insert (new ids n_ids, n_ids + 1, ...); else the envelopes keep the
// listed ids (updates moved out of their leaf group).
int insert_impl(rts_index* ix, const float4* src, const DBox* src64, const uint32_t* ids,
                uint64_t n, cudaStream_t s) {
  if (!ids && ix->n_ids + n >= 0xffffffffull)
    return fail(RTS_ERR_CAPACITY, "ids are 32-bit: at most 2^32-2 envelopes per index");
  int rc;
  // A sub-tree that does not fit behind the used slots, when the live boxes
  // and it would fit once compacted: re-sort first (a few ms) instead of
  // growing the slot arrays (an allocation of the index's size).  Merges
  // fill the arrays up to their capacity, so an index under updates and
  // inserts reaches this point between full re-sorts.
  const uint64_t room = ix->leaf_ids.bytes / sizeof(uint32_t);
  if (!ix->trees.empty() && ix->slot_end + round_up(n, kSlotAlign) + kSlotAlign > room &&
      round_up(ix->n_ids, kSlotAlign) + round_up(n, kSlotAlign) + kSlotAlign <= room &&
      (rc = rebuild_all(ix, s)))
    return rc;
  const uint64_t slot_base = ix->slot_end;
  const uint64_t slot_end = slot_base + round_up(n, kSlotAlign);
  if ((rc = ensure_slots(ix, slot_end, s))) return rc;
  if (!ids && (rc = ensure_ids(ix, ix->n_ids + n, s))) return rc;
  if ((rc = sort_into_slots(ix, src, ids, nullptr, n, ids ? 0 : ix->n_ids, slot_base,
                            leaves_of(ix), ids_of(ix), s, src64, leaves64_of(ix))))
    return rc;
  HostTree t;
  t.id_begin = ids ? 0 : ix->n_ids;
  t.n = n;
  t.slot_base = slot_base;
  const bool big_batch = !ix->trees.empty() && static_cast<double>(n) >
                                                  ix->cfg.rebuild_fraction * static_cast<double>(ix->n_ids);
  const bool at_limit = !ix->trees.empty() && static_cast<int>(ix->trees.size()) >= ix->cfg.max_trees;
  if (!ids) ix->n_ids += n;
  ix->slot_end = slot_end;
  ix->forest_dirty = true;
  ix->version++;
  if (big_batch || at_limit) {
    ix->trees.push_back(t);  // no levels yet; a merge or re-sort only reads its slots
    if (!big_batch && small_trees_mergeable(ix)) return merge_small_trees(ix, s);
    return rebuild_all(ix, s);
  }
  if ((rc = build_tree_levels(ix, t, s))) return rc;
  ix->trees.push_back(t);
  return RTS_OK;
}

// Update of n entries (rts_update_entry, or rts_update_entry_f64 for a double
// index): envelopes that stay inside their leaf group's hull are written in
// place (no hull grows, so nothing is refit); the others leave an empty slot
// and move, with their ids, to a new sub-tree.  Re-sorts everything once the
// updates since the last build pass rebuild_update_fraction of the index.
int update_impl(rts_index* ix, const void* upd, uint64_t n, cudaStream_t s) {
  int rc;
  UpdateTrees T{};
  T.n_trees = static_cast<uint32_t>(ix->trees.size());
  while ((1u << T.log2w) < static_cast<uint32_t>(ix->W)) ++T.log2w;
  for (size_t i = 0; i < ix->trees.size(); ++i) {
    const HostTree& h = ix->trees[i];
    T.slot_base[i] = h.slot_base;
    T.slot_end[i] = h.slot_base + round_up(h.n, kSlotAlign);
    T.group_hull[i] = static_cast<const float4*>(h.nodes.ptr) + h.level_off[1];
  }
  const uint64_t words = (ix->slot_end + 31) / 32;
  const bool f64 = is_f64(ix);
  if ((rc = buf_reserve(ix->upd_bits, 2 * words * sizeof(uint32_t), s, false, 0)) ||
      (rc = buf_reserve(ix->upd_ids, std::max<uint64_t>(n, 1) * sizeof(uint32_t), s, false, 0)) ||
      (rc = buf_reserve(ix->upd_boxes, std::max<uint64_t>(n, 1) * sizeof(float4), s, false, 0)) ||
      (rc = buf_reserve(ix->upd_count, sizeof(uint32_t), s, false, 0)) ||
      (f64 && (rc = buf_reserve(ix->upd_boxes64, std::max<uint64_t>(n, 1) * sizeof(DBox), s,
                                false, 0))))
    return rc;
  auto* bits = static_cast<uint32_t*>(ix->upd_bits.ptr);
  auto* mids = static_cast<uint32_t*>(ix->upd_ids.ptr);
  auto* mboxes = static_cast<float4*>(ix->upd_boxes.ptr);
  auto* mboxes64 = f64 ? static_cast<DBox*>(ix->upd_boxes64.ptr) : nullptr;
  auto* count = static_cast<uint32_t*>(ix->upd_count.ptr);
  if (f64)
    rc = launch_update_split64(static_cast<const rts_update_entry_f64*>(upd), n, ix->n_ids,
                               pos_of(ix), T, ix->slot_end, leaves_of(ix), leaves64_of(ix), bits,
                               mids, mboxes, mboxes64, count, s);
  else
    rc = launch_update_split(static_cast<const rts_update_entry*>(upd), n, ix->n_ids, pos_of(ix),
                             T, ix->slot_end, leaves_of(ix), bits, mids, mboxes, count, s);
  if (rc) return rc;
  uint32_t moved = 0;
  RTS_CUDA_TRY(cudaMemcpyAsync(&moved, count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  RTS_CUDA_TRY(cudaStreamSynchronize(s));
  ix->updated_since_build += n;
  // (a merge rebuild inside insert_impl resets updated_since_build)
  if (moved && (rc = insert_impl(ix, mboxes, mboxes64, mids, moved, s))) return rc;
  if (static_cast<double>(ix->updated_since_build) >
      ix->cfg.rebuild_update_fraction * static_cast<double>(ix->n_ids))
    return rebuild_all(ix, s);
  return RTS_OK;
}

int check_coords(const rts_index* ix, bool f64) {
  if (f64 == is_f64(ix)) return RTS_OK;
  return fail(RTS_ERR_INVALID_ARGUMENT, f64 ? "double call on a float index (coord_bits = 32)"
                                            : "float call on a double index (use the _f64 calls)");
}

}  // namespace rts

extern "C" {

int rts_insert(rts_index* ix, const float* envelopes, uint64_t n, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  int rc = check_coords(ix, false);
  if (rc) return rc;
  if (n == 0) return RTS_OK;  // spatial_index.cuh:144-146
  if (!envelopes) return fail(RTS_ERR_INVALID_ARGUMENT, "envelopes is null");
  return insert_impl(ix, reinterpret_cast<const float4*>(envelopes), nullptr, nullptr, n,
                     static_cast<cudaStream_t>(stream));
}

int rts_insert_f64(rts_index* ix, const double* envelopes, uint64_t n, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  int rc = check_coords(ix, true);
  if (rc) return rc;
  if (n == 0) return RTS_OK;
  if (!envelopes) return fail(RTS_ERR_INVALID_ARGUMENT, "envelopes is null");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const auto* src64 = reinterpret_cast<const DBox*>(envelopes);
  if ((rc = buf_reserve(ix->rounded, n * sizeof(float4), s, false, 0))) return rc;
  auto* rounded = static_cast<float4*>(ix->rounded.ptr);
  if ((rc = launch_round_boxes(src64, n, rounded, s))) return rc;
  return insert_impl(ix, rounded, src64, nullptr, n, s);
}

int rts_delete(rts_index* ix, const uint64_t* ids, uint64_t n, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  if (n == 0 || ix->n_ids == 0) return RTS_OK;
  if (!ids) return fail(RTS_ERR_INVALID_ARGUMENT, "ids is null");
  return launch_delete(ids, n, ix->n_ids, pos_of(ix), leaves_of(ix),
                       static_cast<cudaStream_t>(stream), leaves64_of(ix));
}

int rts_update(rts_index* ix, const rts_update_entry* upd, uint64_t n, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  int rc = check_coords(ix, false);
  if (rc) return rc;
  if (n == 0 || ix->n_ids == 0) return RTS_OK;
  if (!upd) return fail(RTS_ERR_INVALID_ARGUMENT, "updates is null");
  return update_impl(ix, upd, n, static_cast<cudaStream_t>(stream));
}

int rts_update_f64(rts_index* ix, const rts_update_entry_f64* upd, uint64_t n, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  int rc = check_coords(ix, true);
  if (rc) return rc;
  if (n == 0 || ix->n_ids == 0) return RTS_OK;
  if (!upd) return fail(RTS_ERR_INVALID_ARGUMENT, "updates is null");
  return update_impl(ix, upd, n, static_cast<cudaStream_t>(stream));
}

int rts_query_points(rts_index* ix, int predicate, const float* points, uint64_t n, int handler,
                     void* arg, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  if (int rc = check_coords(ix, false)) return rc;
  if (predicate != RTS_PREDICATE_CONTAINS)
    return fail(RTS_ERR_INVALID_ARGUMENT, "points support only the contains predicate");
  return query_one(ix, kPoint, points, n, handler, arg, static_cast<cudaStream_t>(stream));
}

int rts_query_envelopes(rts_index* ix, int predicate, const float* envelopes, uint64_t n,
                        int handler, void* arg, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  if (int rc = check_coords(ix, false)) return rc;
  int pred;
  if (predicate == RTS_PREDICATE_CONTAINS) pred = kContains;
  else if (predicate == RTS_PREDICATE_INTERSECTS) pred = kIntersects;
  else return fail(RTS_ERR_INVALID_ARGUMENT, "unknown predicate");
  return query_one(ix, pred, envelopes, n, handler, arg, static_cast<cudaStream_t>(stream));
}

int rts_query_points_f64(rts_index* ix, int predicate, const double* points, uint64_t n,
                         int handler, void* arg, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  if (int rc = check_coords(ix, true)) return rc;
  if (predicate != RTS_PREDICATE_CONTAINS)
    return fail(RTS_ERR_INVALID_ARGUMENT, "points support only the contains predicate");
  return query_one(ix, kPoint64, reinterpret_cast<const float*>(points), n, handler, arg,
                   static_cast<cudaStream_t>(stream));
}

int rts_query_envelopes_f64(rts_index* ix, int predicate, const double* envelopes, uint64_t n,
                            int handler, void* arg, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  if (int rc = check_coords(ix, true)) return rc;
  int pred;
  if (predicate == RTS_PREDICATE_CONTAINS) pred = kContains64;
  else if (predicate == RTS_PREDICATE_INTERSECTS) pred = kIntersects64;
  else return fail(RTS_ERR_INVALID_ARGUMENT, "unknown predicate");
  return query_one(ix, pred, reinterpret_cast<const float*>(envelopes), n, handler, arg,
                   static_cast<cudaStream_t>(stream));
}

int rts_query_batched(rts_index* ix, const rts_batch* batches, uint32_t n_batches, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  if (n_batches == 0) return RTS_OK;
  if (!batches) return fail(RTS_ERR_INVALID_ARGUMENT, "batches is null");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  LaunchPlan plan = plan_for(ix, launch_pred(batches, n_batches), sum_queries(batches, n_batches));
  std::vector<BatchDesc> descs;
  uint64_t chunks = 0;
  int rc = make_descs(ix, batches, n_batches, plan, descs, chunks);
  if (rc) return rc;
  if ((rc = handler_plan(ix, descs.data(), static_cast<uint32_t>(descs.size()), plan))) return rc;
  if (descs.empty() || ix->n_ids == 0) return RTS_OK;
  if ((rc = refresh_forest(ix))) return rc;
  if ((rc = buf_reserve(ix->qs.work, sizeof(uint32_t), s, false, 0))) return rc;
  uint64_t total = 0;
  for (const auto& d : descs) total += d.n;
  const bool sorted = want_sort(ix, total);
  plan.merged = sorted && merge_batches(plan, descs.data(), static_cast<uint32_t>(descs.size()));
  plan.chunk_order = sorted && !plan.merged && !plan.frontier && descs.size() > 1;
  if (sorted && (rc = plan_order(ix->qs, plan, descs.data(), static_cast<uint32_t>(descs.size()),
                                 total, chunks, s)))
    return rc;
  void* ddev = nullptr;
  if (descs.size() > 1 &&
      (rc = ix->staging.put(descs.data(), descs.size() * sizeof(BatchDesc), s, &ddev)))
    return rc;
  if (sorted && (rc = fill_order(ix, ix->qs, plan, descs.data(), static_cast<const BatchDesc*>(ddev),
                                 static_cast<uint32_t>(descs.size()), total, chunks, s)))
    return rc;
  return run_launch(ix, ix->qs, plan, descs.data(), static_cast<const BatchDesc*>(ddev),
                    static_cast<uint32_t>(descs.size()), total, chunks, s);
}

int rts_report_query_time(rts_index* ix, double query_ms, float* rebuild_update_fraction) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  if (!(query_ms > 0)) return fail(RTS_ERR_INVALID_ARGUMENT, "query time must be positive");
  if (ix->rebuild_timed) {
    float ms = 0;
    if (cudaEventQuery(ix->ev_rebuild1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, ix->ev_rebuild0, ix->ev_rebuild1) == cudaSuccess) {
      ix->rebuild_ms = ms;
      ix->rebuild_timed = false;
    }
  }
  const double n = static_cast<double>(std::max<uint64_t>(ix->n_ids, 1));
  const double f = static_cast<double>(ix->updated_since_build) / n;
  const double df = static_cast<double>(ix->updated_since_build - ix->updated_at_report) / n;
  ix->updated_at_report = ix->updated_since_build;
  if (ix->t0_ms <= 0 || f == 0) {
    ix->t0_ms = (ix->t0_ms <= 0) ? query_ms : std::min(ix->t0_ms, query_ms);
  } else {
    if (df > 0) ix->upd_per_report = (ix->upd_per_report > 0) ? 0.7 * ix->upd_per_report + 0.3 * df : df;
    const double a = std::max(0.0, (query_ms / ix->t0_ms - 1.0) / f);
    ix->slope = (ix->slope > 0) ? 0.7 * ix->slope + 0.3 * a : a;
  }
  // Cost per report of re-sorting every F of updates: R * u / F; expected
  // extra query time per report: t0 * a * F / 2.  Minimum at
  // F* = sqrt(2 R u / (t0 a)).
  if (ix->rebuild_ms > 0 && ix->slope > 0 && ix->upd_per_report > 0 && ix->t0_ms > 0) {
    double F = std::sqrt(2.0 * ix->rebuild_ms * ix->upd_per_report / (ix->t0_ms * ix->slope));
    ix->cfg.rebuild_update_fraction = static_cast<float>(std::min(1.0, std::max(0.005, F)));
  }
  if (rebuild_update_fraction) *rebuild_update_fraction = ix->cfg.rebuild_update_fraction;
  return RTS_OK;
}

int rts_load_handler_module(rts_index* ix, const char* path) {
  if (!ix || !path) return fail(RTS_ERR_INVALID_ARGUMENT, "index or path is null");
  cudaLibrary_t lib = nullptr;
  cudaError_t e = cudaLibraryLoadFromFile(&lib, path, nullptr, nullptr, 0, nullptr, nullptr, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(RTS_ERR_INVALID_ARGUMENT,
                std::string("cannot load handler module ") + path + ": " + cudaGetErrorString(e));
  }
  auto reject = [&](const std::string& why) {
    cudaLibraryUnload(lib);
    cudaGetLastError();
    return fail(RTS_ERR_INVALID_ARGUMENT, std::string("handler module ") + path + ": " + why);
  };
  int vals[2] = {0, 0};
  const char* globals[2] = {"rts_module_abi_version", "rts_module_builtin_handler"};
  for (int i = 0; i < 2; ++i) {
    void* d = nullptr;
    size_t bytes = 0;
    if (cudaLibraryGetGlobal(&d, &bytes, lib, globals[i]) != cudaSuccess || bytes != sizeof(int))
      return reject(std::string("no ") + globals[i]);
    if (cudaMemcpy(&vals[i], d, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      return reject(std::string("cannot read ") + globals[i]);
  }
  if (vals[0] != kHandlerModuleAbi)
    return reject("built for module version " + std::to_string(vals[0]) + ", the library reads " +
                  std::to_string(kHandlerModuleAbi));
  cudaKernel_t k[4] = {};
  const int widths[4] = {4, 8, 16, 32};
  for (int i = 0; i < 4; ++i) {
    const std::string name = "rts_handler_query_v" + std::to_string(kHandlerModuleAbi) + "_w" +
                             std::to_string(widths[i]);
    if (cudaLibraryGetKernel(&k[i], lib, name.c_str()) != cudaSuccess)
      return reject("no kernel " + name);
  }
  if (ix->hmod) {
    cudaDeviceSynchronize();
    cudaLibraryUnload(ix->hmod);
  }
  ix->hmod = lib;
  for (int i = 0; i < 4; ++i) ix->hkern[i] = k[i];
  ix->hmod_builtin = (vals[1] == RTS_HANDLER_COUNT || vals[1] == RTS_HANDLER_COLLECT) ? vals[1] : -1;
  return RTS_OK;
}

int rts_handler_module_builtin(const rts_index* ix) {
  return (ix && ix->hmod) ? ix->hmod_builtin : -1;
}

int rts_device_status(rts_index* ix, uint32_t* status, void* stream) {
  if (!ix || !status) return fail(RTS_ERR_INVALID_ARGUMENT, "index or status is null");
  *status = 0;
  if (!ix->status.ptr) return RTS_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  RTS_CUDA_TRY(cudaMemcpyAsync(status, ix->status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  RTS_CUDA_TRY(cudaStreamSynchronize(s));
  return RTS_OK;
}

uint64_t rts_size(const rts_index* ix) { return ix ? ix->n_ids : 0; }

uint32_t rts_num_trees(const rts_index* ix) {
  return ix ? static_cast<uint32_t>(ix->trees.size()) : 0;
}

uint64_t rts_memory_usage(const rts_index* ix) {
  if (!ix) return 0;
  uint64_t b = ix->leaves.bytes + ix->leaf_ids.bytes + ix->pos.bytes + ix->leaves64.bytes +
               ix->spare_leaves.bytes + ix->spare_ids.bytes + ix->spare_leaves64.bytes +
               ix->spare_nodes.bytes;
  for (const auto& t : ix->trees) b += t.nodes.bytes;
  return b;
}

const char* rts_last_error(void) { return g_err.c_str(); }

const char* rts_version(void) { return "rtspatial_b200 0.1 (sm_100a)"; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched query that allocates nothing.
//
// For callers that must not allocate device memory once they are serving:
// processes that reserve HBM for the index and its buffers at start-up and
// forbid cudaMalloc on the request path (cudaMalloc can synchronize the
// device and its latency is unbounded), host engines that hand this library
// only buffers from their own memory manager, and real-time loops that cannot
// take an allocation failure mid-request.  rts_query_batched keeps its work
// counter and the device copy of the batch descriptors in index-owned device
// buffers that it grows on demand; this variant keeps both in a file-scope
// device array of fixed size instead.
//
// The array exists once per device that loads the library and lives until the
// process exits.  Every call on a device uses the same array: the work
// counter is cleared by each call, the descriptor area keeps the previous
// call's contents, and calls that overlap on the GPU (other streams, other
// threads, other indexes) race on it.  The first call on a device looks up
// the array's device address (cudaGetSymbolAddress).
// ---------------------------------------------------------------------------
namespace {
constexpr uint32_t kNoAllocMaxBatches = RTS_NOALLOC_MAX_BATCHES;
constexpr size_t kNoAllocCounterBytes = 256;
constexpr size_t kNoAllocBytes = kNoAllocCounterBytes + kNoAllocMaxBatches * sizeof(BatchDesc);
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device; the array's name is only a host-side stand-in).
int noalloc_scratch(void** out) {
  int dev = 0;
  RTS_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(RTS_ERR_UNSUPPORTED, "device ordinal beyond the no-allocation table");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return RTS_OK;
}
}  // namespace

extern "C" int rts_query_batched_noalloc(rts_index* ix, const rts_batch* batches,
                                         uint32_t n_batches, void* stream) {
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  if (n_batches == 0) return RTS_OK;
  if (!batches) return fail(RTS_ERR_INVALID_ARGUMENT, "batches is null");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BatchDesc descs[kNoAllocMaxBatches];
  uint32_t nd = 0;
  uint64_t chunks = 0, qsum = 0;
  int rc;
  // The scheme rts_query_batched would pick for these batches; the queries
  // are visited in the callers' order (no visiting-order sort, which needs
  // scratch the size of the launch).
  LaunchPlan plan = plan_for(ix, launch_pred(batches, n_batches), sum_queries(batches, n_batches));
  for (uint32_t i = 0; i < n_batches; ++i) {
    BatchDesc d;
    bool keep = false;
    if ((rc = batch_desc(ix, batches[i], plan, chunks, qsum, d, &keep))) return rc;
    if (!keep) continue;
    if (nd == kNoAllocMaxBatches)
      return fail(RTS_ERR_CAPACITY, "rts_query_batched_noalloc takes at most " +
                                        std::to_string(kNoAllocMaxBatches) +
                                        " non-empty batches per call");
    descs[nd++] = d;
  }
  if ((rc = handler_plan(ix, descs, nd, plan))) return rc;
  if (nd == 0 || ix->n_ids == 0) return RTS_OK;
  void* scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  if ((rc = refresh_forest(ix))) return rc;
  auto* counter = static_cast<uint32_t*>(scratch);
  auto* ddescs = reinterpret_cast<BatchDesc*>(static_cast<unsigned char*>(scratch) +
                                              kNoAllocCounterBytes);
  if (nd > 1)
    RTS_CUDA_TRY(cudaMemcpyAsync(ddescs, descs, nd * sizeof(BatchDesc), cudaMemcpyHostToDevice, s));
  return launch_queries(ix->forest, plan, descs, ddescs, nd, static_cast<uint32_t>(chunks),
                        counter, s);
}
