// Host-side internals shared by the C-ABI implementation and the launchers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "rts_device.cuh"
#include "rts_traverse.cuh"
#include "../../include/rtspatial_b200.h"

namespace rts {

// Record the per-thread message behind rts_last_error() and return the code.
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define RTS_CUDA_TRY(expr)                                 \
  do {                                                     \
    cudaError_t _e = (expr);                               \
    if (_e != cudaSuccess) return ::rts::cuda_fail(_e, #expr); \
  } while (0)

// Device memory owned by the index (stream-ordered allocator).
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};
// Device memory (rts_memory.cu): the library's caching allocator on the
// current device.  A block is usable on stream s in stream order; dev_free
// hands it back once the work queued on s before the free is done.
int dev_alloc(void** p, size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);
int buf_reserve(DevBuf& b, size_t bytes, cudaStream_t s, bool keep_contents, size_t used_bytes);
void buf_free(DevBuf& b, cudaStream_t s);

struct HostTree {
  uint64_t id_begin = 0;   // ids [id_begin, id_begin + n)
  uint64_t n = 0;
  uint64_t slot_base = 0;  // leaves slots [slot_base, slot_base + n)
  uint32_t top = 0;
  uint32_t level_off[kMaxLevels] = {};
  uint32_t level_cnt[kMaxLevels] = {};
  uint64_t node_entries = 0;
  DevBuf nodes;
};

// Level plan of one tree of n envelopes at width W: entries per level and
// their offsets in the node buffer (entry 0 = root box; levels start at W).
void plan_levels(uint64_t n, int W, HostTree& t);

// ---- build kernels (rts_build.cu) -----------------------------------------
// Boxes are read as boxes[idx[i]] when idx is non-null, else boxes[i].
// bounds: 4 device uint32 (order-preserving encodings of the centre bounds).
int launch_center_bounds(const float4* boxes, const uint32_t* idx, uint64_t n, uint32_t* bounds,
                         cudaStream_t s);
// keys[i] = curve index of the centre of box i; vals[i] = idx ? idx[i] : i.
int launch_curve_keys(const float4* boxes, const uint32_t* idx, uint64_t n, const uint32_t* bounds,
                      int curve, uint32_t* keys, uint32_t* vals, cudaStream_t s);
int sort_pairs(const uint32_t* kin, uint32_t* kout, const uint32_t* vin, uint32_t* vout,
               uint64_t n, DevBuf& temp, cudaStream_t s);
// Reserves `temp` for a sort_pairs of up to n pairs.
int reserve_sort_temp(uint64_t n, DevBuf& temp, cudaStream_t s);
// For i < n with o = order[i]: leaves[slot_base+i] = src[o];
// id = src_ids ? src_ids[o] : id_begin + o; leaf_ids[slot_base+i] = id;
// pos[id] = slot_base + i (live_only: only where pos[id] == o, i.e. slot o
// still holds id's envelope).  A double index also gathers src64 into
// leaves64.
int launch_gather(const float4* src, const uint32_t* src_ids, const uint32_t* order, uint64_t n,
                  uint64_t id_begin, uint64_t slot_base, float4* leaves, uint32_t* leaf_ids,
                  uint32_t* pos, cudaStream_t s, const DBox* src64 = nullptr,
                  DBox* leaves64 = nullptr, bool live_only = false);
// out[i] = first + i for i < n.
int launch_iota(uint32_t* out, uint64_t first, uint64_t n, cudaStream_t s);
// Empty boxes (NaN) in slots [from, to); ids = ~0.
int launch_fill_pad(float4* leaves, uint32_t* ids, uint64_t from, uint64_t to, cudaStream_t s,
                    DBox* leaves64 = nullptr);
// Levels 1..top and the root box of a tree from its leaves.
int launch_pack_tree(const float4* leaves, const HostTree& t, int W, cudaStream_t s);
// Visiting order of the queries of nb batches: sorts (batch, curve key of the
// query centre) and writes each batch's query indices to order[qbase ...].
// With `merged` (every batch of one predicate, nb > 1) the queries of all
// batches are sorted together and copied in sorted order to merged_q (float4,
// or float2 for points), with each position's batch index and reported id;
// for collecting batches merged_routes[b] receives a copy of batch b's queue.
int launch_query_order(const BatchDesc* descs, const BatchDesc& b0, uint32_t nb, uint64_t total,
                       const float4* frame_box, int curve, unsigned long long* keys_a,
                       unsigned long long* keys_b, uint32_t* vals_a, uint32_t* order,
                       DevBuf& temp, cudaStream_t s, bool merged = false, void* merged_q = nullptr,
                       uint32_t* merged_batch = nullptr, uint32_t* merged_ident = nullptr,
                       DevQueue* merged_routes = nullptr);
// Chunk visiting order of a sorted, unmerged launch of nb >= 2 batches:
// order = chunk ids sorted by the curve key of each chunk's first query
// (sorted_keys = the sorted query keys the order sort left in keys_b).
int launch_chunk_order(const BatchDesc* descs, uint32_t nb, uint32_t total_chunks, uint32_t chunk,
                       uint64_t total, const unsigned long long* sorted_keys, uint32_t* keys_a,
                       uint32_t* keys_b, uint32_t* vals_a, uint32_t* order, DevBuf& temp,
                       cudaStream_t s);
// Curve bits of the visiting-order keys of a launch of `total` queries in
// `nb` batches (the curve at about 16 cells per query, at most 16 bits per
// axis; fewer, down to 8 per axis, so that an unmerged launch's (batch,
// curve) keys fit in 24 bits).
int order_curve_bits(uint64_t total, uint32_t nb, bool merged);
int chunk_order_temp_bytes(uint32_t total_chunks, size_t* bytes);
// Temporary bytes the order sort of `total` queries in `nb` batches needs
// (an upper bound for the merged sort too).
int query_order_temp_bytes(uint64_t total, uint32_t nb, size_t* bytes);
int launch_delete(const uint64_t* ids, uint64_t n, uint64_t n_ids, const uint32_t* pos,
                  float4* leaves, cudaStream_t s, DBox* leaves64 = nullptr);

// Slot ranges and leaf-group hulls of the sub-trees, for the update split.
struct UpdateTrees {
  uint64_t slot_base[kMaxTrees];
  uint64_t slot_end[kMaxTrees];
  const float4* group_hull[kMaxTrees];  // level-1 entries: hull of each W-group of leaves
  uint32_t n_trees;
  uint32_t log2w;
};
// Update with envelopes that leave their leaf group's hull moved out (their
// slot emptied, (id, envelope) appended to moved / moved64, *n_moved counted);
// the rest written in place.  bits: 2 * ceil(slot_end / 32) words of scratch.
int launch_update_split(const rts_update_entry* upd, uint64_t n, uint64_t n_ids,
                        const uint32_t* pos, const UpdateTrees& T, uint64_t slot_end,
                        float4* leaves, uint32_t* bits, uint32_t* moved_ids, float4* moved,
                        uint32_t* n_moved, cudaStream_t s);
int launch_update_split64(const rts_update_entry_f64* upd, uint64_t n, uint64_t n_ids,
                          const uint32_t* pos, const UpdateTrees& T, uint64_t slot_end,
                          float4* leaves, DBox* leaves64, uint32_t* bits, uint32_t* moved_ids,
                          float4* moved, DBox* moved64, uint32_t* n_moved, cudaStream_t s);
// out[i] = the double envelope in[i] rounded to nearest float.
int launch_round_boxes(const DBox* in, uint64_t n, float4* out, cudaStream_t s);

// ---- frontier traversal (rts_frontier.cu) ---------------------------------
struct FrontierBufs {
  void* qbuf = nullptr;       // float4 per query of the launch
  void* qaux = nullptr;       // float4 per query (range-intersects ray data)
  uint32_t* qbatch = nullptr; // batch index per query
  uint32_t* vis = nullptr;    // visiting order: launch index of the i-th query
  void* fa = nullptr;         // level frontiers (ping-pong), cap entries each
  void* fb = nullptr;
  uint32_t cap = 0;
  uint32_t* counts = nullptr; // frontier sizes, one per level and tree
  size_t counts_cap = 0;
  uint32_t* spill = nullptr;  // bitmap of queries answered by the fallback pass
  uint32_t* any_spill = nullptr;
};
// Counters one launch needs (1 + levels of every sub-tree).
size_t frontier_counts_needed(const Forest& F);
// Breadth-first pass over every batch (all of one predicate and handler).
// Queries that overflow the frontier are flagged in fb.spill for a
// depth-first pass (launch_queries with the same bitmap).
int launch_frontier(const Forest& F, int pred, int mode, const BatchDesc* hb, const BatchDesc* dd,
                    uint32_t nb, uint32_t total, const FrontierBufs& fb, cudaStream_t s);

// ---- query launcher (rts_query.cu) ----------------------------------------
struct LaunchPlan {
  int width = 8;
  bool team = false;
  bool frontier = false;      // breadth-first pass (plus depth-first fallback)
  bool packet = false;        // warp-per-packet depth-first scheme
  bool staged = false;        // thread scheme with groups bulk-copied into shared memory
  const void* user_kernel = nullptr;  // handler module's kernel (cudaKernel_t) for kUser batches
  uint32_t chunk = 32;  // queries per work item
  int min_blocks = 1;         // CTAs of 256 threads per SM the registers are capped for (1-4)
  bool merged = false;        // sort the queries of all batches together (MergedOrder)
  bool chunk_order = false;   // sorted, unmerged, several batches: chunks visited by space
};
// Runs `nb` batches (descriptors in host memory `hb`; device copy `db` when
// nb > 1) in one persistent launch.  work_counter: zeroed device uint32.
// only / only_any (nullable): answer just the queries whose launch index
// (qbase + local) is set in the bitmap, and nothing when *only_any == 0.
int launch_queries(const Forest& F, const LaunchPlan& plan, const BatchDesc* hb,
                   const BatchDesc* db, uint32_t nb, uint32_t total_chunks,
                   uint32_t* work_counter, cudaStream_t s, const uint32_t* only = nullptr,
                   const uint32_t* only_any = nullptr, const MergedOrder* merged = nullptr,
                   const uint32_t* chunk_order = nullptr);
// Sets the chosen query kernel's shared-memory limit on the current device
// (once; call outside stream capture before a launch is captured).
int prepare_query_kernel(const LaunchPlan& plan);
// Number of SMs of the current device (cached).
int device_sm_count();
// Resident CTAs per SM of the chosen query kernel (for sizing the grid).
int query_grid_size(const LaunchPlan& plan, uint32_t total_chunks, bool merged = false);

}  // namespace rts
