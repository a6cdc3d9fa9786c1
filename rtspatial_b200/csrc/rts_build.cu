// Structure maintenance kernels: curve keys, radix sort, leaf packing, level
// refit, Delete and Update.  These replace optixAccelBuild (BUILD and UPDATE
// operations, rtspatial details/rt_engine.h:680-903) with a linear BVH:
// leaves sorted along a Morton or Hilbert curve of the box centres, grouped W
// at a time, and W-wide upper levels computed as hulls of consecutive
// entries.
#include <algorithm>
#include <cub/device/device_radix_sort.cuh>

#include "rts_internal.h"

namespace rts {

namespace {

constexpr int kThreads = 256;

__host__ __device__ inline uint64_t div_up(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// Order-preserving map of floats to unsigned ints (for atomicMin/Max).
__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t o) {
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// Empty slot (padding, or a slot whose envelope moved to another sub-tree):
// NaN in every coordinate fails each comparison of every predicate, so it
// answers no query, even ones with infinite coordinates, and fminf / fmaxf
// leave it out of node hulls.
__device__ __forceinline__ float4 empty_box() {
  return make_float4(__int_as_float(0x7fffffff), __int_as_float(0x7fffffff),
                     __int_as_float(0x7fffffff), __int_as_float(0x7fffffff));
}
__device__ __forceinline__ DBox empty_dbox() {
  const double n = __longlong_as_double(0x7fffffffffffffffll);
  return DBox{make_double2(n, n), make_double2(n, n)};
}

__device__ __forceinline__ float4 hull(float4 b) {
  return make_float4(fminf(b.x, b.z), fminf(b.y, b.w), fmaxf(b.x, b.z), fmaxf(b.y, b.w));
}

__device__ __forceinline__ float2 center(float4 b) {
  float4 h = hull(b);
  return make_float2(0.5f * (h.x + h.z), 0.5f * (h.y + h.w));
}

__global__ void k_center_bounds(const float4* __restrict__ boxes, const uint32_t* __restrict__ idx,
                                uint64_t n, uint32_t* __restrict__ out) {
  float lx = INFINITY, ly = INFINITY, hx = -INFINITY, hy = -INFINITY;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float2 c = center(boxes[idx ? idx[i] : i]);
    lx = fminf(lx, c.x);
    ly = fminf(ly, c.y);
    hx = fmaxf(hx, c.x);
    hy = fmaxf(hy, c.y);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lx = fminf(lx, __shfl_xor_sync(kFull, lx, o));
    ly = fminf(ly, __shfl_xor_sync(kFull, ly, o));
    hx = fmaxf(hx, __shfl_xor_sync(kFull, hx, o));
    hy = fmaxf(hy, __shfl_xor_sync(kFull, hy, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&out[0], f2ord(lx));
    atomicMin(&out[1], f2ord(ly));
    atomicMax(&out[2], f2ord(hx));
    atomicMax(&out[3], f2ord(hy));
  }
}

__device__ __forceinline__ uint32_t spread16(uint32_t x) {
  x &= 0xffffu;
  x = (x | (x << 8)) & 0x00ff00ffu;
  x = (x | (x << 4)) & 0x0f0f0f0fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

// Index along the order-16 Hilbert curve of cell (x, y), x, y < 2^16 (the
// classic iterative rotate-and-reflect conversion).
__device__ __forceinline__ uint32_t hilbert16(uint32_t x, uint32_t y) {
  uint32_t d = 0;
  for (uint32_t s = 1u << 15; s > 0; s >>= 1) {
    uint32_t rx = (x & s) ? 1u : 0u;
    uint32_t ry = (y & s) ? 1u : 0u;
    d += s * s * ((3u * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = 0xffffu - x;
        y = 0xffffu - y;
      }
      uint32_t t = x;
      x = y;
      y = t;
    }
  }
  return d;
}

__global__ void k_curve_keys(const float4* __restrict__ boxes, const uint32_t* __restrict__ idx,
                             uint64_t n, const uint32_t* __restrict__ bounds, int curve,
                             uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float lx = ord2f(bounds[0]), ly = ord2f(bounds[1]);
  const float hx = ord2f(bounds[2]), hy = ord2f(bounds[3]);
  const float sx = (hx > lx) ? 65535.0f / (hx - lx) : 0.0f;
  const float sy = (hy > ly) ? 65535.0f / (hy - ly) : 0.0f;
  const uint32_t src = idx ? idx[i] : static_cast<uint32_t>(i);
  float2 c = center(boxes[src]);
  uint32_t qx = __float2uint_rz(fminf(fmaxf((c.x - lx) * sx, 0.0f), 65535.0f));
  uint32_t qy = __float2uint_rz(fminf(fmaxf((c.y - ly) * sy, 0.0f), 65535.0f));
  keys[i] = (curve == RTS_CURVE_HILBERT) ? hilbert16(qx, qy) : (spread16(qx) | (spread16(qy) << 1));
  vals[i] = src;
}

__global__ void k_gather(const float4* __restrict__ src, const uint32_t* __restrict__ src_ids,
                         const uint32_t* __restrict__ order, uint64_t n, uint64_t id_begin,
                         uint64_t slot_base, float4* __restrict__ leaves,
                         uint32_t* __restrict__ leaf_ids, uint32_t* __restrict__ pos,
                         const DBox* __restrict__ src64, DBox* __restrict__ leaves64,
                         bool live_only) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t o = order[i];
  uint32_t id = src_ids ? src_ids[o] : static_cast<uint32_t>(id_begin + o);
  uint64_t slot = slot_base + i;
  leaves[slot] = src[o];
  if (leaves64) leaves64[slot] = src64[o];
  leaf_ids[slot] = id;
  // An emptied slot (its envelope moved on) keeps a stale id: pos[id] points
  // elsewhere and stays.  New slots lie past every source slot, so a stale
  // copy never matches, whichever order the two copies' threads run in.
  if (!live_only || pos[id] == o) pos[id] = static_cast<uint32_t>(slot);
}

__global__ void k_iota(uint32_t* __restrict__ out, uint64_t first, uint64_t n) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = static_cast<uint32_t>(first + i);
}

__global__ void k_fill_pad(float4* __restrict__ leaves, uint32_t* __restrict__ ids, uint64_t from,
                           uint64_t to, DBox* __restrict__ leaves64) {
  uint64_t i = from + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= to) return;
  leaves[i] = empty_box();
  if (leaves64) leaves64[i] = empty_dbox();
  if (ids) ids[i] = 0xffffffffu;
}

// out[j] = hull of in[j*G .. j*G+G) for j < n_out_pad; entries past n_in are
// empty.  One lane per input entry, shuffles reduce each aligned group.
__global__ void k_pack(const float4* __restrict__ in, uint64_t n_in, float4* __restrict__ out,
                       uint64_t n_out_pad, int log2g) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  float4 b = make_float4(INFINITY, INFINITY, -INFINITY, -INFINITY);
  if (i < n_in) b = hull(in[i]);
  for (int o = 1; o < (1 << log2g); o <<= 1) {
    b.x = fminf(b.x, __shfl_xor_sync(kFull, b.x, o));
    b.y = fminf(b.y, __shfl_xor_sync(kFull, b.y, o));
    b.z = fmaxf(b.z, __shfl_xor_sync(kFull, b.z, o));
    b.w = fmaxf(b.w, __shfl_xor_sync(kFull, b.w, o));
  }
  uint64_t j = i >> log2g;
  if ((i & ((1u << log2g) - 1)) == 0 && j < n_out_pad) out[j] = b;
}


// Delete: Envelope::Invalid() (max := min) on each listed id below n_ids
// (spatial_index.cuh:216-233); the box stays in its slot.
__global__ void k_delete(const uint64_t* __restrict__ ids, uint64_t n, uint64_t n_ids,
                         const uint32_t* __restrict__ pos, float4* __restrict__ leaves,
                         DBox* __restrict__ leaves64) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t id = ids[i];
  if (id >= n_ids) return;
  uint32_t slot = pos[id];
  float4 b = leaves[slot];
  b.z = b.x;
  b.w = b.y;
  leaves[slot] = b;
  if (leaves64) leaves64[slot].hi = leaves64[slot].lo;  // Invalid(): max := min in double
}



// ---- Update split ------------------------------------------------------------
// An updated envelope that stays inside the hull of its leaf group (the
// level-1 entry above its slot) is written in place: no hull has to grow.  One
// that leaves it would stretch every hull up to the root, so its slot becomes
// an empty box (matches nothing) and the envelope moves, with its id, to a new
// sub-tree (rts_update builds it like an insert).  Decided per slot: pass 1
// marks the slots with an outward update, pass 2 writes the unmarked slots in
// place and lets one update per marked slot claim the move, so an id listed
// twice still ends up with exactly one envelope.

__device__ __forceinline__ bool slot_keeps(const UpdateTrees& T, uint32_t slot, float4 b) {
  for (uint32_t t = 0; t < T.n_trees; ++t) {
    if (slot >= T.slot_base[t] && slot < T.slot_end[t]) {
      const float4 H = T.group_hull[t][(slot - T.slot_base[t]) >> T.log2w];
      const float4 h = hull(b);
      return H.x <= h.x && H.y <= h.y && h.z <= H.z && h.w <= H.w;
    }
  }
  return false;
}

__device__ __forceinline__ void set_bit(uint32_t* bits, uint32_t i) {
  atomicOr(bits + (i >> 5), 1u << (i & 31));
}

template <typename E>
__device__ __forceinline__ float4 entry_box(const E& e) {
  if constexpr (sizeof(e.min_x) == 8)
    return round_box(DBox{make_double2(e.min_x, e.min_y), make_double2(e.max_x, e.max_y)});
  else
    return make_float4(e.min_x, e.min_y, e.max_x, e.max_y);
}

template <typename E>
__global__ void k_update_mark(const E* __restrict__ upd, uint64_t n, uint64_t n_ids,
                              const uint32_t* __restrict__ pos, const UpdateTrees T,
                              uint32_t* __restrict__ moves) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const E e = upd[i];
  if (e.id >= n_ids) return;
  const uint32_t slot = pos[e.id];
  if (!slot_keeps(T, slot, entry_box(e))) set_bit(moves, slot);
}

template <typename E>
__global__ void k_update_apply(const E* __restrict__ upd, uint64_t n, uint64_t n_ids,
                               const uint32_t* __restrict__ pos, float4* __restrict__ leaves,
                               DBox* __restrict__ leaves64, const uint32_t* __restrict__ moves,
                               uint32_t* __restrict__ claimed, uint32_t* __restrict__ moved_ids,
                               float4* __restrict__ moved, DBox* __restrict__ moved64,
                               uint32_t* __restrict__ n_moved) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const E e = upd[i];
  if (e.id >= n_ids) return;
  const uint32_t slot = pos[e.id];
  const float4 b = entry_box(e);
  DBox b64{};
  if constexpr (sizeof(e.min_x) == 8)
    b64 = DBox{make_double2(e.min_x, e.min_y), make_double2(e.max_x, e.max_y)};
  const uint32_t bit = 1u << (slot & 31);
  if (!(moves[slot >> 5] & bit)) {  // stays: in place
    leaves[slot] = b;
    if (leaves64) leaves64[slot] = b64;
    return;
  }
  if (atomicOr(claimed + (slot >> 5), bit) & bit) return;  // another update moves this id
  leaves[slot] = empty_box();
  if (leaves64) leaves64[slot] = empty_dbox();
  const uint32_t k = atomicAdd(n_moved, 1u);
  moved_ids[k] = static_cast<uint32_t>(e.id);
  moved[k] = b;
  if (moved64) moved64[k] = b64;
}

// Double index: float rounding of inserted envelopes.
__global__ void k_round_boxes(const DBox* __restrict__ in, uint64_t n, float4* __restrict__ out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = round_box(in[i]);
}

__device__ __forceinline__ uint32_t batch_of_query(const BatchDesc* descs, uint32_t nb,
                                                   uint64_t i) {
  if (nb <= 1) return 0;
  uint32_t lo = 0, hi = nb - 1;  // largest b with qbase <= i
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (descs[mid].qbase <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Visiting order of queries: key = (batch index << 32) | curve index of the
// query's centre in the frame of the first sub-tree's root box; value = the
// query's index within its batch.  Sorting by key groups batches and, within
// a batch, puts queries that walk the same nodes next to each other.  Merged:
// key = curve index alone, value = the query's index in the launch, so the
// sort interleaves the batches by position.
__global__ void k_query_keys(const BatchDesc* __restrict__ descs, const BatchDesc b0, uint32_t nb,
                             uint64_t total, const float4* __restrict__ frame_box, int curve,
                             unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals,
                             bool merged, int curve_bits) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const uint32_t b = batch_of_query(descs, nb, i);
  const BatchDesc& B = (nb > 1) ? descs[b] : b0;
  const uint32_t local = static_cast<uint32_t>(i - B.qbase);
  float2 c;
  if (B.pred == kPoint) {
    c = reinterpret_cast<const float2*>(B.queries)[local];
  } else if (B.pred == kPoint64) {
    const double2 p = reinterpret_cast<const double2*>(B.queries)[local];
    c = make_float2(__double2float_rn(p.x), __double2float_rn(p.y));
  } else if (B.pred >= kPoint64) {
    c = center(round_box(reinterpret_cast<const DBox*>(B.queries)[local]));
  } else {
    c = center(reinterpret_cast<const float4*>(B.queries)[local]);
  }
  const float4 f = *frame_box;
  const float sx = (f.z > f.x) ? 65535.0f / (f.z - f.x) : 0.0f;
  const float sy = (f.w > f.y) ? 65535.0f / (f.w - f.y) : 0.0f;
  uint32_t qx = __float2uint_rz(fminf(fmaxf((c.x - f.x) * sx, 0.0f), 65535.0f));
  uint32_t qy = __float2uint_rz(fminf(fmaxf((c.y - f.y) * sy, 0.0f), 65535.0f));
  uint32_t k = (curve == RTS_CURVE_HILBERT) ? hilbert16(qx, qy) : (spread16(qx) | (spread16(qy) << 1));
  k >>= 32 - curve_bits;  // the curve at 2^(curve_bits/2) cells per axis
  keys[i] = merged ? k : (static_cast<unsigned long long>(b) << curve_bits) | k;
  vals[i] = merged ? static_cast<uint32_t>(i) : local;
}

// Chunk visiting order of an unmerged sorted launch: chunk c of batch b
// starts at sorted position qbase_b + (c - chunk_begin_b) * chunk, whose key
// (batch << 32 | curve) gives the chunk's curve position.  Sorting chunks by
// it makes the chunks in flight, whatever their batch, neighbours in space.
__global__ void k_chunk_keys(const BatchDesc* __restrict__ descs, uint32_t nb,
                             uint32_t total_chunks, uint32_t chunk,
                             const unsigned long long* __restrict__ sorted_keys, uint32_t curve_mask,
                             uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (c >= total_chunks) return;
  uint32_t lo = 0, hi = nb - 1;  // largest b with chunk_begin <= c
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (descs[mid].chunk_begin <= c) lo = mid; else hi = mid - 1;
  }
  const BatchDesc& B = descs[lo];
  const uint64_t pos = B.qbase + static_cast<uint64_t>(c - B.chunk_begin) * chunk;
  keys[c] = static_cast<uint32_t>(sorted_keys[pos]) & curve_mask;
  vals[c] = static_cast<uint32_t>(c);
}

// Merged launch: copies the queries in sorted order (order[j] = index in the
// launch) and records each position's batch and reported query id.  The
// first nb threads also copy the batches' queue headers into routes.
__global__ void k_merge_queries(const BatchDesc* __restrict__ descs, uint32_t nb, uint64_t total,
                                const uint32_t* __restrict__ order, void* __restrict__ out_q,
                                uint32_t* __restrict__ out_batch, uint32_t* __restrict__ out_ident,
                                DevQueue* __restrict__ routes) {
  uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (routes && j < nb) routes[j] = *static_cast<const DevQueue*>(descs[j].arg);
  if (j >= total) return;
  const uint32_t g = order[j];
  const uint32_t b = batch_of_query(descs, nb, g);
  const BatchDesc& B = descs[b];
  const uint32_t local = g - B.qbase;
  if (B.pred == kPoint) {
    reinterpret_cast<float2*>(out_q)[j] = reinterpret_cast<const float2*>(B.queries)[local];
  } else if (B.pred == kPoint64) {
    reinterpret_cast<double2*>(out_q)[j] = reinterpret_cast<const double2*>(B.queries)[local];
  } else if (B.pred >= kPoint64) {
    reinterpret_cast<DBox*>(out_q)[j] = reinterpret_cast<const DBox*>(B.queries)[local];
  } else {
    reinterpret_cast<float4*>(out_q)[j] = reinterpret_cast<const float4*>(B.queries)[local];
  }
  out_batch[j] = b;
  out_ident[j] = local + B.id_offset;
}

inline unsigned grid_for(uint64_t n) {
  uint64_t g = div_up(n, kThreads);
  return static_cast<unsigned>(g ? g : 1);
}

}  // namespace

void plan_levels(uint64_t n, int W, HostTree& t) {
  for (int i = 0; i < kMaxLevels; ++i) t.level_off[i] = t.level_cnt[i] = 0;
  t.level_cnt[0] = static_cast<uint32_t>(n);
  uint64_t cnt = n;
  uint64_t off = static_cast<uint64_t>(W);  // entries 0..W-1: root box + spare
  uint32_t L = 0;
  do {
    ++L;
    cnt = div_up(cnt, W);
    t.level_cnt[L] = static_cast<uint32_t>(cnt);
    t.level_off[L] = static_cast<uint32_t>(off);
    off += div_up(cnt, W) * W;
  } while (cnt > static_cast<uint64_t>(W) && L + 1 < kMaxLevels);
  t.top = L;
  t.node_entries = off;
}

int launch_center_bounds(const float4* boxes, const uint32_t* idx, uint64_t n, uint32_t* bounds,
                         cudaStream_t s) {
  RTS_CUDA_TRY(cudaMemsetAsync(bounds, 0xff, 2 * sizeof(uint32_t), s));
  RTS_CUDA_TRY(cudaMemsetAsync(bounds + 2, 0x00, 2 * sizeof(uint32_t), s));
  if (n == 0) return RTS_OK;
  unsigned g = static_cast<unsigned>(div_up(n, kThreads));
  if (g > 148u * 8u) g = 148u * 8u;
  k_center_bounds<<<g, kThreads, 0, s>>>(boxes, idx, n, bounds);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

int launch_curve_keys(const float4* boxes, const uint32_t* idx, uint64_t n, const uint32_t* bounds,
                      int curve, uint32_t* keys, uint32_t* vals, cudaStream_t s) {
  if (n == 0) return RTS_OK;
  k_curve_keys<<<grid_for(n), kThreads, 0, s>>>(boxes, idx, n, bounds, curve, keys, vals);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

int sort_pairs(const uint32_t* kin, uint32_t* kout, const uint32_t* vin, uint32_t* vout,
               uint64_t n, DevBuf& temp, cudaStream_t s) {
  if (n == 0) return RTS_OK;
  size_t need = 0;
  RTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, kin, kout, vin, vout,
                                                static_cast<int>(n), 0, 32, s));
  int rc = buf_reserve(temp, need, s, false, 0);
  if (rc) return rc;
  RTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.ptr, need, kin, kout, vin, vout,
                                                static_cast<int>(n), 0, 32, s));
  return RTS_OK;
}

int reserve_sort_temp(uint64_t n, DevBuf& temp, cudaStream_t s) {
  if (n == 0) return RTS_OK;
  size_t need = 0;
  RTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, static_cast<const uint32_t*>(nullptr),
                                                static_cast<uint32_t*>(nullptr),
                                                static_cast<const uint32_t*>(nullptr),
                                                static_cast<uint32_t*>(nullptr),
                                                static_cast<int>(n), 0, 32, s));
  return buf_reserve(temp, need, s, false, 0);
}

int launch_gather(const float4* src, const uint32_t* src_ids, const uint32_t* order, uint64_t n,
                  uint64_t id_begin, uint64_t slot_base, float4* leaves, uint32_t* leaf_ids,
                  uint32_t* pos, cudaStream_t s, const DBox* src64, DBox* leaves64,
                  bool live_only) {
  if (n == 0) return RTS_OK;
  k_gather<<<grid_for(n), kThreads, 0, s>>>(src, src_ids, order, n, id_begin, slot_base, leaves,
                                            leaf_ids, pos, src64, leaves64, live_only);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

int launch_iota(uint32_t* out, uint64_t first, uint64_t n, cudaStream_t s) {
  if (n == 0) return RTS_OK;
  k_iota<<<grid_for(n), kThreads, 0, s>>>(out, first, n);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

int launch_fill_pad(float4* leaves, uint32_t* ids, uint64_t from, uint64_t to, cudaStream_t s,
                    DBox* leaves64) {
  if (to <= from) return RTS_OK;
  k_fill_pad<<<grid_for(to - from), kThreads, 0, s>>>(leaves, ids, from, to, leaves64);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

int launch_pack_tree(const float4* leaves, const HostTree& t, int W, cudaStream_t s) {
  int log2w = 0;
  while ((1 << log2w) < W) ++log2w;
  float4* nodes = static_cast<float4*>(t.nodes.ptr);
  for (uint32_t L = 1; L <= t.top; ++L) {
    const float4* in = (L == 1) ? leaves : nodes + t.level_off[L - 1];
    uint64_t n_in = t.level_cnt[L - 1];
    uint64_t n_out_pad = div_up(t.level_cnt[L], W) * W;
    uint64_t threads = n_out_pad << log2w;
    k_pack<<<grid_for(threads), kThreads, 0, s>>>(in, n_in, nodes + t.level_off[L], n_out_pad,
                                                  log2w);
    RTS_CUDA_TRY(cudaGetLastError());
  }
  // Root box and the spare entries 1..W-1 of the first group.
  k_pack<<<grid_for(static_cast<uint64_t>(W) << log2w), kThreads, 0, s>>>(
      nodes + t.level_off[t.top], t.level_cnt[t.top], nodes, W, log2w);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}


static int order_batch_bits(uint32_t nb, bool merged) {
  int bbits = 0;
  while (!merged && bbits < 32 && (1ull << bbits) < nb) ++bbits;
  return bbits;
}

int order_curve_bits(uint64_t total, uint32_t nb, bool merged) {
  int lg = 0;
  while (lg < 40 && (1ull << lg) < total) ++lg;
  int bits = 2 * std::min(16, (lg + 1) / 2 + 2);  // about 16 cells per query
  // (batch, curve) keys of an unmerged launch: fit them in three 8-bit radix
  // passes where that leaves at least 8 bits per axis (the curve orders
  // queries within their own batch, which holds a share of the total).
  const int bbits = order_batch_bits(nb, merged);
  if (bbits > 0 && bits + bbits > 24) bits = std::max(16, std::min(bits, (24 - bbits) & ~1));
  return bits;
}

static int order_end_bit(uint64_t total, uint32_t nb, bool merged) {
  return order_curve_bits(total, nb, merged) + order_batch_bits(nb, merged);
}

int launch_query_order(const BatchDesc* descs, const BatchDesc& b0, uint32_t nb, uint64_t total,
                       const float4* frame_box, int curve, unsigned long long* keys_a,
                       unsigned long long* keys_b, uint32_t* vals_a, uint32_t* order,
                       DevBuf& temp, cudaStream_t s, bool merged, void* merged_q,
                       uint32_t* merged_batch, uint32_t* merged_ident, DevQueue* merged_routes) {
  if (total == 0) return RTS_OK;
  merged = merged && nb > 1;
  k_query_keys<<<grid_for(total), kThreads, 0, s>>>(descs, b0, nb, total, frame_box, curve, keys_a,
                                                    vals_a, merged,
                                                    order_curve_bits(total, nb, merged));
  RTS_CUDA_TRY(cudaGetLastError());
  const int end_bit = order_end_bit(total, nb, merged);
  size_t need = 0;
  RTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, keys_a, keys_b, vals_a, order,
                                                static_cast<int>(total), 0, end_bit, s));
  int rc = buf_reserve(temp, need, s, false, 0);
  if (rc) return rc;
  RTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.ptr, need, keys_a, keys_b, vals_a, order,
                                                static_cast<int>(total), 0, end_bit, s));
  if (merged) {
    // nb <= total: every batch of a merged launch is non-empty
    k_merge_queries<<<grid_for(total), kThreads, 0, s>>>(descs, nb, total, order, merged_q,
                                                         merged_batch, merged_ident,
                                                         merged_routes);
    RTS_CUDA_TRY(cudaGetLastError());
  }
  return RTS_OK;
}

int launch_chunk_order(const BatchDesc* descs, uint32_t nb, uint32_t total_chunks, uint32_t chunk,
                       uint64_t total, const unsigned long long* sorted_keys, uint32_t* keys_a,
                       uint32_t* keys_b, uint32_t* vals_a, uint32_t* order, DevBuf& temp,
                       cudaStream_t s) {
  if (total_chunks == 0 || nb < 2) return RTS_OK;
  const int cbits = order_curve_bits(total, nb, false);  // as the unmerged query keys
  const uint32_t mask = cbits >= 32 ? 0xffffffffu : ((1u << cbits) - 1u);
  k_chunk_keys<<<grid_for(total_chunks), kThreads, 0, s>>>(descs, nb, total_chunks, chunk,
                                                           sorted_keys, mask, keys_a, vals_a);
  RTS_CUDA_TRY(cudaGetLastError());
  size_t need = 0;
  RTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, keys_a, keys_b, vals_a, order,
                                                static_cast<int>(total_chunks), 0, cbits, s));
  int rc = buf_reserve(temp, need, s, false, 0);
  if (rc) return rc;
  RTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.ptr, need, keys_a, keys_b, vals_a, order,
                                                static_cast<int>(total_chunks), 0, cbits, s));
  return RTS_OK;
}

int chunk_order_temp_bytes(uint32_t total_chunks, size_t* bytes) {
  *bytes = 0;
  RTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(
      nullptr, *bytes, static_cast<const uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
      static_cast<const uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
      static_cast<int>(total_chunks), 0, 32));
  return RTS_OK;
}

int query_order_temp_bytes(uint64_t total, uint32_t nb, size_t* bytes) {
  const int end_bit = order_end_bit(total, nb, false);  // a merged order uses fewer bits
  *bytes = 0;
  RTS_CUDA_TRY(cub::DeviceRadixSort::SortPairs(
      nullptr, *bytes, static_cast<const unsigned long long*>(nullptr),
      static_cast<unsigned long long*>(nullptr), static_cast<const uint32_t*>(nullptr),
      static_cast<uint32_t*>(nullptr), static_cast<int>(total), 0, end_bit));
  return RTS_OK;
}

int launch_delete(const uint64_t* ids, uint64_t n, uint64_t n_ids, const uint32_t* pos,
                  float4* leaves, cudaStream_t s, DBox* leaves64) {
  if (n == 0) return RTS_OK;
  k_delete<<<grid_for(n), kThreads, 0, s>>>(ids, n, n_ids, pos, leaves, leaves64);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}


template <typename E>
int launch_update_split_t(const E* upd, uint64_t n, uint64_t n_ids, const uint32_t* pos,
                          const UpdateTrees& T, uint64_t slot_end, float4* leaves, DBox* leaves64,
                          uint32_t* bits, uint32_t* moved_ids, float4* moved, DBox* moved64,
                          uint32_t* n_moved, cudaStream_t s) {
  const uint64_t words = (slot_end + 31) / 32;
  RTS_CUDA_TRY(cudaMemsetAsync(bits, 0, 2 * words * sizeof(uint32_t), s));
  RTS_CUDA_TRY(cudaMemsetAsync(n_moved, 0, sizeof(uint32_t), s));
  if (n == 0) return RTS_OK;
  k_update_mark<E><<<grid_for(n), kThreads, 0, s>>>(upd, n, n_ids, pos, T, bits);
  RTS_CUDA_TRY(cudaGetLastError());
  k_update_apply<E><<<grid_for(n), kThreads, 0, s>>>(upd, n, n_ids, pos, leaves, leaves64, bits,
                                                     bits + words, moved_ids, moved, moved64,
                                                     n_moved);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

int launch_update_split(const rts_update_entry* upd, uint64_t n, uint64_t n_ids,
                        const uint32_t* pos, const UpdateTrees& T, uint64_t slot_end,
                        float4* leaves, uint32_t* bits, uint32_t* moved_ids, float4* moved,
                        uint32_t* n_moved, cudaStream_t s) {
  return launch_update_split_t(upd, n, n_ids, pos, T, slot_end, leaves, nullptr, bits, moved_ids,
                               moved, nullptr, n_moved, s);
}

int launch_update_split64(const rts_update_entry_f64* upd, uint64_t n, uint64_t n_ids,
                          const uint32_t* pos, const UpdateTrees& T, uint64_t slot_end,
                          float4* leaves, DBox* leaves64, uint32_t* bits, uint32_t* moved_ids,
                          float4* moved, DBox* moved64, uint32_t* n_moved, cudaStream_t s) {
  return launch_update_split_t(upd, n, n_ids, pos, T, slot_end, leaves, leaves64, bits, moved_ids,
                               moved, moved64, n_moved, s);
}


int launch_round_boxes(const DBox* in, uint64_t n, float4* out, cudaStream_t s) {
  if (n == 0) return RTS_OK;
  k_round_boxes<<<grid_for(n), kThreads, 0, s>>>(in, n, out);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

}  // namespace rts
