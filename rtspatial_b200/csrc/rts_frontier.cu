// Breadth-first ("frontier") traversal for large batched range queries.
//
// The depth-first kernel keeps one query per lane and walks it to the end;
// its lanes diverge and each step waits on one dependent node load.  For
// large launches this path instead processes the whole launch level by level:
// the frontier of a level is a list of (query, group) entries, and one
// grid-stride kernel tests every child of every entry (one thread per child:
// no per-query state, no divergence, W consecutive 16-byte loads per entry).
// Hits of a level become the next level's frontier; hits at the leaves are
// emitted.  Outputs are staged per block in shared memory (one global atomic
// per tile of 4096 tests); at the leaves the staged pairs are grouped by batch
// through a small shared-memory table so that each batch's queue takes one
// atomic per tile.
//
// Frontier buffers have a fixed capacity.  An entry that does not fit marks
// its query as spilled (bitmap): the leaf kernel emits nothing for spilled
// queries and a depth-first pass answers exactly those queries afterwards, so
// results are exact whatever the capacity.
#include <algorithm>

#include "rts_internal.h"

namespace rts {
namespace {

constexpr int kFrThreads = 256;
constexpr int kFrIter = 16;
constexpr uint32_t kFrTile = kFrThreads * kFrIter;
constexpr int kBatchSlots = 8;

// A frontier entry: query index in the launch and (sub-tree << 28 | group).
struct FrEntry {
  uint32_t g;
  uint32_t tg;
};
constexpr uint32_t kGroupBits = 28;
constexpr uint32_t kGroupMask = (1u << kGroupBits) - 1u;

__device__ __forceinline__ uint32_t batch_of(const BatchDesc* descs, uint32_t nb, uint32_t g) {
  if (nb <= 1) return 0;
  uint32_t lo = 0, hi = nb - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (__ldg(&descs[mid].qbase) <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ bool spilled(const uint32_t* spill, uint32_t g) {
  return (__ldg(spill + (g >> 5)) >> (g & 31)) & 1u;
}

// Node test against the launch copy of a query (points stored as (x,y,x,y)).
template <int PRED>
__device__ __forceinline__ bool fr_node(float4 e, float4 q, float2 mag) {
  if constexpr (PRED == kPoint) {
    return contains_point(e, make_float2(q.x, q.y));
  } else if constexpr (PRED == kContains) {
    return contains_box(e, q);
  } else {
    IsectQuery Q;
    Q.q = q;
    isect_set_margin(Q, mag);
    return overlaps(e, Q.nb);
  }
}

// Exact leaf predicate.  aux = (origin.x, origin.y, 1/dx, 1/dy) of the
// query's anti-diagonal ray, precomputed once per query.
template <int PRED>
__device__ __forceinline__ bool fr_leaf(float4 g, float4 q, float4 aux, float2 mag) {
  if constexpr (PRED == kPoint) {
    return contains_point(g, make_float2(q.x, q.y));
  } else if constexpr (PRED == kContains) {
    return contains_box(g, q);
  } else {
    IsectQuery Q;
    Q.q = q;
    Q.ox = aux.x;
    Q.oy = aux.y;
    Q.invx = aux.z;
    Q.invy = aux.w;
    isect_set_margin(Q, mag);
    return isect_leaf(g, Q);
  }
}

__device__ __forceinline__ void load_forest(Forest& dst, const Forest& src) {
  const uint32_t* a = reinterpret_cast<const uint32_t*>(&src);
  uint32_t* b = reinterpret_cast<uint32_t*>(&dst);
  for (uint32_t i = threadIdx.x; i < sizeof(Forest) / 4; i += blockDim.x) b[i] = a[i];
  __syncthreads();
}

// Copies the launch's queries into the frontier's query buffer and writes
// the visiting order vis[i] = launch index of the i-th query visited.
template <int PRED>
__global__ void k_fr_init(const BatchDesc* __restrict__ descs, const BatchDesc b0, uint32_t nb,
                          uint32_t total, float4* __restrict__ qbuf, float4* __restrict__ qaux,
                          uint32_t* __restrict__ qbatch, uint32_t* __restrict__ vis) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += gridDim.x * blockDim.x) {
    const uint32_t b = batch_of(descs, nb, i);
    const BatchDesc& B = (nb > 1) ? descs[b] : b0;
    const uint32_t local = B.order ? B.order[i - B.qbase] : (i - B.qbase);
    const uint32_t g = B.qbase + local;
    float4 q;
    if constexpr (PRED == kPoint) {
      float2 p = reinterpret_cast<const float2*>(B.queries)[local];
      q = make_float4(p.x, p.y, p.x, p.y);
    } else {
      q = reinterpret_cast<const float4*>(B.queries)[local];
    }
    qbuf[g] = q;
    qbatch[g] = b;
    if constexpr (PRED == kIntersects) {
      IsectQuery Q = make_isect_query(q);
      qaux[g] = make_float4(Q.ox, Q.oy, Q.invx, Q.invy);
    }
    vis[i] = g;
  }
}

// Level L of every sub-tree at once (sub-trees aligned at their leaves):
// tests the W children of every entry; hits form the frontier of level L-1.
// Entries [0, nin) come from level L+1; the entries after them are implicit:
// every query at group 0 of each sub-tree whose top level is L (start_mask).
template <int PRED, int W>
__global__ void __launch_bounds__(kFrThreads)
    k_fr_expand(const __grid_constant__ Forest Fp, uint32_t L, uint32_t start_mask,
                const FrEntry* __restrict__ fin, const uint32_t* __restrict__ nin_p,
                FrEntry* __restrict__ fout, uint32_t* __restrict__ nout_p, uint32_t cap,
                const float4* __restrict__ qbuf, const uint32_t* __restrict__ vis, uint32_t total,
                uint32_t* __restrict__ spill, uint32_t* __restrict__ any_spill) {
  __shared__ Forest F;
  __shared__ FrEntry stage[kFrTile];
  __shared__ uint32_t s_count, s_base;
  load_forest(F, Fp);
  const uint32_t nin = nin_p ? min(*nin_p, cap) : 0;
  const uint32_t n_start = __popc(start_mask);
  const uint64_t entries = static_cast<uint64_t>(nin) + static_cast<uint64_t>(n_start) * total;
  const uint64_t work = entries * W;
  const uint32_t lane = lane_id();
  for (uint64_t tile = blockIdx.x; tile * kFrTile < work; tile += gridDim.x) {
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < kFrIter; ++k) {
      const uint64_t idx = tile * kFrTile + static_cast<uint64_t>(k) * kFrThreads + threadIdx.x;
      bool hit = false;
      FrEntry o{0, 0};
      if (idx < work) {
        const uint64_t e = idx / W;
        FrEntry fe;
        if (e < nin) {
          fe = fin[e];
        } else {
          const uint64_t r = e - nin;
          uint32_t k_tree = static_cast<uint32_t>(r / total), m = start_mask, t = 0;
          for (;;) {  // k_tree-th set bit of start_mask
            t = __ffs(m) - 1;
            if (k_tree == 0) break;
            m &= m - 1;
            --k_tree;
          }
          fe = FrEntry{__ldg(vis + (r % total)), t << kGroupBits};
        }
        const uint32_t t = fe.tg >> kGroupBits;
        const TreeDesc& T = F.tree[t];
        const uint32_t child = (fe.tg & kGroupMask) * W + static_cast<uint32_t>(idx % W);
        if (child < T.level_cnt[L]) {
          hit = fr_node<PRED>(__ldg(T.nodes + T.level_off[L] + child), __ldg(qbuf + fe.g),
                              root_magnitude(T.nodes[0]));
          o = FrEntry{fe.g, (t << kGroupBits) | child};
        }
      }
      const uint32_t bal = __ballot_sync(kFull, hit);
      uint32_t wb = 0;
      if (lane == 0 && bal) wb = atomicAdd(&s_count, static_cast<uint32_t>(__popc(bal)));
      wb = __shfl_sync(kFull, wb, 0);
      if (hit) stage[wb + __popc(bal & lanemask_lt())] = o;
    }
    __syncthreads();
    const uint32_t cnt = s_count;
    if (threadIdx.x == 0) s_base = cnt ? atomicAdd(nout_p, cnt) : 0;
    __syncthreads();
    const uint32_t base = s_base;
    for (uint32_t i = threadIdx.x; i < cnt; i += kFrThreads) {
      const uint64_t pos = static_cast<uint64_t>(base) + i;
      if (pos < cap) {
        fout[pos] = stage[i];
      } else {
        const uint32_t g = stage[i].g;
        atomicOr(spill + (g >> 5), 1u << (g & 31));
        *any_spill = 1u;
      }
    }
    __syncthreads();
  }
}

// Leaves of every sub-tree: exact tests of the W boxes of every entry's leaf
// group; pairs of queries that did not spill go to their batch's handler.
// Runs after every expansion, so a spilled query emits nothing here.
template <int PRED, int MODE, int W>
__global__ void __launch_bounds__(kFrThreads)
    k_fr_leaves(const __grid_constant__ Forest Fp, const FrEntry* __restrict__ fin,
                const uint32_t* __restrict__ nin_p, uint32_t cap, const float4* __restrict__ qbuf,
                const float4* __restrict__ qaux, const uint32_t* __restrict__ qbatch,
                const BatchDesc* __restrict__ descs, const BatchDesc b0, uint32_t nb,
                const uint32_t* __restrict__ spill) {
  __shared__ Forest F;
  __shared__ uint2 stage[kFrTile];  // (geom id, query index g)
  __shared__ uint32_t s_count;
  __shared__ uint32_t s_key[kBatchSlots];
  __shared__ uint32_t s_num[kBatchSlots];
  __shared__ uint32_t s_base[kBatchSlots];
  load_forest(F, Fp);
  const uint32_t nin = min(*nin_p, cap);
  const uint64_t work = static_cast<uint64_t>(nin) * W;
  const uint32_t lane = lane_id();
  for (uint64_t tile = blockIdx.x; tile * kFrTile < work; tile += gridDim.x) {
    if (threadIdx.x == 0) s_count = 0;
    if (threadIdx.x < kBatchSlots) {
      s_key[threadIdx.x] = 0xffffffffu;
      s_num[threadIdx.x] = 0;
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < kFrIter; ++k) {
      const uint64_t idx = tile * kFrTile + static_cast<uint64_t>(k) * kFrThreads + threadIdx.x;
      bool hit = false;
      uint2 o = make_uint2(0, 0);
      if (idx < work) {
        const FrEntry fe = fin[idx / W];
        const TreeDesc& T = F.tree[fe.tg >> kGroupBits];
        const uint32_t slot = (fe.tg & kGroupMask) * W + static_cast<uint32_t>(idx % W);
        if (slot < T.n && !spilled(spill, fe.g)) {
          float4 aux = make_float4(0.f, 0.f, 0.f, 0.f);
          if constexpr (PRED == kIntersects) aux = __ldg(qaux + fe.g);
          hit = fr_leaf<PRED>(__ldg(T.leaves + slot), __ldg(qbuf + fe.g), aux,
                              root_magnitude(T.nodes[0]));
          if (hit) o = make_uint2(__ldg(T.ids + slot), fe.g);
        }
      }
      const uint32_t bal = __ballot_sync(kFull, hit);
      uint32_t wb = 0;
      if (lane == 0 && bal) wb = atomicAdd(&s_count, static_cast<uint32_t>(__popc(bal)));
      wb = __shfl_sync(kFull, wb, 0);
      if (hit) stage[wb + __popc(bal & lanemask_lt())] = o;
    }
    __syncthreads();
    const uint32_t cnt = s_count;
    // Group the staged pairs by batch: each pair claims a slot of the small
    // table for its batch (linear probing) and its rank within the batch.
    uint32_t my_slot[kFrIter];
    uint32_t my_rank[kFrIter];
#pragma unroll
    for (int j = 0; j < kFrIter; ++j) {
      const uint32_t i = threadIdx.x + j * kFrThreads;
      my_slot[j] = kBatchSlots;
      my_rank[j] = 0;
      if (i < cnt) {
        const uint32_t b = __ldg(qbatch + stage[i].y);
        for (int t = 0; t < kBatchSlots; ++t) {
          const int sl = static_cast<int>((b + t) % kBatchSlots);
          const uint32_t prev = atomicCAS(&s_key[sl], 0xffffffffu, b);
          if (prev == 0xffffffffu || prev == b) {
            my_slot[j] = sl;
            my_rank[j] = atomicAdd(&s_num[sl], 1u);
            break;
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x < kBatchSlots && s_num[threadIdx.x]) {
      const uint32_t b = s_key[threadIdx.x];
      const BatchDesc& B = (nb > 1) ? descs[b] : b0;
      if (MODE == kCollect) {
        s_base[threadIdx.x] =
            atomicAdd(static_cast<const DevQueue*>(B.arg)->size, s_num[threadIdx.x]);
      } else {
        atomicAdd(static_cast<unsigned long long*>(B.arg),
                  static_cast<unsigned long long>(s_num[threadIdx.x]));
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kFrIter; ++j) {
      const uint32_t i = threadIdx.x + j * kFrThreads;
      if (i >= cnt) continue;
      if (MODE == kCount && my_slot[j] < kBatchSlots) continue;
      const uint2 pr = stage[i];
      const uint32_t b = __ldg(qbatch + pr.y);
      const BatchDesc& B = (nb > 1) ? descs[b] : b0;
      if (my_slot[j] < kBatchSlots) {
        const DevQueue* qu = static_cast<const DevQueue*>(B.arg);
        const unsigned long long p =
            static_cast<unsigned long long>(s_base[my_slot[j]]) + my_rank[j];
        if (p < qu->capacity) qu->data[p] = DevPair{pr.x, pr.y - B.qbase + B.id_offset};
      } else if (MODE == kCollect) {  // more batches in the tile than table slots
        const DevQueue* qu = static_cast<const DevQueue*>(B.arg);
        const unsigned long long p = atomicAdd(qu->size, 1u);
        if (p < qu->capacity) qu->data[p] = DevPair{pr.x, pr.y - B.qbase + B.id_offset};
      } else {
        atomicAdd(static_cast<unsigned long long*>(B.arg), 1ull);
      }
    }
    __syncthreads();
  }
}

template <int PRED, int MODE, int W>
int launch_levels(const Forest& F, const BatchDesc* dd, const BatchDesc& b0, uint32_t nb,
                  uint32_t total, const FrontierBufs& fb, int grid, cudaStream_t s) {
  uint32_t max_top = 0;
  for (uint32_t t = 0; t < F.n_trees; ++t) max_top = max(max_top, F.tree[t].top);
  auto* bufs = reinterpret_cast<FrEntry*>(fb.fa);
  FrEntry* fbuf[2] = {static_cast<FrEntry*>(fb.fa), static_cast<FrEntry*>(fb.fb)};
  (void)bufs;
  const FrEntry* in = nullptr;
  const uint32_t* nin = nullptr;
  int flip = 0;
  for (uint32_t L = max_top; L >= 1; --L) {
    uint32_t start_mask = 0;
    for (uint32_t t = 0; t < F.n_trees; ++t)
      if (F.tree[t].top == L) start_mask |= 1u << t;
    FrEntry* out = fbuf[flip];
    uint32_t* nout = fb.counts + L;
    k_fr_expand<PRED, W><<<grid, kFrThreads, 0, s>>>(
        F, L, start_mask, in, nin, out, nout, fb.cap, static_cast<const float4*>(fb.qbuf),
        fb.vis, total, fb.spill, fb.any_spill);
    RTS_CUDA_TRY(cudaGetLastError());
    in = out;
    nin = nout;
    flip ^= 1;
  }
  k_fr_leaves<PRED, MODE, W><<<grid, kFrThreads, 0, s>>>(
      F, in, nin, fb.cap, static_cast<const float4*>(fb.qbuf), static_cast<const float4*>(fb.qaux),
      fb.qbatch, dd, b0, nb, fb.spill);
  RTS_CUDA_TRY(cudaGetLastError());
  return RTS_OK;
}

template <int PRED, int MODE>
int launch_levels_w(const Forest& F, const BatchDesc* dd, const BatchDesc& b0, uint32_t nb,
                    uint32_t total, const FrontierBufs& fb, int grid, cudaStream_t s) {
  switch (F.width) {
    case 4: return launch_levels<PRED, MODE, 4>(F, dd, b0, nb, total, fb, grid, s);
    case 8: return launch_levels<PRED, MODE, 8>(F, dd, b0, nb, total, fb, grid, s);
    case 16: return launch_levels<PRED, MODE, 16>(F, dd, b0, nb, total, fb, grid, s);
    default: return launch_levels<PRED, MODE, 32>(F, dd, b0, nb, total, fb, grid, s);
  }
}

}  // namespace

size_t frontier_counts_needed(const Forest& F) {
  uint32_t max_top = 0;
  for (uint32_t t = 0; t < F.n_trees; ++t) max_top = std::max(max_top, F.tree[t].top);
  return static_cast<size_t>(max_top) + 1;
}

int launch_frontier(const Forest& F, int pred, int mode, const BatchDesc* hb, const BatchDesc* dd,
                    uint32_t nb, uint32_t total, const FrontierBufs& fb, cudaStream_t s) {
  if (total == 0 || F.n_trees == 0) return RTS_OK;
  const size_t ncounts = frontier_counts_needed(F);
  if (ncounts > fb.counts_cap) return fail(RTS_ERR_CAPACITY, "frontier counter array too small");
  RTS_CUDA_TRY(cudaMemsetAsync(fb.counts, 0, ncounts * sizeof(uint32_t), s));
  RTS_CUDA_TRY(cudaMemsetAsync(fb.spill, 0, ((total + 31) / 32) * sizeof(uint32_t), s));
  RTS_CUDA_TRY(cudaMemsetAsync(fb.any_spill, 0, sizeof(uint32_t), s));
  const int grid = device_sm_count() * 4;
  const unsigned ig = static_cast<unsigned>(std::min<uint64_t>((total + 255) / 256, 148 * 32));
  const BatchDesc& b0 = hb[0];
  auto* qb = static_cast<float4*>(fb.qbuf);
  auto* qa = static_cast<float4*>(fb.qaux);
  switch (pred) {
    case kPoint: k_fr_init<kPoint><<<ig, 256, 0, s>>>(dd, b0, nb, total, qb, qa, fb.qbatch, fb.vis); break;
    case kContains: k_fr_init<kContains><<<ig, 256, 0, s>>>(dd, b0, nb, total, qb, qa, fb.qbatch, fb.vis); break;
    default: k_fr_init<kIntersects><<<ig, 256, 0, s>>>(dd, b0, nb, total, qb, qa, fb.qbatch, fb.vis);
  }
  RTS_CUDA_TRY(cudaGetLastError());
  const int grid_ = grid;
  switch (pred * 2 + mode) {
    case kPoint * 2 + kCount: return launch_levels_w<kPoint, kCount>(F, dd, b0, nb, total, fb, grid_, s);
    case kPoint * 2 + kCollect: return launch_levels_w<kPoint, kCollect>(F, dd, b0, nb, total, fb, grid_, s);
    case kContains * 2 + kCount: return launch_levels_w<kContains, kCount>(F, dd, b0, nb, total, fb, grid_, s);
    case kContains * 2 + kCollect: return launch_levels_w<kContains, kCollect>(F, dd, b0, nb, total, fb, grid_, s);
    case kIntersects * 2 + kCount: return launch_levels_w<kIntersects, kCount>(F, dd, b0, nb, total, fb, grid_, s);
    default: return launch_levels_w<kIntersects, kCollect>(F, dd, b0, nb, total, fb, grid_, s);
  }
}

}  // namespace rts
