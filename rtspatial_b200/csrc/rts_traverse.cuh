// Traversal of the implicit W-wide forest, one warp at a time.
//
// Two warp-level schemes over the same layout:
//  - thread: each lane owns one query and tests a whole group of W children
//    per step (W float4 loads, W predicate evaluations);
//  - team:   W lanes own one query and each tests one child per step (one
//    coalesced 16*W-byte load per team, a ballot builds the child mask).
// Both keep, per query, the child masks of every level on the way down
// (MaskStack) instead of a pointer stack: descending takes the lowest set bit
// of the current level's mask; ascending divides the group index by W.
//
// A warp works through a chunk [cbeg, cend) of one batch's queries.  Lanes
// (or teams) whose query is finished take the next unstarted query of the
// chunk at the end of each step (ballot + popc ranking), so the warp stays
// full while the chunk lasts even when per-query work is heavily skewed.
#pragma once

#include "rts_device.cuh"

namespace rts {

// Parameters of one batch (one reference Query call).
struct BatchDesc {
  const float* queries;
  void* arg;              // counter (count) or DevQueue* (collect)
  uint32_t n;             // queries in the batch
  int32_t pred;           // PredKind
  int32_t mode;           // HandlerKind
  uint32_t chunk_begin;   // index of the batch's first chunk in the launch
  const uint32_t* order;  // optional visiting order (query ids), or nullptr
  uint32_t qbase;         // offset of the batch in the launch's concatenated order
  uint32_t id_offset;     // added to every reported query id (0 for a Query call)
};

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <int PRED, int W>
struct TravState {
  typename QueryOps<PRED>::Q q;
  MaskStack<W> ms;
  uint32_t qid;   // id reported for this query
  uint32_t t;     // tree
  uint32_t L;     // level of the group being visited
  uint32_t g;     // group index at level L
};

// Starts query qid (visiting slot `slot` of the batch) at the top of tree 0.
// Returns false when the forest is empty.
template <int PRED, int W>
__device__ __forceinline__ bool trav_start(const Forest& F, const BatchDesc& B, uint32_t slot,
                                           TravState<PRED, W>& s, const uint32_t* only) {
  s.qid = B.order ? B.order[slot] : slot;
  if (only) {
    const uint32_t g = B.qbase + s.qid;
    if (!((__ldg(only + (g >> 5)) >> (g & 31)) & 1u)) return false;
  }
  s.q = QueryOps<PRED>::load(B.queries, s.qid);
  s.ms.clear();
  s.t = 0;
  if (F.n_trees == 0) return false;
  const TreeDesc& T = F.tree[0];
  s.L = T.top;
  s.g = 0;
  QueryOps<PRED>::enter_tree(s.q, __ldg(T.nodes));
  return true;
}

// After a group was visited: moves to the next group to visit.  Returns false
// when the query is finished in every tree.
template <int PRED, int W>
__device__ __forceinline__ bool trav_advance(const Forest& F, TravState<PRED, W>& s) {
  for (;;) {
    uint32_t top = F.tree[s.t].top;
    while (s.L == 0 || s.ms.get(s.L) == 0) {
      if (s.L == top) break;
      s.L += 1;
      s.g /= W;
    }
    if (s.L != 0 && s.ms.get(s.L) != 0) {
      uint32_t m = s.ms.get(s.L);
      uint32_t c = __ffs(m) - 1;
      s.ms.set(s.L, m & (m - 1));
      s.g = s.g * W + c;
      s.L -= 1;
      return true;
    }
    // This tree is exhausted: enter the next one at its top group.
    s.t += 1;
    if (s.t >= F.n_trees) return false;
    const TreeDesc& T = F.tree[s.t];
    s.ms.clear();
    s.L = T.top;
    s.g = 0;
    QueryOps<PRED>::enter_tree(s.q, __ldg(T.nodes));
    return true;
  }
}

// ---------------------------------------------------------------------------
// thread scheme
// ---------------------------------------------------------------------------
template <int PRED, int MODE, int W>
__device__ __forceinline__ void run_chunk_thread(const Forest& F, const BatchDesc& B,
                                                 uint32_t cbeg, uint32_t cend, DevPair* wbuf,
                                                 const uint32_t* only) {
  using Ops = QueryOps<PRED>;
  const uint32_t lane = lane_id();
  TravState<PRED, W> s;
  uint32_t next = cbeg;
  bool active = false;
  {
    uint32_t slot = next + lane;
    if (slot < cend) active = trav_start<PRED, W>(F, B, slot, s, only);
    next = min(cend, next + 32u);
  }
  DevQueue qu{};
  if (MODE == kCollect) qu = *static_cast<const DevQueue*>(B.arg);
  WarpOut out{wbuf, 0, F.ids_base};
  unsigned long long cnt = 0;

  for (;;) {
    if (!__any_sync(kFull, active)) {
      // Every lane is idle (with a query filter, refills can all be rejected):
      // refill again until the chunk is exhausted.
      if (next >= cend) break;
      uint32_t slot = next + lane;
      if (slot < cend) active = trav_start<PRED, W>(F, B, slot, s, only);
      next = min(cend, next + 32u);
      continue;
    }
    uint32_t leafm = 0;
    uint32_t leafslot = 0;
    if (active) {
      // One load-and-test path for leaves and nodes (no divergent copies).
      const TreeDesc& T = F.tree[s.t];
      const uint32_t first = s.g * W;
      const bool at_leaf = (s.L == 0);
      const float4* p = at_leaf ? T.leaves + first : T.nodes + T.level_off[s.L] + first;
      const uint32_t lim = (at_leaf ? T.n : T.level_cnt[s.L]) - first;
      float4 e[W];
#pragma unroll
      for (int c = 0; c < W; ++c) e[c] = __ldg(p + c);
      uint32_t m = 0;
#pragma unroll
      for (int c = 0; c < W; ++c)
        if (static_cast<uint32_t>(c) < lim && Ops::coarse(e[c], s.q)) m |= 1u << c;
      if (at_leaf) {
        if constexpr (Ops::kRefine) {
#pragma unroll
          for (int c = 0; c < W; ++c)
            if (((m >> c) & 1u) && !Ops::exact(e[c], s.q)) m &= ~(1u << c);
        }
        leafm = m;
        leafslot = static_cast<uint32_t>(T.ids - F.ids_base) + first;
      } else {
        s.ms.set(s.L, m);
      }
    }
    if (MODE == kCollect) {
      out.template add<W>(qu, leafm, leafslot, s.qid + B.id_offset);
    } else {
      cnt += __popc(leafm);
    }
    if (active) active = trav_advance<PRED, W>(F, s);
    // Refill finished lanes from the chunk.
    uint32_t idle = __ballot_sync(kFull, !active);
    if (idle != 0 && next < cend) {
      uint32_t slot = next + __popc(idle & lanemask_lt());
      if (!active && slot < cend) active = trav_start<PRED, W>(F, B, slot, s, only);
      next = min(cend, next + __popc(idle));
    }
  }
  if (MODE == kCollect) out.flush(qu);
  if (MODE == kCount) count_flush_warp(static_cast<unsigned long long*>(B.arg), cnt);
}

// ---------------------------------------------------------------------------
// team scheme: W lanes per query, 32 / W queries in flight per warp
// ---------------------------------------------------------------------------
template <int PRED, int MODE, int W>
__device__ __forceinline__ void run_chunk_team(const Forest& F, const BatchDesc& B,
                                               uint32_t cbeg, uint32_t cend, DevPair* wbuf,
                                               const uint32_t* only) {
  using Ops = QueryOps<PRED>;
  constexpr uint32_t kTeams = 32 / W;
  constexpr uint32_t kTeamMask = (W == 32) ? kFull : ((1u << W) - 1u);
  const uint32_t lane = lane_id();
  const uint32_t team = lane / W;
  const uint32_t tl = lane % W;
  TravState<PRED, W> s;
  uint32_t next = cbeg;
  bool active = false;
  {
    uint32_t slot = next + team;
    if (slot < cend) active = trav_start<PRED, W>(F, B, slot, s, only);
    next = min(cend, next + kTeams);
  }
  DevQueue qu{};
  if (MODE == kCollect) qu = *static_cast<const DevQueue*>(B.arg);
  WarpOut out{wbuf, 0, F.ids_base};
  unsigned long long cnt = 0;

  for (;;) {
    if (!__any_sync(kFull, active)) {
      if (next >= cend) break;  // see run_chunk_thread
      uint32_t slot = next + team;
      if (slot < cend) active = trav_start<PRED, W>(F, B, slot, s, only);
      next = min(cend, next + kTeams);
      continue;
    }
    bool hit = false, leaf_hit = false;
    uint32_t gid = 0;
    if (active) {
      const TreeDesc& T = F.tree[s.t];
      const uint32_t first = s.g * W;
      if (s.L == 0) {
        float4 e = __ldg(T.leaves + first + tl);
        hit = (first + tl < T.n) && Ops::leaf(e, s.q);
        leaf_hit = hit;
        if (leaf_hit) gid = static_cast<uint32_t>(T.ids - F.ids_base) + first + tl;
      } else {
        float4 e = __ldg(T.nodes + T.level_off[s.L] + first + tl);
        hit = (first + tl < T.level_cnt[s.L]) && Ops::node(e, s.q);
      }
    }
    const uint32_t bal = __ballot_sync(kFull, hit);
    if (MODE == kCollect) {
      out.add_one(qu, leaf_hit, gid, s.qid + B.id_offset);
    } else {
      cnt += leaf_hit ? 1u : 0u;
    }
    if (active) {
      if (s.L != 0) s.ms.set(s.L, (bal >> (team * W)) & kTeamMask);
      active = trav_advance<PRED, W>(F, s);
    }
    // Refill finished teams from the chunk (all lanes of a team agree).
    uint32_t idle = __ballot_sync(kFull, !active);
    if (idle != 0 && next < cend) {
      uint32_t below = (team == 0) ? 0u : (idle & ((1u << (team * W)) - 1u));
      uint32_t slot = next + __popc(below) / W;
      if (!active && slot < cend) active = trav_start<PRED, W>(F, B, slot, s, only);
      next = min(cend, next + __popc(idle) / W);
    }
  }
  if (MODE == kCollect) out.flush(qu);
  if (MODE == kCount) count_flush_warp(static_cast<unsigned long long*>(B.arg), cnt);
}

}  // namespace rts
