// Traversal of the implicit W-wide forest, one warp at a time.
//
// Warp-level schemes over the same layout:
//  - thread: each lane owns one query and tests a whole group of W children
//    per step (W float4 loads, W predicate evaluations);
//  - staged: the thread scheme with each group bulk-copied into shared memory;
//  - team:   W lanes own one query and each tests one child per step (one
//    coalesced 16*W-byte load per team, a ballot builds the child mask);
//  - packet: one warp walks up to 32 queries together, one entry per lane.
// All keep, per query (or packet), the child masks of every level on the way
// down (MaskStack) instead of a pointer stack: descending takes the lowest set
// bit of the current level's mask; ascending divides the group index by W.
//
// A warp works through a chunk [cbeg, cend) of one batch's queries.  Lanes
// (or teams) whose query is finished take the next unstarted query of the
// chunk at the end of each step (ballot + popc ranking), so the warp stays
// full while the chunk lasts even when per-query work is heavily skewed.
// In a merged launch (MergedOrder) the batch is the launch's sorted query
// array and results are routed to each query's own batch.
#pragma once

#include "rts_device.cuh"

namespace rts {

// ceil of a lane that walks a whole query (every sub-tree of the forest).
constexpr uint32_t kWholeQuery = 0xffffffffu;

template <int PRED, int W>
struct TravState {
  typename QueryOps<PRED>::Q q;
  MaskStack<W> ms;
  uint32_t qid;   // id reported for this query (merged launch: sorted position)
  uint32_t rb;    // merged launch: the query's batch
  uint32_t t;     // tree
  uint32_t L;     // level of the group being visited
  uint32_t g;     // group index at level L
  uint32_t ceil;  // kWholeQuery, or the top level of a sub-tree taken over from
                  // another lane (walked alone: no climb above it, no next tree)
};

// Starts query qid (visiting slot `slot` of the batch) at the top of tree 0.
// Returns false when the forest is empty.
template <int PRED, int W, bool ROUTED>
__device__ __forceinline__ bool trav_start(const Forest& F, const BatchDesc& B, uint32_t slot,
                                           TravState<PRED, W>& s, const uint32_t* only,
                                           const MergedOrder& M) {
  s.qid = B.order ? B.order[slot] : slot;
  s.rb = ROUTED ? __ldg(M.batch + slot) : 0u;
  if (only) {
    const uint32_t g = B.qbase + s.qid;
    if (!((__ldg(only + (g >> 5)) >> (g & 31)) & 1u)) return false;
  }
  s.q = QueryOps<PRED>::load(B.queries, s.qid);
  s.ms.clear();
  s.t = 0;
  s.ceil = kWholeQuery;
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
    const bool whole = s.ceil == kWholeQuery;
    uint32_t top = whole ? F.tree[s.t].top : s.ceil;
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
    if (!whole) return false;  // a taken-over sub-tree is done
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

// Work sharing (warp-collective).  Per-query work is heavily skewed (a query
// in a dense cluster walks ten times the groups of a typical one), so once a
// chunk has no unstarted query, lanes whose queries finished would idle until
// the slowest query of the warp ends.  Instead the k-th idle lane takes over
// one pending entry of the k-th lane that still has some: the donor clears
// the highest bit of its mask stack (an entry of its shallowest pending level,
// the largest sub-tree it has left) and the receiver walks that entry's
// sub-tree alone (ceil = its top level).  The pairs are the same, found by
// another lane of the same warp, with the same query id and batch.
template <int PRED, int W>
__device__ __forceinline__ void share_work(TravState<PRED, W>& s, bool& active) {
  const uint32_t idle = __ballot_sync(kFull, !active);
  if (idle == 0) return;
  const uint32_t donors = __ballot_sync(kFull, active && s.ms.any());
  if (donors == 0) return;
  const uint32_t lane = lane_id();
  const uint32_t lt = lanemask_lt();
  const uint32_t k = min(__popc(idle), __popc(donors));
  uint32_t give_l = 0, give_g = 0;
  if (((donors >> lane) & 1u) && static_cast<uint32_t>(__popc(donors & lt)) < k) {
    const uint32_t p = static_cast<uint32_t>(s.ms.pop_highest());
    const uint32_t lp = p / W + 1;  // level of the pending entry (> s.L)
    const uint32_t gp = s.g >> (log2_width<W>() * (lp - s.L));  // its group, on this lane's path
    give_l = lp - 1;
    give_g = gp * W + (p % W);
  }
  const uint32_t irank = __popc(idle & lt);
  const bool take = !active && irank < k;
  uint32_t src = lane;
  if (take) {  // the irank-th donor
    uint32_t m = donors;
    for (uint32_t j = 0; j < irank; ++j) m &= m - 1;
    src = __ffs(m) - 1;
  }
  const auto q = shfl_words(s.q, static_cast<int>(src));
  const uint32_t qid = __shfl_sync(kFull, s.qid, src);
  const uint32_t rb = __shfl_sync(kFull, s.rb, src);
  const uint32_t t = __shfl_sync(kFull, s.t, src);
  const uint32_t gl = __shfl_sync(kFull, give_l, src);
  const uint32_t gg = __shfl_sync(kFull, give_g, src);
  if (take) {
    s.q = q;
    s.qid = qid;
    s.rb = rb;
    s.t = t;
    s.L = gl;
    s.g = gg;
    s.ceil = gl;
    s.ms.clear();
    active = true;
  }
}

// ---------------------------------------------------------------------------
// thread scheme
// ---------------------------------------------------------------------------
// MODE kUser: H::call<PRED>(geom_id, query_id, arg) once per pair, the
// reference's per-hit handler contract (ROUTED false).
template <int PRED, int MODE, int W, bool ROUTED, class H = NoUserHandler, bool SHARE = true>
__device__ __forceinline__ void run_chunk_thread(const Forest& F, const BatchDesc& B,
                                                 uint32_t cbeg, uint32_t cend, DevPair* wbuf, uint32_t* wbat,
                                                 const uint32_t* only,
                                                 const MergedOrder& M) {
  using Ops = QueryOps<PRED>;
  const uint32_t lane = lane_id();
  TravState<PRED, W> s;
  uint32_t next = cbeg;
  bool active = false;
  {
    uint32_t slot = next + lane;
    if (slot < cend) active = trav_start<PRED, W, ROUTED>(F, B, slot, s, only, M);
    next = min(cend, next + 32u);
  }
  DevQueue qu{};
  if (MODE == kCollect && !ROUTED) qu = *static_cast<const DevQueue*>(B.arg);
  WarpOut<ROUTED> out(wbuf, wbat, F.ids_base, M);
  unsigned long long cnt = 0;

  for (;;) {
    if (!__any_sync(kFull, active)) {
      // Every lane is idle (with a query filter, refills can all be rejected):
      // refill again until the chunk is exhausted.
      if (next >= cend) break;
      uint32_t slot = next + lane;
      if (slot < cend) active = trav_start<PRED, W, ROUTED>(F, B, slot, s, only, M);
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
      if (MODE == kCount ? F.stream_count : F.stream_collect) {  // the same for every lane
#pragma unroll
        for (int c = 0; c < W; c += 2) ldg_box_pair_stream(p + c, e[c], e[c + 1]);
      } else {
#pragma unroll
        for (int c = 0; c < W; c += 2) ldg_box_pair(p + c, e[c], e[c + 1]);
      }
      uint32_t m = 0;
#pragma unroll
      for (int c = 0; c < W; ++c)
        if (static_cast<uint32_t>(c) < lim && Ops::coarse(e[c], s.q)) m |= 1u << c;
      if (at_leaf) {
        if constexpr (Ops::kNeeds64) {  // exact test on the slots' double envelopes
          const DBox* p64 = T.leaves64 + first;
#pragma unroll
          for (int c = 0; c < W; ++c)
            if (((m >> c) & 1u) && !Ops::exact64(load_dbox(p64 + c), s.q)) m &= ~(1u << c);
        } else if constexpr (Ops::kRefine) {
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
    if constexpr (MODE == kCollect) {
      out.template add<W>(qu, leafm, leafslot, s.qid + B.id_offset, s.rb);
    } else if constexpr (MODE == kUser) {
      for (uint32_t m = leafm; m; m &= m - 1) {
        const uint32_t c = __ffs(m) - 1;
        H::template call<PRED>(__ldg(F.ids_base + leafslot + c), s.qid + B.id_offset, B.arg);
      }
    } else {
      cnt += __popc(leafm);
    }
    if (active) {
      active = trav_advance<PRED, W>(F, s);
      if (MODE == kCount && ROUTED && !active) {
        count_routed(M, s.rb, cnt);
        cnt = 0;
      }
    }
    // Refill finished lanes from the chunk, then share the rest of the work.
    uint32_t idle = __ballot_sync(kFull, !active);
    if (idle != 0 && next < cend) {
      uint32_t slot = next + __popc(idle & lanemask_lt());
      if (!active && slot < cend) active = trav_start<PRED, W, ROUTED>(F, B, slot, s, only, M);
      next = min(cend, next + __popc(idle));
    }
    if (SHARE && next >= cend) share_work<PRED, W>(s, active);
  }
  if constexpr (MODE == kCollect) out.flush(qu);
  if constexpr (MODE == kCount && !ROUTED)
    count_flush_warp(static_cast<unsigned long long*>(B.arg), cnt);
}

// ---------------------------------------------------------------------------
// staged scheme: the thread scheme with every group moved into shared memory
// by the copy engine
// ---------------------------------------------------------------------------
// Each lane still owns one query and visits one W-group per step, but the
// group's boxes (and, at a leaf group, its W geom ids) are not loaded into
// registers: the lane issues cp.async.bulk copies into its own slot of the
// warp's shared-memory area, all lanes arrive on the warp's mbarrier (the
// active ones announcing their bytes), and after the wait each lane tests the
// W boxes from shared memory one at a time.  So the group holds no registers
// while it is in flight (the thread scheme's W float4 are its register
// ceiling), the bytes bypass L1, and hits are staged with their geom ids
// already read, so the output flush issues no id loads.  Reads start at the
// lane's rotation (c + lane) mod W: a quarter-warp of lanes then reads eight
// different 16-byte bank groups of their slots.  Results, visiting order and
// output contract are those of the thread scheme.  Node width W <= 16.
template <int W>
struct StageWarp {
  float4 grp[32][W];     // each lane's current group
  uint32_t sid[32][W];   // each lane's leaf ids (leaf steps)
  unsigned long long bar;  // mbarrier: 32 arrivals per phase plus the copies' bytes
  uint32_t phase;          // parity of the phase the next wait completes
  uint32_t pad;
};

template <int PRED, int MODE, int W, bool ROUTED>
__device__ __forceinline__ bool run_chunk_staged(const Forest& F, const BatchDesc& B,
                                                 uint32_t cbeg, uint32_t cend, DevPair* wbuf,
                                                 uint32_t* wbat, const uint32_t* only,
                                                 const MergedOrder& M, StageWarp<W>& S) {
  static_assert(W <= 16, "a staged lane slot holds at most 16 boxes");
  using Ops = QueryOps<PRED>;
  const uint32_t lane = lane_id();
  const uint32_t bar = smem_u32(&S.bar);
  const uint32_t grp_dst = smem_u32(&S.grp[lane][0]);
  const uint32_t sid_dst = smem_u32(&S.sid[lane][0]);
  uint32_t phase = S.phase;
  TravState<PRED, W> s;
  uint32_t next = cbeg;
  bool active = false;
  {
    uint32_t slot = next + lane;
    if (slot < cend) active = trav_start<PRED, W, ROUTED>(F, B, slot, s, only, M);
    next = min(cend, next + 32u);
  }
  DevQueue qu{};
  if (MODE == kCollect && !ROUTED) qu = *static_cast<const DevQueue*>(B.arg);
  WarpOut<ROUTED, true> out(wbuf, wbat, F.ids_base, M);
  unsigned long long cnt = 0;
  bool ok = true;

  for (;;) {
    if (!__any_sync(kFull, active)) {
      if (next >= cend) break;  // see run_chunk_thread
      uint32_t slot = next + lane;
      if (slot < cend) active = trav_start<PRED, W, ROUTED>(F, B, slot, s, only, M);
      next = min(cend, next + 32u);
      continue;
    }
    // Issue this step's copies.  The fence orders the lane's reads of its
    // slot in the previous step before the copy engine overwrites it.
    uint32_t first = 0, lim = 0;
    bool at_leaf = false;
    fence_proxy_async_smem();
    if (active) {
      const TreeDesc& T = F.tree[s.t];
      first = s.g * W;
      at_leaf = (s.L == 0);
      const float4* p = at_leaf ? T.leaves + first : T.nodes + T.level_off[s.L] + first;
      lim = (at_leaf ? T.n : T.level_cnt[s.L]) - first;
      mbar_arrive_tx(bar, at_leaf ? W * 20u : W * 16u);
      bulk_copy_g2s(grp_dst, p, W * 16u, bar);
      if (at_leaf) bulk_copy_g2s(sid_dst, T.ids + first, W * 4u, bar);
    } else {
      mbar_arrive(bar);
    }
    {  // bounded wait for the phase: every lane arrived, every byte landed
      uint32_t spins = 0;
      bool done = false;
      while (!(done = mbar_try_wait(bar, phase)) && ++spins < kWaitSpinLimit) {
      }
      if (!__all_sync(kFull, done)) {
        if (lane == 0 && F.err) atomicOr(F.err, kErrWaitTimeout);
        // give the copies in flight a second bounded wait before leaving
        spins = 0;
        while (!mbar_try_wait(bar, phase) && ++spins < kWaitSpinLimit) {
        }
        ok = false;
        break;
      }
      phase ^= 1u;
    }
    uint32_t leafm = 0;
    if (active) {
      const float4* gl = S.grp[lane];
      uint32_t m = 0;
#pragma unroll
      for (int c = 0; c < W; ++c) {
        const uint32_t idx = (static_cast<uint32_t>(c) + lane) & (W - 1);
        const float4 e = gl[idx];
        if (idx < lim && Ops::coarse(e, s.q)) m |= 1u << idx;
      }
      if (at_leaf) {
        if constexpr (Ops::kNeeds64) {  // exact test on the slots' double envelopes
          const DBox* p64 = F.tree[s.t].leaves64 + first;
#pragma unroll
          for (int c = 0; c < W; ++c)
            if (((m >> c) & 1u) && !Ops::exact64(load_dbox(p64 + c), s.q)) m &= ~(1u << c);
        } else if constexpr (Ops::kRefine) {
#pragma unroll
          for (int c = 0; c < W; ++c) {
            const uint32_t idx = (static_cast<uint32_t>(c) + lane) & (W - 1);
            if (((m >> idx) & 1u) && !Ops::exact(gl[idx], s.q)) m &= ~(1u << idx);
          }
        }
        leafm = m;
      } else {
        s.ms.set(s.L, m);
      }
    }
    if (MODE == kCollect) {
      out.template add_resolved<W>(qu, leafm, S.sid[lane], s.qid + B.id_offset, s.rb);
    } else {
      cnt += __popc(leafm);
    }
    if (active) {
      active = trav_advance<PRED, W>(F, s);
      if (MODE == kCount && ROUTED && !active) {
        count_routed(M, s.rb, cnt);
        cnt = 0;
      }
    }
    uint32_t idle = __ballot_sync(kFull, !active);
    if (idle != 0 && next < cend) {
      uint32_t slot = next + __popc(idle & lanemask_lt());
      if (!active && slot < cend) active = trav_start<PRED, W, ROUTED>(F, B, slot, s, only, M);
      next = min(cend, next + __popc(idle));
    }
  }
  if (MODE == kCollect) out.flush(qu);
  if (MODE == kCount && !ROUTED) count_flush_warp(static_cast<unsigned long long*>(B.arg), cnt);
  __syncwarp();
  if (lane == 0) S.phase = phase;
  __syncwarp();
  return ok;
}

// ---------------------------------------------------------------------------
// team scheme: W lanes per query, 32 / W queries in flight per warp (float
// indexes only: double launches use the thread or packet scheme)
// ---------------------------------------------------------------------------
template <int PRED, int MODE, int W>
__device__ __forceinline__ void run_chunk_team(const Forest& F, const BatchDesc& B,
                                               uint32_t cbeg, uint32_t cend, DevPair* wbuf, uint32_t* wbat,
                                               const uint32_t* only) {
  using Ops = QueryOps<PRED>;
  constexpr uint32_t kTeams = 32 / W;
  constexpr uint32_t kTeamMask = (W == 32) ? kFull : ((1u << W) - 1u);
  const uint32_t lane = lane_id();
  const uint32_t team = lane / W;
  const uint32_t tl = lane % W;
  const MergedOrder M{};  // the team scheme runs batch by batch
  TravState<PRED, W> s;
  uint32_t next = cbeg;
  bool active = false;
  {
    uint32_t slot = next + team;
    if (slot < cend) active = trav_start<PRED, W, false>(F, B, slot, s, only, M);
    next = min(cend, next + kTeams);
  }
  DevQueue qu{};
  if (MODE == kCollect) qu = *static_cast<const DevQueue*>(B.arg);
  WarpOut<false> out(wbuf, wbat, F.ids_base, M);
  unsigned long long cnt = 0;

  for (;;) {
    if (!__any_sync(kFull, active)) {
      if (next >= cend) break;  // see run_chunk_thread
      uint32_t slot = next + team;
      if (slot < cend) active = trav_start<PRED, W, false>(F, B, slot, s, only, M);
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
      out.add_one(qu, leaf_hit, gid, s.qid + B.id_offset, s.rb);
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
      if (!active && slot < cend) active = trav_start<PRED, W, false>(F, B, slot, s, only, M);
      next = min(cend, next + __popc(idle) / W);
    }
  }
  if (MODE == kCollect) out.flush(qu);
  if (MODE == kCount) count_flush_warp(static_cast<unsigned long long*>(B.arg), cnt);
}

}  // namespace rts

namespace rts {

// ---------------------------------------------------------------------------
// packet scheme: one warp walks up to 32 queries together
// ---------------------------------------------------------------------------
// The warp descends the forest once for a packet of queries (consecutive in
// the launch's visiting order, so spatially close when the order is sorted).
// Lanes map to the W entries of the group being visited (32 / W queries are
// tested per round when W < 32); each entry's test result is a 32-bit mask of
// the packet's queries it satisfies.  An upper-level entry with a non-empty
// mask becomes a group to visit with that mask; at the leaves the masks are
// the packet's pairs.  Each group is loaded once per packet instead of once
// per query, and every lane of a round does useful work.  The tests are the
// ones the other schemes make (node test at upper levels, exact predicate at
// the leaves), so results are identical.
// Position of the highest set bit of a non-zero word (one bfind).
__device__ __forceinline__ uint32_t high_bit(uint32_t x) {
  uint32_t r;
  asm("bfind.u32 %0, %1;" : "=r"(r) : "r"(x));
  return r;
}

template <int PRED, int W>
struct PacketSmem {
  typename QueryOps<PRED>::Q q[32];  // the packet's queries (prepared per sub-tree)
  uint32_t rid[32];                  // reported id (merged launch: sorted position)
  uint32_t rb[32];                   // merged launch: batch of each query
  uint32_t over[32];                 // merged counting: per-query carries out of the slices
  uint32_t stk[MaskStack<W>::kLevels + 1][W];  // query masks of the path's pending entries
};

// Merged counting in the packet scheme: each entry lane keeps, for the 32
// queries of the packet, how many of its entries' tests hit, as kSlices
// bit-planes (bit j of plane k = bit k of query j's count), so adding a leaf
// group's hit mask costs a few logic operations whatever the number of hits.
constexpr int kSlices = 8;

template <int W>
constexpr size_t packet_smem_bytes() {
  size_t m = sizeof(PacketSmem<kPoint, W>);
  m = sizeof(PacketSmem<kContains, W>) > m ? sizeof(PacketSmem<kContains, W>) : m;
  m = sizeof(PacketSmem<kIntersects, W>) > m ? sizeof(PacketSmem<kIntersects, W>) : m;
  m = sizeof(PacketSmem<kIntersects64, W>) > m ? sizeof(PacketSmem<kIntersects64, W>) : m;
  return m;
}

template <int PRED, int MODE, int W, bool ROUTED>
__device__ __forceinline__ void run_chunk_packet(const Forest& F, const BatchDesc& B,
                                                 uint32_t cbeg, uint32_t cend, DevPair* wbuf,
                                                 uint32_t* wbat, void* praw,
                                                 const MergedOrder& M) {
  using Ops = QueryOps<PRED>;
  using Q = typename Ops::Q;
  constexpr uint32_t kGroups = 32 / W;  // queries tested per round
  constexpr uint32_t kEntryMask = (W == 32) ? kFull : ((1u << W) - 1u);
  PacketSmem<PRED, W>& P = *static_cast<PacketSmem<PRED, W>*>(praw);
  const uint32_t lane = lane_id();
  const uint32_t part = lane / W;  // which query of a round this lane tests
  const uint32_t c = lane % W;     // which entry of the group
  DevQueue qu{};
  if (MODE == kCollect && !ROUTED) qu = *static_cast<const DevQueue*>(B.arg);
  WarpOut<ROUTED> out(wbuf, wbat, F.ids_base, M);
  unsigned long long cnt = 0;  // unmerged counting: this lane's pairs

  for (uint32_t pk = cbeg; pk < cend; pk += 32) {
    const uint32_t np = min(32u, cend - pk);
    const uint32_t all = (np == 32) ? kFull : ((1u << np) - 1u);
    Q myq{};
    if (lane < np) {
      const uint32_t slot = pk + lane;
      const uint32_t qid = B.order ? B.order[slot] : slot;
      myq = Ops::load(B.queries, qid);
      P.rid[lane] = qid + B.id_offset;
      P.rb[lane] = ROUTED ? __ldg(M.batch + slot) : 0u;
    }
    uint32_t planes[kSlices];  // merged counting: this lane's per-query counts, bit-sliced
#pragma unroll
    for (int k = 0; k < kSlices; ++k) planes[k] = 0;
    P.over[lane] = 0;

    for (uint32_t t = 0; t < F.n_trees; ++t) {
      const TreeDesc& T = F.tree[t];
      __syncwarp();
      if (lane < np) {
        Q qq = myq;
        Ops::enter_tree(qq, __ldg(T.nodes));
        P.q[lane] = qq;
      }
      __syncwarp();
      MaskStack<W> pend;
      pend.clear();
      uint32_t L = T.top, g = 0, qm = all;
      for (;;) {
        // Visit group g of level L for the queries in qm.
        const uint32_t first = g * W;
        const bool at_leaf = (L == 0);
        const float4* p = at_leaf ? T.leaves + first : T.nodes + T.level_off[L] + first;
        const uint32_t lim = (at_leaf ? T.n : T.level_cnt[L]) - first;
        const float4 e = __ldg(p + c);
        const bool valid = c < lim;
        uint32_t hm = 0;
        uint32_t rm = qm;
        // Per entry, prepared once for all the packet's queries: the hull of
        // a stored box (the intersects prefilter), its diagonal reciprocals
        // and (double index) its double envelope, the last two on first use.
        const float4 eh =
            make_float4(fminf(e.x, e.z), fminf(e.y, e.w), fmaxf(e.x, e.z), fmaxf(e.y, e.w));
        float gix = 0.f, giy = 0.f;
        bool have_rcp = false;
        DBox g64{};
        bool have64 = false;
        auto test = [&](uint32_t j) -> bool {
          if constexpr (Ops::kNeeds64) {
            bool hit = at_leaf ? overlaps(eh, P.q[j].nb) : Ops::node(e, P.q[j]);
            if (hit && at_leaf) {
              if (!have64) {
                g64 = load_dbox(T.leaves64 + first + c);
                have64 = true;
              }
              hit = Ops::exact64(g64, P.q[j]);
            }
            return hit;
          } else if constexpr (PRED == kIntersects) {
            return at_leaf ? isect_leaf_pre(e, eh, gix, giy, have_rcp, P.q[j])
                           : Ops::node(e, P.q[j]);
          } else {
            return at_leaf ? Ops::leaf(e, P.q[j]) : Ops::node(e, P.q[j]);
          }
        };
        if constexpr (kGroups == 1) {
          bool done = false;
          if constexpr (PRED == kIntersects) {
            if (at_leaf) {
              // Two phases: the hull prefilter of every live query gives each
              // lane its candidates, then every lane takes its own candidates
              // one per round through the exact (slab) test, so a round pays
              // one exact test for up to 32 candidates of different lanes.
              uint32_t cand = 0;
              if (valid) {
                if (rm == kFull) {
#pragma unroll 4
                  for (uint32_t j = 0; j < 32; ++j)
                    if (overlaps(eh, P.q[j].nb)) cand |= 1u << j;
                } else {
                  for (uint32_t m = rm; m;) {
                    const uint32_t j = high_bit(m);
                    m ^= 1u << j;
                    if (overlaps(eh, P.q[j].nb)) cand |= 1u << j;
                  }
                }
              }
              while (__any_sync(kFull, cand != 0)) {
                if (cand) {
                  const uint32_t j = high_bit(cand);
                  cand ^= 1u << j;
                  if (isect_leaf_post(e, gix, giy, have_rcp, P.q[j])) hm |= 1u << j;
                }
              }
              done = true;
            }
          }
          // Measured on range-intersects, 10M x 1M (B200): 1.170 ms per step
          // with one loop for all levels, 1.143 ms with the full-packet loop,
          // 0.989 ms with the two leaf phases as well; full-packet loops also
          // for packets with >= 20 (or 12) live queries, with a bit test per
          // position, were slower (1.049, 1.074 ms).
          if (done) {
          } else if (rm == kFull) {
            // uniform: all 32 queries in turn, no mask arithmetic (the top
            // levels, where every query of a sorted packet is live)
            if (valid) {
#pragma unroll 4
              for (uint32_t j = 0; j < 32; ++j)
                if (test(j)) hm |= 1u << j;
            }
          } else {
            while (rm) {  // uniform: two queries per round, highest bits first
              const uint32_t j1 = high_bit(rm);
              rm ^= 1u << j1;
              uint32_t j2 = 32;
              if (rm) {
                j2 = high_bit(rm);
                rm ^= 1u << j2;
              }
              if (valid) {
                if (test(j1)) hm |= 1u << j1;
                if (j2 < 32 && test(j2)) hm |= 1u << j2;
              }
            }
          }
        } else {
          while (rm) {  // uniform: kGroups queries per round
            uint32_t mine = rm;
#pragma unroll
            for (uint32_t k = 0; k + 1 < kGroups; ++k)
              if (k < part) mine &= mine - 1;
#pragma unroll
            for (uint32_t k = 0; k < kGroups; ++k) rm &= rm - 1;
            if (mine && valid) {
              const uint32_t j = __ffs(mine) - 1;
              if (test(j)) hm |= 1u << j;
            }
          }
        }
#pragma unroll
        for (uint32_t o = W; o < 32; o <<= 1) hm |= __shfl_xor_sync(kFull, hm, o);
        if (part != 0) hm = 0;  // lanes 0..W-1 own the entries from here on
        if (at_leaf) {
          const uint32_t slot0 = static_cast<uint32_t>(T.ids - F.ids_base) + first;
          if (MODE == kCollect) {
            out.add_masks(qu, hm, slot0 + c, P.rid, P.rb);
          } else if (!ROUTED) {
            cnt += __popc(hm);
          } else {
            uint32_t carry = hm;  // ripple-carry add of one hit per set bit
#pragma unroll
            for (int k = 0; k < kSlices; ++k) {
              const uint32_t t = planes[k] & carry;
              planes[k] ^= carry;
              carry = t;
            }
            while (carry) {  // a count passed 2^kSlices - 1 (rare)
              const uint32_t j = __ffs(carry) - 1;
              carry &= carry - 1;
              atomicAdd(&P.over[j], 1u);
            }
          }
        } else {
          if (part == 0) P.stk[L][c] = hm;
          pend.set(L, __ballot_sync(kFull, hm != 0) & kEntryMask);
        }
        // Next group: the lowest pending entry of the deepest level that has one.
        while (L == 0 || pend.get(L) == 0) {
          if (L == T.top) break;
          L += 1;
          g /= W;
        }
        if (L == 0 || pend.get(L) == 0) break;  // sub-tree done
        const uint32_t m = pend.get(L);
        const uint32_t cc = __ffs(m) - 1;
        pend.set(L, m & (m - 1));
        __syncwarp();
        qm = P.stk[L][cc];
        g = g * W + cc;
        L -= 1;
      }
    }
    if (MODE == kCount && ROUTED) {
      // Lane j gathers query j's count from every lane's planes.
      unsigned long long qcount = 0;
      uint32_t touched = 0;
#pragma unroll
      for (int k = 0; k < kSlices; ++k) touched |= planes[k];
      touched = __reduce_or_sync(kFull, touched);
      while (touched) {  // uniform
        const uint32_t j = __ffs(touched) - 1;
        touched &= touched - 1;
        unsigned long long v = 0;
#pragma unroll
        for (int k = 0; k < kSlices; ++k)
          v += static_cast<unsigned long long>(__popc(__ballot_sync(kFull, (planes[k] >> j) & 1u)))
               << k;
        if (lane == j) qcount = v;
      }
      __syncwarp();
      if (lane < np) {
        qcount += static_cast<unsigned long long>(P.over[lane]) << kSlices;
        count_routed(M, P.rb[lane], qcount);
      }
    }
    __syncwarp();
  }
  if (MODE == kCollect) out.flush(qu);
  if (MODE == kCount && !ROUTED) count_flush_warp(static_cast<unsigned long long*>(B.arg), cnt);
}

}  // namespace rts
