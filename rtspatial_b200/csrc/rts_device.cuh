// Device-side types and exact predicates of the rtspatial_b200 index.
//
// Index layout in HBM (one "tree" per insert batch until a merge rebuild):
//   leaves[slot]    float4 {min.x, min.y, max.x, max.y}: the stored envelopes,
//                   grouped by tree and packed along a space-filling curve
//   leaf_ids[slot]  uint32 insertion-order id of the envelope in that slot
//   pos[id]         slot of an id (Delete/Update write through it)
//   nodes (per tree) float4 boxes of the upper levels; level L >= 1 entry j is
//                   the hull of entries [j*W, j*W+W) of level L-1 (level 0 =
//                   the tree's leaves).  nodes[0] holds the tree's root box.
// The tree is implicit: the children of level-L entry j are entries
// [j*W, j*W+W) of level L-1, so no child pointers are stored and a refit is
// one coalesced pass per level.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rts {

constexpr int kMaxLevels = 16;
constexpr int kMaxTrees = 16;
constexpr uint32_t kFull = 0xffffffffu;

// The *64 kinds are the queries of a double index (SpatialIndex<double, 2>).
enum PredKind : int {
  kPoint = 0,
  kContains = 1,
  kIntersects = 2,
  kPoint64 = 3,
  kContains64 = 4,
  kIntersects64 = 5
};
constexpr int kNumPreds = 6;

// A double envelope {min.x, min.y, max.x, max.y} as two 16-byte halves.
struct __align__(16) DBox {
  double2 lo, hi;
};
__device__ __forceinline__ DBox load_dbox(const DBox* p) {
  return DBox{__ldg(&p->lo), __ldg(&p->hi)};
}
// kUser: the caller's own device handlers (rtspatial_handle_*), called once
// per pair by the kernels of a handler module compiled with them.
enum HandlerKind : int { kCount = 0, kCollect = 1, kUser = 2 };

// Handler type of the kernels that do not call user handlers.
struct NoUserHandler {
  template <int PRED>
  static __device__ __forceinline__ void call(uint32_t, uint32_t, void*) {}
};

// Two consecutive boxes with one 32-byte read-only load (sm_100 256-bit
// vector load, four 64-bit lanes).  p must be 32-byte aligned: every W-group
// starts 16 * W bytes after a multiple of 512 (sub-trees start on 32-slot
// boundaries, node levels on W-entry ones), so the pairs (2c, 2c + 1) of a
// group are; refresh_forest checks the buffers' bases.
__device__ __forceinline__ void ldg_box_pair(const float4* p, float4& a, float4& b) {
  unsigned long long x0, x1, x2, x3;
  asm("ld.global.nc.v4.b64 {%0, %1, %2, %3}, [%4];"
      : "=l"(x0), "=l"(x1), "=l"(x2), "=l"(x3)
      : "l"(p));
  a = make_float4(__uint_as_float(static_cast<uint32_t>(x0)),
                  __uint_as_float(static_cast<uint32_t>(x0 >> 32)),
                  __uint_as_float(static_cast<uint32_t>(x1)),
                  __uint_as_float(static_cast<uint32_t>(x1 >> 32)));
  b = make_float4(__uint_as_float(static_cast<uint32_t>(x2)),
                  __uint_as_float(static_cast<uint32_t>(x2 >> 32)),
                  __uint_as_float(static_cast<uint32_t>(x3)),
                  __uint_as_float(static_cast<uint32_t>(x3 >> 32)));
}

// ---------------------------------------------------------------------------
// Bulk copies into shared memory (the staged traversal scheme).  A copy is
// issued by one thread with cp.async.bulk (the TMA unit moves the bytes from
// L2 into shared memory without passing through L1 or registers) and
// completes on an mbarrier whose transaction count it decrements.  Each copy
// writes the issuing CTA's own shared memory from this GPU's global memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t arrivals) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(arrivals) : "memory");
}
// Makes barrier initialisations visible to the async proxy.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Arrives on the barrier and raises its expected transaction bytes.
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Orders this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy (bulk copy) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// bytes (a multiple of 16) from global src (16-byte aligned) to shared dst
// (16-byte aligned), completing on barrier bar.
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                              uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
// Spin limit of a barrier wait (each try_wait also suspends for a
// hardware-chosen time): far beyond any copy's latency, so reaching it means
// the copy engine stopped answering; the kernel then records kErrWaitTimeout
// and returns instead of spinning on.
constexpr uint32_t kWaitSpinLimit = 1u << 22;
constexpr uint32_t kErrWaitTimeout = 1u;

// ldg_box_pair for streaming group loads: no L1 allocation (groups of a large
// index are rarely reused before eviction and would push out the kernel's
// own working set) and a 256-byte L2 fetch on a miss (a W16 group is two
// 128-byte lines, 256-byte aligned).
__device__ __forceinline__ void ldg_box_pair_stream(const float4* p, float4& a, float4& b) {
  unsigned long long x0, x1, x2, x3;
  asm("ld.global.nc.L1::no_allocate.L2::256B.v4.b64 {%0, %1, %2, %3}, [%4];"
      : "=l"(x0), "=l"(x1), "=l"(x2), "=l"(x3)
      : "l"(p));
  a = make_float4(__uint_as_float(static_cast<uint32_t>(x0)),
                  __uint_as_float(static_cast<uint32_t>(x0 >> 32)),
                  __uint_as_float(static_cast<uint32_t>(x1)),
                  __uint_as_float(static_cast<uint32_t>(x1 >> 32)));
  b = make_float4(__uint_as_float(static_cast<uint32_t>(x2)),
                  __uint_as_float(static_cast<uint32_t>(x2 >> 32)),
                  __uint_as_float(static_cast<uint32_t>(x3)),
                  __uint_as_float(static_cast<uint32_t>(x3 >> 32)));
}

// A leaf slot's geom id, for the output: read without L1 allocation (the ids
// of a large index are rarely reused, and L1 holds the kernel's spills and
// upper tree levels).  Measured on config 2: 1.354 -> 1.336 ms.
__device__ __forceinline__ uint32_t ldg_geom_id(const uint32_t* p) {
  uint32_t v;
  asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

struct TreeDesc {
  const float4* leaves;  // first slot of this tree
  const DBox* leaves64;  // double index: the double envelopes of the same slots
  const uint32_t* ids;   // leaf_ids of the first slot
  const float4* nodes;   // nodes[0] = root box; level L at nodes + level_off[L]
  uint32_t n;            // envelopes in this tree
  uint32_t top;          // highest level (>= 1); it holds <= W entries
  uint32_t level_off[kMaxLevels];
  uint32_t level_cnt[kMaxLevels];
};

struct Forest {
  TreeDesc tree[kMaxTrees];
  const uint32_t* ids_base;  // leaf_ids of slot 0 (all sub-trees share the array)
  uint32_t* err;             // device status word of the index (kErr* bits), or nullptr
  uint32_t n_trees;
  uint32_t width;
  // thread scheme: group loads bypass L1 allocation, for launches that
  // collect (or call user handlers) and for launches that count
  uint32_t stream_collect, stream_count;
};

// Collecting handler target: member layout of
// rtspatial::dev::Queue<thrust::pair<uint32_t,uint32_t>> (utils/queue.h:60-62).
struct DevPair {
  uint32_t geom_id;
  uint32_t query_id;
};
struct DevQueue {
  DevPair* data;
  unsigned long long capacity;
  uint32_t* size;
};

// ---------------------------------------------------------------------------
// Exact predicates (float32, IEEE round-to-nearest, no contraction).
// ---------------------------------------------------------------------------

// nextafterf(1.0f, FLT_MAX) (details/ray_params.h:139).
constexpr float kT1 = 0x1.000002p+0f;
// 1 + 2 * FLT_GAMMA(3) in float arithmetic = 1 + 6 * 2^-23
// (details/ray_params.h:40,158).
constexpr float kSlabK = 0x1.00000cp+0f;

// RayParams<float,2>::IsHit (details/ray_params.h:137-166) with the two
// reciprocals of the ray direction supplied by the caller (the reference
// computes the same 1/d inside the loop).  NaN slab values leave [t0, t1]
// unchanged, like the reference's ternaries.
__device__ __forceinline__ bool slab_hit(float ox, float oy, float invx, float invy,
                                         float4 b) {
  float t0 = 0.0f, t1 = kT1;
  float tn = __fmul_rn(__fsub_rn(b.x, ox), invx);
  float tf = __fmul_rn(__fsub_rn(b.z, ox), invx);
  if (tn > tf) {
    float t = tn;
    tn = tf;
    tf = t;
  }
  tf = __fmul_rn(tf, kSlabK);
  t0 = tn > t0 ? tn : t0;
  t1 = tf < t1 ? tf : t1;
  if (t0 > t1) return false;
  tn = __fmul_rn(__fsub_rn(b.y, oy), invy);
  tf = __fmul_rn(__fsub_rn(b.w, oy), invy);
  if (tn > tf) {
    float t = tn;
    tn = tf;
    tf = t;
  }
  tf = __fmul_rn(tf, kSlabK);
  t0 = tn > t0 ? tn : t0;
  t1 = tf < t1 ? tf : t1;
  return !(t0 > t1);
}

// Envelope::Contains(point) (geom/envelope.cuh:29-38), closed intervals.
__device__ __forceinline__ bool contains_point(float4 g, float2 p) {
  return p.x >= g.x && p.x <= g.z && p.y >= g.y && p.y <= g.w;
}

// Envelope::Contains(envelope) (geom/envelope.cuh:40-53).
__device__ __forceinline__ bool contains_box(float4 g, float4 q) {
  return q.x >= g.x && q.z <= g.z && q.y >= g.y && q.w <= g.w;
}

// Per-query state of a range-intersects query.
struct IsectQuery {
  float4 q;            // the query envelope
  float ox, oy;        // origin of its anti-diagonal ray: (max.x, min.y)
  float invx, invy;    // 1 / (min.x - max.x), 1 / (max.y - min.y)
  float4 nb;           // hull of q inflated by the conservative margin
};

__device__ __forceinline__ IsectQuery make_isect_query(float4 q) {
  IsectQuery Q;
  Q.q = q;
  // RayParams::Compute(query, true) (details/ray_params.h:67-84).
  Q.ox = q.z;
  Q.oy = q.y;
  Q.invx = __frcp_rn(__fsub_rn(q.x, q.z));
  Q.invy = __frcp_rn(__fsub_rn(q.w, q.y));
  Q.nb = make_float4(0.f, 0.f, 0.f, 0.f);
  return Q;
}

// Margin for the node test of range-intersects.  If the reference's
// predicate accepts (g, q), some t* in [t0, t1] certifies it.  Along the
// computed direction d~ = fl(p2 - p1) every slab value carries a relative
// error <= 3u (u = 2^-24); the far value is scaled by 1 + 12u and rounded once
// more; t* <= 1 + 2u and d~ is within u of p2 - p1.  So the point o + t* d~
// lies within 3u|p2 - p1| of the ray's box and within 17u*max(|min - o|,
// |max - o|) of the target box per axis: the two hulls are apart by at most
// 40u*M, M the largest coordinate magnitude of the pair.  Zero or subnormal
// directions give infinite or NaN slab values, which only accept when the
// origin lies within the slab.  The margin 2^-17*M + 2^-120 = (128u)*M + tiny
// exceeds the bound with room for the rounding of the inflated bounds.
// The bound needs finite coordinates: with an infinite one in the query or
// the tree (M infinite), or a NaN in the query, the window is the whole
// plane and the exact leaf test alone decides.
// mag = per-axis magnitude bound of the tree's boxes.
__device__ __forceinline__ void isect_set_margin(IsectQuery& Q, float2 mag) {
  const float4 q = Q.q;
  float mx = fmaxf(mag.x, fmaxf(fabsf(q.x), fabsf(q.z)));
  float my = fmaxf(mag.y, fmaxf(fabsf(q.y), fabsf(q.w)));
  float ex = __fadd_rn(__fmul_rn(mx, 0x1p-17f), 0x1p-120f);
  float ey = __fadd_rn(__fmul_rn(my, 0x1p-17f), 0x1p-120f);
  Q.nb.x = __fsub_rn(fminf(q.x, q.z), ex);
  Q.nb.y = __fsub_rn(fminf(q.y, q.w), ey);
  Q.nb.z = __fadd_rn(fmaxf(q.x, q.z), ex);
  Q.nb.w = __fadd_rn(fmaxf(q.y, q.w), ey);
  const bool finite = ex < INFINITY && ey < INFINITY && q.x == q.x && q.y == q.y &&
                      q.z == q.z && q.w == q.w;
  if (!finite) Q.nb = make_float4(-INFINITY, -INFINITY, INFINITY, INFINITY);
}

// Closed overlap of a (hull) box with the inflated query box.
__device__ __forceinline__ bool overlaps(float4 e, float4 nb) {
  return e.x <= nb.z && e.z >= nb.x && e.y <= nb.w && e.w >= nb.y;
}

// Range-intersects result set of the reference for pair (g, q):
//   backward pass (shaders_intersects_envelope_query_2d.cu:75-129): g valid
//     and g's main diagonal hits q;
//   forward pass (same file :14-41): q's anti-diagonal hits g and g's main
//     diagonal misses q.
// i.e. hit2 = IsHit(g main diagonal, q); result = hit2 ? g.IsValid() : hit1.
__device__ __forceinline__ bool isect_exact(float4 g, const IsectQuery& Q) {
  float gix = __frcp_rn(__fsub_rn(g.z, g.x));
  float giy = __frcp_rn(__fsub_rn(g.w, g.y));
  if (slab_hit(g.x, g.y, gix, giy, Q.q)) return g.x < g.z && g.y < g.w;
  return slab_hit(Q.ox, Q.oy, Q.invx, Q.invy, g);
}

// Leaf test: the exact predicate behind the (sound) inflated-hull prefilter.
__device__ __forceinline__ bool isect_leaf(float4 g, const IsectQuery& Q) {
  float4 h = make_float4(fminf(g.x, g.z), fminf(g.y, g.w), fmaxf(g.x, g.z), fmaxf(g.y, g.w));
  if (!overlaps(h, Q.nb)) return false;
  return isect_exact(g, Q);
}

// isect_leaf for a stored box g tested against many queries: its hull h is
// computed once, and its diagonal reciprocals the first time a query passes
// the prefilter (gix, giy, have carry them between calls).  The same
// operations as isect_leaf, so the same results.
__device__ __forceinline__ bool isect_leaf_post(float4 g, float& gix, float& giy, bool& have,
                                                const IsectQuery& Q);
__device__ __forceinline__ bool isect_leaf_pre(float4 g, float4 h, float& gix, float& giy,
                                               bool& have, const IsectQuery& Q) {
  if (!overlaps(h, Q.nb)) return false;
  return isect_leaf_post(g, gix, giy, have, Q);
}

// The part of isect_leaf_pre after its hull prefilter passed.
__device__ __forceinline__ bool isect_leaf_post(float4 g, float& gix, float& giy, bool& have,
                                                const IsectQuery& Q) {
  if (!have) {
    gix = __frcp_rn(__fsub_rn(g.z, g.x));
    giy = __frcp_rn(__fsub_rn(g.w, g.y));
    have = true;
  }
  if (slab_hit(g.x, g.y, gix, giy, Q.q)) return g.x < g.z && g.y < g.w;
  return slab_hit(Q.ox, Q.oy, Q.invx, Q.invy, g);
}

// Magnitude bound of a tree from its root box (node boxes are hulls).
__device__ __forceinline__ float2 root_magnitude(float4 r) {
  return make_float2(fmaxf(fabsf(r.x), fabsf(r.z)), fmaxf(fabsf(r.y), fabsf(r.w)));
}

// ---------------------------------------------------------------------------
// Double index (SpatialIndex<double, 2>).  Its float leaves hold each double
// envelope rounded to nearest, which is what Envelope::Contains compares
// (Point<double,2>::get_coordinate returns float, geom/point.cuh:68-71), so
// point- and range-contains run the float predicates on rounded queries.
// Range-intersects runs RayParams<double,2>::IsHit in double.
// ---------------------------------------------------------------------------

// 1 + 2 * DBL_GAMMA(3) in double arithmetic = 1 + 6 * 2^-52
// (details/ray_params.h:41,283).
constexpr double kSlabK64 = 0x1.0000000000006p+0;

__device__ __forceinline__ float4 round_box(DBox b) {
  return make_float4(__double2float_rn(b.lo.x), __double2float_rn(b.lo.y),
                     __double2float_rn(b.hi.x), __double2float_rn(b.hi.y));
}

// RayParams<double,2>::IsHit (details/ray_params.h:260-290); t1 starts at
// nextafterf(1.0, DBL_MAX), a float value.
__device__ __forceinline__ bool slab_hit64(double ox, double oy, double invx, double invy,
                                           DBox b) {
  double t0 = 0.0, t1 = static_cast<double>(kT1);
  double tn = __dmul_rn(__dsub_rn(b.lo.x, ox), invx);
  double tf = __dmul_rn(__dsub_rn(b.hi.x, ox), invx);
  if (tn > tf) {
    double t = tn;
    tn = tf;
    tf = t;
  }
  tf = __dmul_rn(tf, kSlabK64);
  t0 = tn > t0 ? tn : t0;
  t1 = tf < t1 ? tf : t1;
  if (t0 > t1) return false;
  tn = __dmul_rn(__dsub_rn(b.lo.y, oy), invy);
  tf = __dmul_rn(__dsub_rn(b.hi.y, oy), invy);
  if (tn > tf) {
    double t = tn;
    tn = tf;
    tf = t;
  }
  tf = __dmul_rn(tf, kSlabK64);
  t0 = tn > t0 ? tn : t0;
  t1 = tf < t1 ? tf : t1;
  return !(t0 > t1);
}

struct IsectQuery64 {
  DBox q;               // the query envelope
  double ox, oy;        // anti-diagonal ray origin (max.x, min.y)
  double invx, invy;    // 1 / (min.x - max.x), 1 / (max.y - min.y)
  float4 nb;            // float hull of q inflated by the node-test margin
};

__device__ __forceinline__ IsectQuery64 make_isect_query64(DBox q) {
  IsectQuery64 Q;
  Q.q = q;
  // RayParams<double,2>::Compute(query, true) (details/ray_params.h:193-210).
  Q.ox = q.hi.x;
  Q.oy = q.lo.y;
  Q.invx = __drcp_rn(__dsub_rn(q.lo.x, q.hi.x));
  Q.invy = __drcp_rn(__dsub_rn(q.hi.y, q.lo.y));
  Q.nb = make_float4(0.f, 0.f, 0.f, 0.f);
  return Q;
}

// Node-test margin of the double predicate, on float hulls.  A pair accepted
// by the double slab test has boxes at most (2^-23 + 2^-50)*|d| + 2^-50*M
// apart (t1 = 1 + 2^-23); rounding both to float moves each bound by at most
// 2^-24*M.  That is < 8*2^-24*M, far inside the margin 2^-17*M + 2^-120 of
// isect_set_margin, applied to the rounded query.
__device__ __forceinline__ void isect_set_margin64(IsectQuery64& Q, float2 mag) {
  IsectQuery t;
  t.q = round_box(Q.q);
  isect_set_margin(t, mag);
  Q.nb = t.nb;
}

// The double index's range-intersects result set: the composition of
// isect_exact with RayParams<double,2> (Compute / IsHit in double).
__device__ __forceinline__ bool isect_exact64(DBox g, const IsectQuery64& Q) {
  double gix = __drcp_rn(__dsub_rn(g.hi.x, g.lo.x));
  double giy = __drcp_rn(__dsub_rn(g.hi.y, g.lo.y));
  if (slab_hit64(g.lo.x, g.lo.y, gix, giy, Q.q)) return g.lo.x < g.hi.x && g.lo.y < g.hi.y;
  return slab_hit64(Q.ox, Q.oy, Q.invx, Q.invy, g);
}

// ---------------------------------------------------------------------------
// Query adaptors: one per predicate, same interface.
// ---------------------------------------------------------------------------
template <int PRED>
struct QueryOps;

// node():   test of an upper-level entry (a hull);
// leaf():   exact predicate on a stored box;
// coarse(): a test valid at both levels that implies nothing is missed;
// kRefine:  leaves that pass coarse() still need the exact test.
template <>
struct QueryOps<kPoint> {
  using Q = float2;
  static constexpr bool kRefine = false;
  static constexpr bool kNeeds64 = false;
  static __device__ __forceinline__ bool coarse(float4 e, const Q& p) { return contains_point(e, p); }
  static __device__ __forceinline__ Q load(const float* qs, uint32_t i) {
    return reinterpret_cast<const float2*>(qs)[i];
  }
  static __device__ __forceinline__ void enter_tree(Q&, float4) {}
  static __device__ __forceinline__ bool node(float4 e, const Q& p) { return contains_point(e, p); }
  static __device__ __forceinline__ bool leaf(float4 g, const Q& p) { return contains_point(g, p); }
};

template <>
struct QueryOps<kContains> {
  using Q = float4;
  static constexpr bool kRefine = false;
  static constexpr bool kNeeds64 = false;
  static __device__ __forceinline__ bool coarse(float4 e, const Q& q) { return contains_box(e, q); }
  static __device__ __forceinline__ Q load(const float* qs, uint32_t i) {
    return reinterpret_cast<const float4*>(qs)[i];
  }
  static __device__ __forceinline__ void enter_tree(Q&, float4) {}
  // A box containing q lies inside a node hull that then contains q too.
  static __device__ __forceinline__ bool node(float4 e, const Q& q) { return contains_box(e, q); }
  static __device__ __forceinline__ bool leaf(float4 g, const Q& q) { return contains_box(g, q); }
};

template <>
struct QueryOps<kIntersects> {
  using Q = IsectQuery;
  static constexpr bool kRefine = true;
  static constexpr bool kNeeds64 = false;
  static __device__ __forceinline__ bool coarse(float4 e, const Q& q) {
    return overlaps(make_float4(fminf(e.x, e.z), fminf(e.y, e.w), fmaxf(e.x, e.z), fmaxf(e.y, e.w)),
                    q.nb);
  }
  static __device__ __forceinline__ bool exact(float4 g, const Q& q) { return isect_exact(g, q); }
  static __device__ __forceinline__ Q load(const float* qs, uint32_t i) {
    return make_isect_query(reinterpret_cast<const float4*>(qs)[i]);
  }
  static __device__ __forceinline__ void enter_tree(Q& q, float4 root) {
    isect_set_margin(q, root_magnitude(root));
  }
  static __device__ __forceinline__ bool node(float4 e, const Q& q) { return overlaps(e, q.nb); }
  static __device__ __forceinline__ bool leaf(float4 g, const Q& q) { return isect_leaf(g, q); }
};

// Double index, contains predicates: the float operations on the query
// rounded to nearest.
template <>
struct QueryOps<kPoint64> : QueryOps<kPoint> {
  static __device__ __forceinline__ Q load(const float* qs, uint32_t i) {
    const double2 p = reinterpret_cast<const double2*>(qs)[i];
    return make_float2(__double2float_rn(p.x), __double2float_rn(p.y));
  }
};

template <>
struct QueryOps<kContains64> : QueryOps<kContains> {
  static __device__ __forceinline__ Q load(const float* qs, uint32_t i) {
    return round_box(reinterpret_cast<const DBox*>(qs)[i]);
  }
};

// Double index, range-intersects: float hull tests (sound by the margin),
// then the exact double predicate on the slot's double envelope (exact64).
template <>
struct QueryOps<kIntersects64> {
  using Q = IsectQuery64;
  static constexpr bool kRefine = true;
  static constexpr bool kNeeds64 = true;
  static __device__ __forceinline__ bool coarse(float4 e, const Q& q) {
    return overlaps(make_float4(fminf(e.x, e.z), fminf(e.y, e.w), fmaxf(e.x, e.z), fmaxf(e.y, e.w)),
                    q.nb);
  }
  static __device__ __forceinline__ bool exact64(DBox g, const Q& q) { return isect_exact64(g, q); }
  static __device__ __forceinline__ Q load(const float* qs, uint32_t i) {
    return make_isect_query64(reinterpret_cast<const DBox*>(qs)[i]);
  }
  static __device__ __forceinline__ void enter_tree(Q& q, float4 root) {
    isect_set_margin64(q, root_magnitude(root));
  }
  static __device__ __forceinline__ bool node(float4 e, const Q& q) { return overlaps(e, q.nb); }
};

// ---------------------------------------------------------------------------
// Per-level child masks of one traversal, packed W bits per level.
// ---------------------------------------------------------------------------
template <int W>
struct MaskStack {
  static constexpr int kWords = (W == 32) ? 3 : 2;
  static constexpr int kLevels = kWords * 64 / W;  // levels 1..kLevels storable
  static constexpr uint64_t kMask = (W == 32) ? 0xffffffffull : ((1ull << W) - 1ull);
  uint64_t w[kWords];

  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int i = 0; i < kWords; ++i) w[i] = 0;
  }
  __device__ __forceinline__ uint32_t get(int level) const {
    int off = (level - 1) * W;
    int wi = off >> 6, sh = off & 63;
    uint64_t v = 0;
#pragma unroll
    for (int i = 0; i < kWords; ++i) v = (i == wi) ? w[i] : v;
    return static_cast<uint32_t>((v >> sh) & kMask);
  }
  __device__ __forceinline__ void set(int level, uint32_t m) {
    int off = (level - 1) * W;
    int wi = off >> 6, sh = off & 63;
#pragma unroll
    for (int i = 0; i < kWords; ++i)
      if (i == wi) w[i] = (w[i] & ~(kMask << sh)) | (static_cast<uint64_t>(m) << sh);
  }
  __device__ __forceinline__ bool any() const {
    uint64_t v = 0;
#pragma unroll
    for (int i = 0; i < kWords; ++i) v |= w[i];
    return v != 0;
  }
  // Clears the highest set bit and returns its index p (level p / W + 1, entry
  // p % W of its group): a pending entry of the shallowest pending level, the
  // largest sub-tree still to walk.  -1 when empty.
  __device__ __forceinline__ int pop_highest() {
#pragma unroll
    for (int i = kWords - 1; i >= 0; --i) {
      if (w[i] != 0) {
        const int b = 63 - __clzll(static_cast<long long>(w[i]));
        w[i] &= ~(1ull << b);
        return b + 64 * i;
      }
    }
    return -1;
  }
};

template <int W>
constexpr uint32_t log2_width() {
  return W == 4 ? 2u : W == 8 ? 3u : W == 16 ? 4u : 5u;
}

// v as lane `src` holds it, for any struct of 32-bit words.
template <class T>
__device__ __forceinline__ T shfl_words(const T& v, int src) {
  static_assert(sizeof(T) % 4 == 0, "whole 32-bit words");
  T out;
  const uint32_t* a = reinterpret_cast<const uint32_t*>(&v);
  uint32_t* b = reinterpret_cast<uint32_t*>(&out);
#pragma unroll
  for (int i = 0; i < static_cast<int>(sizeof(T) / 4); ++i) b[i] = __shfl_sync(kFull, a[i], src);
  return out;
}

// ---------------------------------------------------------------------------
// Output: the two handler behaviours, warp-aggregated.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }


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

// Launch-wide visiting order.  When every batch of a launch shares one
// predicate and handler, the queries of all batches are sorted together and
// copied into one array, which the kernel runs as a single batch; results are
// routed back per query.  batch == nullptr: the launch runs batch by batch.
struct MergedOrder {
  const BatchDesc* descs;  // the launch's batches (device copy)
  const uint32_t* batch;   // sorted position -> batch index
  const uint32_t* ident;   // sorted position -> query id reported to that batch
  const DevQueue* routes;  // collect: copy of each batch's queue header, by batch index
};

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Warp exclusive prefix sum (and total) of per-lane counts below 2^kBits,
// from one ballot per bit: the ballots are independent, unlike the dependent
// chain of a shuffle scan.
template <int kBits>
__device__ __forceinline__ uint32_t warp_excl_prefix(uint32_t cnt, uint32_t& total) {
  const uint32_t lt = lanemask_lt();
  uint32_t excl = 0;
  total = 0;
#pragma unroll
  for (int b = 0; b < kBits; ++b) {
    const uint32_t v = __ballot_sync(kFull, (cnt >> b) & 1u);
    excl += static_cast<uint32_t>(__popc(v & lt)) << b;
    total += static_cast<uint32_t>(__popc(v)) << b;
  }
  return excl;
}

// Counting handler of a merged launch: adds one finished query's count to
// its batch (b) counter.
__device__ __forceinline__ void count_routed(const MergedOrder& mo, uint32_t b,
                                             unsigned long long c) {
  if (c == 0) return;
  atomicAdd(static_cast<unsigned long long*>(mo.descs[b].arg), c);
}

// Warp-private staging of collected pairs in shared memory.  Pairs found in a
// step are written to the warp's buffer as (leaf slot, query id); the buffer
// is flushed to the queue with one atomicAdd and coalesced 8-byte stores when
// it would overflow and when the warp finishes its chunk.  The flush turns
// slots into ids: those loads are independent, so they overlap once per flush
// instead of adding a dependent load to the query's path at every leaf.  All
// calls are made by all 32 lanes.
constexpr uint32_t kWarpOutCap = 256;
// Batch table of a merged launch's flush (per warp, after the batch indices).
constexpr uint32_t kRouteBits = 6;
constexpr uint32_t kRouteSlots = 1u << kRouteBits;
constexpr uint32_t kWarpBatWords = kWarpOutCap + 3 * kRouteSlots;

// RESOLVED: the staged entries already hold geom ids (the staged scheme reads
// them from its shared-memory copy of the leaf group); otherwise leaf slots,
// turned into ids at the flush.
template <bool ROUTED, bool RESOLVED = false>
struct WarpOut {
  DevPair* buf;              // kWarpOutCap entries in shared memory, private to the warp
  uint32_t* bat;             // merged launch: batch index of each entry, then the
                             // flush's batch table (kWarpBatWords, shared memory)
  uint32_t n;                // pairs buffered (same value in every lane)
  const uint32_t* ids;       // leaf_ids of slot 0
  // Routing of a merged launch (ROUTED), kept in registers.
  const uint32_t* ident;
  const DevQueue* routes;

  __device__ __forceinline__ WarpOut(DevPair* b, uint32_t* bt, const uint32_t* leaf_ids,
                                     const MergedOrder& mo)
      : buf(b), bat(bt), n(0), ids(leaf_ids), ident(mo.ident),
        routes(mo.routes) {}

  __device__ __forceinline__ void flush(const DevQueue& qu) {
    if (n == 0) return;
    __syncwarp();
    if constexpr (ROUTED) {
      flush_routed();
    } else {
      uint32_t base = 0;
      if (lane_id() == 0) base = atomicAdd(qu.size, n);
      base = __shfl_sync(kFull, base, 0);
      // Four rows of 32 at a time: their id loads are issued before any of
      // their stores, so a flush waits for ceil(n / 128) id round trips.
      constexpr int kRows = 4;
      for (uint32_t i0 = 0; i0 < n; i0 += 32 * kRows) {
        uint32_t gid[kRows], qid[kRows];
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
          const uint32_t i = i0 + lane_id() + 32u * r;
          if (i < n) {
            const DevPair e = buf[i];
            gid[r] = RESOLVED ? e.geom_id : ldg_geom_id(ids + e.geom_id);
            qid[r] = e.query_id;
          }
        }
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
          const uint32_t i = i0 + lane_id() + 32u * r;
          const unsigned long long p = static_cast<unsigned long long>(base) + i;
          if (i < n && p < qu.capacity) qu.data[p] = DevPair{gid[r], qid[r]};
        }
      }
    }
    __syncwarp();
    n = 0;
  }

  // Merged launch: buffered query ids are sorted positions, bat[] their
  // batches.  The buffer is grouped by batch in a small hash table in shared
  // memory (tab, kRouteSlots keys + counts + bases): each entry takes a rank
  // within its batch with a shared-memory atomic, then one global atomicAdd
  // per distinct batch reserves that batch's slots — all of them issued at
  // once — and every entry writes to base + rank.  Entries whose batch finds
  // no free table slot reserve their own slot directly.
  __device__ __forceinline__ void flush_routed() {
    constexpr uint32_t kEmpty = 0xffffffffu;
    const uint32_t lane = lane_id();
    uint32_t* keys = bat + kWarpOutCap;
    uint32_t* cnts = keys + kRouteSlots;
    uint32_t* bases = cnts + kRouteSlots;
    for (uint32_t k = lane; k < kRouteSlots; k += 32) {
      keys[k] = kEmpty;
      cnts[k] = 0;
    }
    __syncwarp();
    for (uint32_t i = lane; i < n; i += 32) {
      const uint32_t b = bat[i];
      const uint32_t h = (b * 0x9E3779B1u) >> (32 - kRouteBits);
      uint32_t slot = kRouteSlots;
      for (uint32_t probe = 0; probe < kRouteSlots; ++probe) {
        const uint32_t k = (h + probe) & (kRouteSlots - 1);
        const uint32_t prev = atomicCAS(&keys[k], kEmpty, b);
        if (prev == kEmpty || prev == b) {
          slot = k;
          break;
        }
      }
      if (slot < kRouteSlots) {
        bat[i] = (slot << 16) | atomicAdd(&cnts[slot], 1u);
      } else {  // table full: this entry reserves its own slot
        const DevPair e = buf[i];
        const DevQueue Q = routes[b];
        const unsigned long long p = atomicAdd(Q.size, 1u);
        if (p < Q.capacity)
          Q.data[p] = DevPair{RESOLVED ? e.geom_id : ldg_geom_id(ids + e.geom_id),
                              __ldg(ident + e.query_id)};
        bat[i] = kEmpty;
      }
    }
    __syncwarp();
    for (uint32_t k = lane; k < kRouteSlots; k += 32)
      if (cnts[k]) bases[k] = atomicAdd(routes[keys[k]].size, cnts[k]);
    __syncwarp();
    for (uint32_t i = lane; i < n; i += 32) {
      const uint32_t v = bat[i];
      if (v == kEmpty) continue;
      const DevPair e = buf[i];
      const uint32_t slot = v >> 16;
      const DevQueue Q = routes[keys[slot]];
      const unsigned long long p = static_cast<unsigned long long>(bases[slot]) + (v & 0xffffu);
      if (p < Q.capacity)
        Q.data[p] = DevPair{RESOLVED ? e.geom_id : ldg_geom_id(ids + e.geom_id),
                            __ldg(ident + e.query_id)};
    }
  }

  // Adds, for every lane, (slot0 + c, qid) for each set bit c of m (c < W);
  // rb = the query's batch in a merged launch.
  template <int W>
  __device__ __forceinline__ void add(const DevQueue& qu, uint32_t m, uint32_t slot0,
                                      uint32_t qid, uint32_t rb) {
    if (!__any_sync(kFull, m != 0)) return;
    const uint32_t lane = lane_id();
    const uint32_t cnt = __popc(m);
    uint32_t total;
    const uint32_t excl = warp_excl_prefix<(W >= 32 ? 6 : W >= 16 ? 5 : W >= 8 ? 4 : 3)>(cnt, total);
    if (n + total > kWarpOutCap) flush(qu);
    if (ROUTED && total > kWarpOutCap) {  // more than a buffer, merged launch
      if (cnt) {
        const DevQueue Q = routes[rb];
        const uint32_t rid = __ldg(ident + qid);
        const unsigned long long p0 = atomicAdd(Q.size, cnt);
#pragma unroll
        for (int c = 0; c < W; ++c) {
          if ((m >> c) & 1u) {
            unsigned long long p = p0 + __popc(m & ((1u << c) - 1u));
            if (p < Q.capacity) Q.data[p] = DevPair{ldg_geom_id(ids + slot0 + c), rid};
          }
        }
      }
      return;
    }
    if (total > kWarpOutCap) {  // more than a buffer: straight to the queue
      uint32_t base = 0;
      if (lane == 31) base = atomicAdd(qu.size, total);
      base = __shfl_sync(kFull, base, 31);
      const unsigned long long p0 = static_cast<unsigned long long>(base) + excl;
#pragma unroll
      for (int c = 0; c < W; ++c) {
        if ((m >> c) & 1u) {
          unsigned long long p = p0 + __popc(m & ((1u << c) - 1u));
          if (p < qu.capacity) qu.data[p] = DevPair{ldg_geom_id(ids + slot0 + c), qid};
        }
      }
      return;
    }
    uint32_t k = n + excl;
#pragma unroll
    for (int c = 0; c < W; ++c) {  // the set bits, lowest first (predicated, no divergence)
      if ((m >> c) & 1u) {
        buf[k] = DevPair{slot0 + c, qid};
        if constexpr (ROUTED) bat[k] = rb;
        ++k;
      }
    }
    n += total;
  }

  // Staged scheme: like add<W>, with the geom ids of the lane's leaf group in
  // shared memory (sid[0..W)); the set bits are visited starting at the
  // lane's own rotation (c + lane) mod W, which spreads the lanes' reads of
  // sid over the banks.  The pair order within a flush does not matter.
  template <int W>
  __device__ __forceinline__ void add_resolved(const DevQueue& qu, uint32_t m,
                                               const uint32_t* sid, uint32_t qid, uint32_t rb) {
    static_assert(RESOLVED, "add_resolved stages geom ids");
    if (!__any_sync(kFull, m != 0)) return;
    const uint32_t lane = lane_id();
    const uint32_t cnt = __popc(m);
    uint32_t total;
    const uint32_t excl = warp_excl_prefix<(W >= 32 ? 6 : W >= 16 ? 5 : W >= 8 ? 4 : 3)>(cnt, total);
    if (n + total > kWarpOutCap) flush(qu);
    if (total > kWarpOutCap) {  // more than a buffer: straight to the queue(s)
      if constexpr (ROUTED) {
        if (cnt) {
          const DevQueue Q = routes[rb];
          const uint32_t rid = __ldg(ident + qid);
          const unsigned long long p0 = atomicAdd(Q.size, cnt);
          unsigned long long p = p0;
#pragma unroll
          for (int c = 0; c < W; ++c) {
            if ((m >> c) & 1u) {
              if (p < Q.capacity) Q.data[p] = DevPair{sid[c], rid};
              ++p;
            }
          }
        }
      } else {
        uint32_t base = 0;
        if (lane == 31) base = atomicAdd(qu.size, total);
        base = __shfl_sync(kFull, base, 31);
        unsigned long long p = static_cast<unsigned long long>(base) + excl;
#pragma unroll
        for (int c = 0; c < W; ++c) {
          if ((m >> c) & 1u) {
            if (p < qu.capacity) qu.data[p] = DevPair{sid[c], qid};
            ++p;
          }
        }
      }
      return;
    }
    uint32_t k = n + excl;
#pragma unroll
    for (int c = 0; c < W; ++c) {  // predicated, no divergence
      const uint32_t idx = (static_cast<uint32_t>(c) + lane) & (W - 1);
      if ((m >> idx) & 1u) {
        buf[k] = DevPair{sid[idx], qid};
        if constexpr (ROUTED) bat[k] = rb;
        ++k;
      }
    }
    n += total;
  }

  // Packet scheme: every lane adds (slot, rid[j]) for each set bit j of hm;
  // rbt[j] = batch of query j in a merged launch.
  __device__ __forceinline__ void add_masks(const DevQueue& qu, uint32_t hm, uint32_t slot,
                                            const uint32_t* rid, const uint32_t* rbt) {
    if (!__any_sync(kFull, hm != 0)) return;
    const uint32_t lane = lane_id();
    const uint32_t cnt = __popc(hm);
    uint32_t total;
    const uint32_t excl = warp_excl_prefix<6>(cnt, total);
    if (n + total > kWarpOutCap) flush(qu);
    if (total > kWarpOutCap) {  // more than a buffer: straight to the queues
      if (hm == 0) return;
      const uint32_t gid = ldg_geom_id(ids + slot);
      if constexpr (ROUTED) {
        while (hm) {
          const uint32_t j = __ffs(hm) - 1;
          hm &= hm - 1;
          const DevQueue Q = routes[rbt[j]];
          const unsigned long long p = atomicAdd(Q.size, 1u);
          if (p < Q.capacity) Q.data[p] = DevPair{gid, __ldg(ident + rid[j])};
        }
      } else {
        unsigned long long p = atomicAdd(qu.size, cnt);
        while (hm) {
          const uint32_t j = __ffs(hm) - 1;
          hm &= hm - 1;
          if (p < qu.capacity) qu.data[p] = DevPair{gid, rid[j]};
          ++p;
        }
      }
      return;
    }
    uint32_t k = n + excl;
    while (hm) {
      const uint32_t j = __ffs(hm) - 1;
      hm &= hm - 1;
      buf[k] = DevPair{slot, rid[j]};
      if constexpr (ROUTED) bat[k] = rbt[j];
      ++k;
    }
    n += total;
  }

  // Team scheme: each lane has at most one pair (its leaf slot).
  __device__ __forceinline__ void add_one(const DevQueue& qu, bool hit, uint32_t slot,
                                          uint32_t qid, uint32_t rb) {
    const uint32_t bal = __ballot_sync(kFull, hit);
    if (bal == 0) return;
    const uint32_t total = __popc(bal);
    if (n + total > kWarpOutCap) flush(qu);
    if (hit) {
      const uint32_t k = n + __popc(bal & lanemask_lt());
      buf[k] = DevPair{slot, qid};
      if constexpr (ROUTED) bat[k] = rb;
    }
    n += total;
  }
};

// Lane-count reduction for the counting handler, one atomic per warp.
__device__ __forceinline__ void count_flush_warp(unsigned long long* counter,
                                                 unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  if (lane_id() == 0 && v) atomicAdd(counter, v);
}

}  // namespace rts
