/*
 * TEST INFRASTRUCTURE ONLY — the reference's own predicate code, compiled for
 * the host from the reference's headers (geom/envelope.cuh,
 * details/ray_params.h) with the OptiX POD stand-ins in ref_shim/, and run
 * through the same bulk loops as the restated oracle (grid_driver.h).
 * Built by oracle/Makefile into oracle/_ref/ only where the reference source
 * tree is present; used to pin the restatement (rts_predicates.h) and, when
 * present, as the bench's CPU reference arm.  Exported prefix: ob_ref_.
 *
 * The reference has no CPU query path.  What is the reference's here is the
 * per-pair arithmetic (Envelope::Contains, RayParams::Compute/IsHit,
 * Envelope::IsValid); the pass composition follows
 * src/shaders/shaders_intersects_envelope_query_2d.cu:14-41 (forward IS:
 * query anti-diagonal hits geom and geom main diagonal misses query) and
 * :75-129 (backward: geom valid and its main diagonal hits query).
 */
#include "rtspatial/details/ray_params.h"
#include "rtspatial/geom/envelope.cuh"

#include "rts_predicates.h"

namespace {
using ref_point_t = rtspatial::Point<float, 2>;
using ref_env_t = rtspatial::Envelope<ref_point_t>;

inline ref_env_t to_env(const ob_box* b) {
  return ref_env_t(ref_point_t(b->minx, b->miny), ref_point_t(b->maxx, b->maxy));
}

inline int ref_contains_point(const ob_box* g, float px, float py) {
  return to_env(g).Contains(ref_point_t(px, py)) ? 1 : 0;
}

inline int ref_contains_box(const ob_box* g, const ob_box* q) {
  return to_env(g).Contains(to_env(q)) ? 1 : 0;
}

// SpatialIndex<double, 2>: Point<double,2>, Envelope<Point<double,2>> and
// RayParams<double,2> (geom/point.cuh:44-75, details/ray_params.h:169-292).
using ref_point64_t = rtspatial::Point<double, 2>;
using ref_env64_t = rtspatial::Envelope<ref_point64_t>;

inline ref_env64_t to_env64(const ob_box64* b) {
  return ref_env64_t(ref_point64_t(b->minx, b->miny), ref_point64_t(b->maxx, b->maxy));
}

inline int ref_contains_point64(const ob_box64* g, double px, double py) {
  return to_env64(g).Contains(ref_point64_t(px, py)) ? 1 : 0;
}

inline int ref_contains_box64(const ob_box64* g, const ob_box64* q) {
  return to_env64(g).Contains(to_env64(q)) ? 1 : 0;
}

inline int ref_intersects64(const ob_box64* g, const ob_box64* q) {
  ref_env64_t ge = to_env64(g), qe = to_env64(q);
  rtspatial::details::RayParams<double, 2> rp;
  rp.Compute(ge, false);
  bool box_hit = rp.IsHit(qe);
  bool backward = ge.IsValid() && box_hit;
  rp.Compute(qe, true);
  bool query_hit = rp.IsHit(ge);
  bool forward = query_hit && !box_hit;
  return (backward || forward) ? 1 : 0;
}

inline int ref_intersects(const ob_box* g, const ob_box* q) {
  ref_env_t ge = to_env(g), qe = to_env(q);
  rtspatial::details::RayParams<float, 2> rp;
  rp.Compute(ge, false);
  bool box_hit = rp.IsHit(qe);
  bool backward = ge.IsValid() && box_hit;
  rp.Compute(qe, true);
  bool query_hit = rp.IsHit(ge);
  bool forward = query_hit && !box_hit;
  return (backward || forward) ? 1 : 0;
}
}  // namespace

extern "C" {
#define OB_PFX(name) ob_ref_##name
#define OB_PRED_POINT(g, px, py) ref_contains_point((g), (px), (py))
#define OB_PRED_CONTAINS(g, q) ref_contains_box((g), (q))
#define OB_PRED_INTERSECTS(g, q) ref_intersects((g), (q))
#include "grid_driver.h"

void ob_ref_eval_pairs(int kind, const ob_box* g, const float* q, uint64_t n,
                       uint8_t* out) {
  for (uint64_t i = 0; i < n; i++) {
    if (kind == OB_KIND_POINT)
      out[i] = (uint8_t)ref_contains_point(&g[i], q[2 * i], q[2 * i + 1]);
    else if (kind == OB_KIND_CONTAINS)
      out[i] = (uint8_t)ref_contains_box(&g[i], (const ob_box*)(q + 4 * i));
    else
      out[i] = (uint8_t)ref_intersects(&g[i], (const ob_box*)(q + 4 * i));
  }
}

/* Envelope::Invalid() applied through the reference's own class. */
void ob_ref_invalidate(ob_box* boxes, const uint64_t* ids, uint64_t n) {
  for (uint64_t i = 0; i < n; i++) {
    ref_env_t e = to_env(&boxes[ids[i]]);
    e.Invalid();
    boxes[ids[i]].minx = e.get_min().get_x();
    boxes[ids[i]].miny = e.get_min().get_y();
    boxes[ids[i]].maxx = e.get_max().get_x();
    boxes[ids[i]].maxy = e.get_max().get_y();
  }
}
}

extern "C" {
#define OB64_PFX(name) ob64_ref_##name
#define OB64_PRED_POINT(g, px, py) ref_contains_point64((g), (px), (py))
#define OB64_PRED_CONTAINS(g, q) ref_contains_box64((g), (q))
#define OB64_PRED_INTERSECTS(g, q) ref_intersects64((g), (q))
#include "brute64_driver.h"

/* Envelope<Point<double,2>>::Invalid() through the reference's own class. */
void ob64_ref_invalidate(ob_box64* boxes, const uint64_t* ids, uint64_t n) {
  for (uint64_t i = 0; i < n; i++) {
    ref_env64_t e = to_env64(&boxes[ids[i]]);
    e.Invalid();
    boxes[ids[i]].minx = e.get_min().get_x();
    boxes[ids[i]].miny = e.get_min().get_y();
    boxes[ids[i]].maxx = e.get_max().get_x();
    boxes[ids[i]].maxy = e.get_max().get_y();
  }
}
}  // extern "C"
