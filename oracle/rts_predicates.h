/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle for the rtspatial_b200 parity tests.
 * Nothing in the product path (the CUDA library, the C-ABI, the Python
 * mirror) includes, links or calls this file.
 *
 * Plain-C restatement of the reference's per-pair predicates for float32 2-D
 * boxes ("envelopes") and points.  Every function names the reference lines
 * it follows (paths relative to the RTSpatial project root).
 *
 * Compile without -ffast-math and with -ffp-contract=off: the intersects
 * predicate depends on IEEE single-precision division and on the absence of
 * fused multiply-add.
 */
#ifndef RTS_ORACLE_PREDICATES_H
#define RTS_ORACLE_PREDICATES_H

#include <float.h>
#include <stdint.h>

typedef struct {
  float minx, miny, maxx, maxy;
} ob_box; /* layout of Envelope<Point<float,2>> (geom/envelope.cuh:107-108) */

typedef struct {
  float x, y;
} ob_point; /* layout of Point<float,2> (geom/point.cuh:40-41) */

/* t1 start value: nextafterf(1.0, FLT_MAX) (details/ray_params.h:139). */
#define OB_T1 1.00000011920928955078125f

/* 1 + 2 * FLT_GAMMA(3) evaluated in float (details/ray_params.h:40,158).
 * FLT_GAMMA(3) = (3*FLT_EPSILON)/(1-3*FLT_EPSILON); all operands are float,
 * so the product rounds to 1 + 6*2^-23 (bits 0x3f800006). */
static inline float ob_slab_k(void) {
  volatile float three_eps = 3 * FLT_EPSILON;
  volatile float gamma3 = three_eps / (1 - three_eps);
  volatile float k = 1 + 2 * gamma3;
  return k;
}

/* Envelope::Contains(point): closed interval per dimension
 * (geom/envelope.cuh:29-38). */
static inline int ob_contains_point(const ob_box* g, float px, float py) {
  return px >= g->minx && px <= g->maxx && py >= g->miny && py <= g->maxy;
}

/* Envelope::Contains(envelope): other.min >= min && other.max <= max per
 * dimension (geom/envelope.cuh:40-53). */
static inline int ob_contains_box(const ob_box* g, const ob_box* q) {
  return q->minx >= g->minx && q->maxx <= g->maxx && q->miny >= g->miny &&
         q->maxy <= g->maxy;
}

/* Envelope::IsValid: strict min < max in x and y (geom/envelope.cuh:103-105).
 */
static inline int ob_is_valid(const ob_box* g) {
  return g->minx < g->maxx && g->miny < g->maxy;
}

/* RayParams<float,2>::IsHit (details/ray_params.h:137-166): PBRT-style slab
 * test of the segment o + t*d, t in [0, nextafterf(1)], with the far slab
 * distance scaled by 1 + 2*gamma(3).  Comparisons against NaN are false, so a
 * slab whose t values are NaN leaves [t0, t1] unchanged, exactly as the
 * reference's ternaries do. */
static inline int ob_ray_hit(float ox, float oy, float dx, float dy,
                             const ob_box* b, float k) {
  float t0 = 0.0f, t1 = OB_T1;
  float inv, tn, tf, tmp;

  inv = 1.0f / dx;
  tn = (b->minx - ox) * inv;
  tf = (b->maxx - ox) * inv;
  if (tn > tf) {
    tmp = tn;
    tn = tf;
    tf = tmp;
  }
  tf = tf * k;
  t0 = tn > t0 ? tn : t0;
  t1 = tf < t1 ? tf : t1;
  if (t0 > t1) return 0;

  inv = 1.0f / dy;
  tn = (b->miny - oy) * inv;
  tf = (b->maxy - oy) * inv;
  if (tn > tf) {
    tmp = tn;
    tn = tf;
    tf = tmp;
  }
  tf = tf * k;
  t0 = tn > t0 ? tn : t0;
  t1 = tf < t1 ? tf : t1;
  if (t0 > t1) return 0;
  return 1;
}

/* Range-intersects result set of the reference, pair (g, q):
 *   backward pass (shaders_intersects_envelope_query_2d.cu:75-129): only for
 *     g.IsValid(); ray = g's main diagonal (RayParams::Compute(g, false),
 *     details/ray_params.h:67-84: o = min, d = max - min), reported when it
 *     hits q;
 *   forward pass (same file :14-73): ray = q's anti-diagonal
 *     (Compute(q, true): o = (q.maxx, q.miny), d = (q.minx - q.maxx,
 *     q.maxy - q.miny)); reported when it hits g and g's main diagonal does
 *     NOT hit q (the de-duplication against the backward pass).
 * Combined: hit2 = IsHit(g main diagonal, q);
 *           result = hit2 ? g.IsValid() : IsHit(q anti-diagonal, g). */
static inline int ob_intersects(const ob_box* g, const ob_box* q, float k) {
  float gdx = g->maxx - g->minx;
  float gdy = g->maxy - g->miny;
  if (ob_ray_hit(g->minx, g->miny, gdx, gdy, q, k)) return ob_is_valid(g);
  {
    float qdx = q->minx - q->maxx;
    float qdy = q->maxy - q->miny;
    return ob_ray_hit(q->maxx, q->miny, qdx, qdy, g, k);
  }
}

/* Envelope::Invalid (geom/envelope.cuh:101): a deleted box keeps its min and
 * collapses max onto it; it stays in the index. */
static inline void ob_invalidate(ob_box* g) {
  g->maxx = g->minx;
  g->maxy = g->miny;
}

#endif /* RTS_ORACLE_PREDICATES_H */
