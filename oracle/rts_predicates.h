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

/* ---- double-precision index (SpatialIndex<double, 2>) -------------------- */

typedef struct {
  double minx, miny, maxx, maxy;
} ob_box64; /* layout of Envelope<Point<double,2>> */

/* Point<double,2>::get_coordinate returns float (geom/point.cuh:68-71), and
 * Envelope::Contains compares get_coordinate values (geom/envelope.cuh:29-53):
 * a double index's contains predicates compare the coordinates rounded to the
 * nearest float. */
static inline int ob_contains_point64(const ob_box64* g, double px, double py) {
  float x = (float)px, y = (float)py;
  return x >= (float)g->minx && x <= (float)g->maxx && y >= (float)g->miny &&
         y <= (float)g->maxy;
}

static inline int ob_contains_box64(const ob_box64* g, const ob_box64* q) {
  return (float)q->minx >= (float)g->minx && (float)q->maxx <= (float)g->maxx &&
         (float)q->miny >= (float)g->miny && (float)q->maxy <= (float)g->maxy;
}

/* Envelope::IsValid uses get_x/get_y, which return double
 * (geom/envelope.cuh:103-105, geom/point.cuh:58-64). */
static inline int ob_is_valid64(const ob_box64* g) {
  return g->minx < g->maxx && g->miny < g->maxy;
}

/* 1 + 2 * DBL_GAMMA(3) evaluated in double (details/ray_params.h:41,283). */
static inline double ob_slab_k64(void) {
  volatile double three_eps = 3 * DBL_EPSILON;
  volatile double gamma3 = three_eps / (1 - three_eps);
  volatile double k = 1 + 2 * gamma3;
  return k;
}

/* RayParams<double,2>::IsHit (details/ray_params.h:260-290): the slab test in
 * double; its t1 start value is nextafterf(1.0, DBL_MAX), a float function,
 * i.e. 1 + 2^-23 (OB_T1) widened to double. */
static inline int ob_ray_hit64(double ox, double oy, double dx, double dy,
                               const ob_box64* b, double k) {
  double t0 = 0.0, t1 = (double)OB_T1;
  double inv, tn, tf, tmp;

  inv = 1.0 / dx;
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

  inv = 1.0 / dy;
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

/* Range-intersects result set of a double index: the same two-pass
 * composition as ob_intersects (shaders_intersects_envelope_query_2d.cu
 * compiled with FLOAT_TYPE = double), with RayParams<double,2>::Compute
 * (details/ray_params.h:193-210) and IsHit in double. */
static inline int ob_intersects64(const ob_box64* g, const ob_box64* q, double k) {
  double gdx = g->maxx - g->minx;
  double gdy = g->maxy - g->miny;
  if (ob_ray_hit64(g->minx, g->miny, gdx, gdy, q, k)) return ob_is_valid64(g);
  {
    double qdx = q->minx - q->maxx;
    double qdy = q->maxy - q->miny;
    return ob_ray_hit64(q->maxx, q->miny, qdx, qdy, g, k);
  }
}

static inline void ob_invalidate64(ob_box64* g) {
  g->maxx = g->minx;
  g->maxy = g->miny;
}

#endif /* RTS_ORACLE_PREDICATES_H */
