/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle (plain C + OpenMP) for the
 * rtspatial_b200 parity tests, the bench's CPU baseline and the reference arm
 * when the reference headers were not compiled.  The product path never links
 * or calls it.
 *
 * The predicates are the restatement in rts_predicates.h; the bulk loops are
 * grid_driver.h.  Exported symbols carry the prefix ob_port_.
 */
#include "rts_predicates.h"

#define OB_PFX(name) ob_port_##name
#define OB_PRED_POINT(g, px, py) ob_contains_point((g), (px), (py))
#define OB_PRED_CONTAINS(g, q) ob_contains_box((g), (q))
#define OB_PRED_INTERSECTS(g, q) ob_intersects((g), (q), k)
#include "grid_driver.h"

/* The slab constant 1 + 2*FLT_GAMMA(3) as the oracle evaluates it. */
float ob_port_slab_k(void) { return ob_slab_k(); }

/* Element-wise predicate over n (box, query) pairs: out[i] = pred(g[i], q[i]).
 * kind 0: q is a point (2 floats per entry); 1: contains; 2: intersects. */
void ob_port_eval_pairs(int kind, const ob_box* g, const float* q, uint64_t n,
                        uint8_t* out) {
  float k = ob_slab_k();
  uint64_t i;
  for (i = 0; i < n; i++) {
    if (kind == OB_KIND_POINT)
      out[i] = (uint8_t)ob_contains_point(&g[i], q[2 * i], q[2 * i + 1]);
    else if (kind == OB_KIND_CONTAINS)
      out[i] = (uint8_t)ob_contains_box(&g[i], (const ob_box*)(q + 4 * i));
    else
      out[i] = (uint8_t)ob_intersects(&g[i], (const ob_box*)(q + 4 * i), k);
  }
}

/* Applies Delete semantics (Envelope::Invalid) to ids in a host box array. */
void ob_port_invalidate(ob_box* boxes, const uint64_t* ids, uint64_t n) {
  uint64_t i;
  for (i = 0; i < n; i++) ob_invalidate(&boxes[ids[i]]);
}

/* Double indexes: restated predicates behind the brute-force driver
 * (exported prefix ob64_port_). */
#define OB64_PFX(name) ob64_port_##name
#define OB64_PRED_POINT(g, px, py) ob_contains_point64((g), (px), (py))
#define OB64_PRED_CONTAINS(g, q) ob_contains_box64((g), (q))
#define OB64_PRED_INTERSECTS(g, q) ob_intersects64((g), (q), ob_slab_k64())
#include "brute64_driver.h"

double ob64_port_slab_k(void) { return ob_slab_k64(); }

void ob64_port_invalidate(ob_box64* boxes, const uint64_t* ids, uint64_t n) {
  uint64_t i;
  for (i = 0; i < n; i++) ob_invalidate64(&boxes[ids[i]]);
}
