/*
 * TEST INFRASTRUCTURE ONLY — bulk driver of the CPU oracle for double
 * indexes (SpatialIndex<double, 2>): brute force over every box, OpenMP over
 * queries, counts or (geom_id, query_id) pairs sorted by (query_id, geom_id).
 *
 * The including file defines, before including this header:
 *   OB64_PFX(name)                symbol prefix of the exported functions
 *   OB64_PRED_POINT(g, px, py)    point-contains (ob_box64* g, doubles)
 *   OB64_PRED_CONTAINS(g, q)      box-contains (ob_box64* g, q)
 *   OB64_PRED_INTERSECTS(g, q)    box-intersects (ob_box64* g, q)
 * so the same loops run over the restated predicates (rts_oracle.c) and the
 * reference's own code (ref_driver.cu).
 */
#ifndef OB64_PFX
#error "define OB64_PFX before including brute64_driver.h"
#endif

#include <stdint.h>
#include <stdlib.h>

#include "rts_predicates.h"

static int OB64_PFX(pred)(const ob_box64* g, int kind, const double* q) {
  if (kind == 0) return OB64_PRED_POINT(g, q[0], q[1]);
  if (kind == 1) return OB64_PRED_CONTAINS(g, (const ob_box64*)q);
  return OB64_PRED_INTERSECTS(g, (const ob_box64*)q);
}

/* Runs `kind` (0 point-contains, 1 range-contains, 2 range-intersects) for
 * all queries (2 or 4 doubles each).  per_query (nullable) receives each
 * query's count; pairs (nullable, 2*cap uint32) the pairs when they fit.
 * Returns the total. */
uint64_t OB64_PFX(run)(const ob_box64* boxes, uint64_t nb, int kind, const double* queries,
                       uint64_t nq, uint64_t* per_query, uint32_t* pairs, uint64_t cap,
                       int n_threads) {
  const int width = kind == 0 ? 2 : 4;
  uint64_t* counts = per_query;
  uint64_t total = 0;
  int own = 0;
  if (n_threads <= 0) n_threads = 1;
  if (!counts) {
    counts = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nq ? nq : 1));
    own = 1;
  }
  {
    int64_t q;
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 16) reduction(+ : total)
    for (q = 0; q < (int64_t)nq; q++) {
      uint64_t c = 0, i;
      for (i = 0; i < nb; i++) c += (uint64_t)OB64_PFX(pred)(&boxes[i], kind, queries + width * q);
      counts[q] = c;
      total += c;
    }
  }
  if (pairs && total <= cap) {
    uint64_t* offs = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nq + 1));
    uint64_t qi;
    int64_t q;
    offs[0] = 0;
    for (qi = 0; qi < nq; qi++) offs[qi + 1] = offs[qi] + counts[qi];
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 16)
    for (q = 0; q < (int64_t)nq; q++) {
      uint64_t o = offs[q], i;
      if (counts[q] == 0) continue;
      for (i = 0; i < nb; i++) {
        if (OB64_PFX(pred)(&boxes[i], kind, queries + width * q)) {
          pairs[2 * o] = (uint32_t)i;
          pairs[2 * o + 1] = (uint32_t)q;
          ++o;
        }
      }
    }
    free(offs);
  }
  if (own) free(counts);
  return total;
}

/* Element-wise predicate over n (box, query) pairs. */
void OB64_PFX(eval_pairs)(int kind, const ob_box64* g, const double* q, uint64_t n,
                          uint8_t* out) {
  const int width = kind == 0 ? 2 : 4;
  uint64_t i;
  for (i = 0; i < n; i++) out[i] = (uint8_t)OB64_PFX(pred)(&g[i], kind, q + width * i);
}
