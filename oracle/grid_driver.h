/*
 * TEST INFRASTRUCTURE ONLY — bulk driver of the CPU oracle.
 *
 * Evaluates one of the three per-pair predicates over (boxes x queries),
 * either by brute force over every box or behind a uniform grid whose
 * candidate sets are provably supersets of the predicate's result set, and
 * returns counts, (geom_id, query_id) pairs sorted by (query_id, geom_id), or
 * per-query digests of the pair set (run_digest: the sum modulo 2^64 of a
 * 64-bit mix of every pair, independent of the order the pairs are found in,
 * so a GPU result set can be compared without sorting it).
 *
 * The including file defines, before including this header:
 *   OB_PFX(name)                 symbol prefix for the exported functions
 *   OB_PRED_POINT(g, px, py)     point-contains predicate (ob_box* g)
 *   OB_PRED_CONTAINS(g, q)       box-contains predicate (ob_box* g, q)
 *   OB_PRED_INTERSECTS(g, q)     box-intersects predicate (ob_box* g, q)
 * so the same loops run over the restated predicates (rts_oracle.c) and over
 * the reference's own predicate code (ref_driver.cpp).
 *
 * Grid soundness.  Cells are indexed by cell(v) = clamp(floor((v - lo) *
 * inv), 0, G - 1) in double precision, which is monotone in v.
 *  - point-contains: g contains p  =>  g.min <= p <= g.max  =>  cell(p) lies
 *    in [cell(g.min), cell(g.max)]; one cell per query.
 *  - box-contains (q.min <= q.max): g contains q  =>  g contains q's min
 *    corner; one cell per query.  Inverted queries use brute force.
 *  - intersects: the ray-slab predicate can accept a pair whose boxes are
 *    apart by at most 36 * 2^-24 * M per axis (M = largest coordinate
 *    magnitude of the two boxes); the query range is inflated by
 *    2^-17 * M + 2^-120 per axis, then candidates are de-duplicated.
 * Boxes are registered by their hull (min/max of the two stored bounds).
 */
#ifndef OB_PFX
#error "define OB_PFX before including grid_driver.h"
#endif

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "rts_predicates.h"

#ifndef OB_GRID_TYPES_DEFINED
#define OB_GRID_TYPES_DEFINED
enum { OB_KIND_POINT = 0, OB_KIND_CONTAINS = 1, OB_KIND_INTERSECTS = 2 };

typedef struct ob_grid {
  double lox, loy, invx, invy;
  int64_t gx, gy;
  uint64_t* start; /* gx*gy + 1 */
  uint32_t* items; /* box ids, ascending within a cell */
  float magx, magy; /* max |coordinate| over all boxes, per axis */
} ob_grid;

static inline int64_t ob_cell(double v, double lo, double inv, int64_t g) {
  double c = floor((v - lo) * inv);
  if (!(c >= 0)) return 0; /* also catches NaN */
  if (c >= (double)(g - 1)) return g - 1;
  return (int64_t)c;
}

static inline float ob_fmin(float a, float b) { return a < b ? a : b; }
static inline float ob_fmax(float a, float b) { return a > b ? a : b; }
static inline float ob_fabs(float a) { return a < 0 ? -a : a; }

static int ob_cmp_u32(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return (x > y) - (x < y);
}

/* Digest term of one pair: the splitmix64 finaliser (Steele, Lea and Flood,
 * "Fast splittable pseudorandom number generators", OOPSLA 2014; constants of
 * Vigna's published splitmix64) applied to (geom_id << 32 | query_id).  A
 * bijection of the 64-bit key, so distinct pairs give unrelated terms. */
static inline uint64_t ob_pair_mix(uint32_t geom_id, uint32_t query_id) {
  uint64_t x = ((uint64_t)geom_id << 32) | (uint64_t)query_id;
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  x ^= x >> 31;
  return x;
}

/* Cell range of a box's hull. */
static inline void ob_box_cells(const ob_grid* g, const ob_box* b, int64_t* cx0, int64_t* cx1,
                                int64_t* cy0, int64_t* cy1) {
  *cx0 = ob_cell(ob_fmin(b->minx, b->maxx), g->lox, g->invx, g->gx);
  *cx1 = ob_cell(ob_fmax(b->minx, b->maxx), g->lox, g->invx, g->gx);
  *cy0 = ob_cell(ob_fmin(b->miny, b->maxy), g->loy, g->invy, g->gy);
  *cy1 = ob_cell(ob_fmax(b->miny, b->maxy), g->loy, g->invy, g->gy);
}
#endif

/* Builds a grid with about `boxes_per_cell` boxes per cell, with every
 * host thread (OpenMP): bounds by reduction, per-cell counts and the fill by
 * atomic increments, then each cell's ids sorted ascending (the fill order
 * is not deterministic; the sorted cells are). */
ob_grid* OB_PFX(grid_build)(const ob_box* boxes, uint64_t nb,
                            double boxes_per_cell) {
  ob_grid* g = (ob_grid*)calloc(1, sizeof(ob_grid));
  double lox = 1e300, loy = 1e300, hix = -1e300, hiy = -1e300;
  float magx = 0, magy = 0;
  int64_t ncell, c, i;
  uint64_t* cursor;
#pragma omp parallel for reduction(min : lox, loy) reduction(max : hix, hiy, magx, magy)
  for (i = 0; i < (int64_t)nb; i++) {
    const ob_box* b = &boxes[i];
    double x0 = ob_fmin(b->minx, b->maxx), x1 = ob_fmax(b->minx, b->maxx);
    double y0 = ob_fmin(b->miny, b->maxy), y1 = ob_fmax(b->miny, b->maxy);
    if (x0 < lox) lox = x0;
    if (y0 < loy) loy = y0;
    if (x1 > hix) hix = x1;
    if (y1 > hiy) hiy = y1;
    magx = ob_fmax(magx, ob_fmax(ob_fabs(b->minx), ob_fabs(b->maxx)));
    magy = ob_fmax(magy, ob_fmax(ob_fabs(b->miny), ob_fabs(b->maxy)));
  }
  if (nb == 0) {
    lox = loy = 0;
    hix = hiy = 1;
  }
  {
    double side = sqrt((double)(nb ? nb : 1) / (boxes_per_cell > 0 ? boxes_per_cell : 1));
    int64_t n1 = (int64_t)side;
    if (n1 < 1) n1 = 1;
    if (n1 > 8192) n1 = 8192;
    g->gx = g->gy = n1;
  }
  g->lox = lox;
  g->loy = loy;
  g->invx = (hix > lox) ? (double)g->gx / (hix - lox) : 0.0;
  g->invy = (hiy > loy) ? (double)g->gy / (hiy - loy) : 0.0;
  g->magx = magx;
  g->magy = magy;
  ncell = g->gx * g->gy;
  g->start = (uint64_t*)calloc((size_t)ncell + 1, sizeof(uint64_t));
#pragma omp parallel for schedule(static, 4096)
  for (i = 0; i < (int64_t)nb; i++) {
    int64_t cx0, cx1, cy0, cy1, cx, cy;
    ob_box_cells(g, &boxes[i], &cx0, &cx1, &cy0, &cy1);
    for (cy = cy0; cy <= cy1; cy++)
      for (cx = cx0; cx <= cx1; cx++) {
#pragma omp atomic update
        g->start[cy * g->gx + cx + 1]++;
      }
  }
  for (c = 0; c < ncell; c++) g->start[c + 1] += g->start[c];
  g->items = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(g->start[ncell] + 1));
  cursor = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(ncell ? ncell : 1));
  memcpy(cursor, g->start, sizeof(uint64_t) * (size_t)ncell);
#pragma omp parallel for schedule(static, 4096)
  for (i = 0; i < (int64_t)nb; i++) {
    int64_t cx0, cx1, cy0, cy1, cx, cy;
    ob_box_cells(g, &boxes[i], &cx0, &cx1, &cy0, &cy1);
    for (cy = cy0; cy <= cy1; cy++)
      for (cx = cx0; cx <= cx1; cx++) {
        uint64_t at;
#pragma omp atomic capture
        at = cursor[cy * g->gx + cx]++;
        g->items[at] = (uint32_t)i;
      }
  }
  free(cursor);
#pragma omp parallel for schedule(dynamic, 4096)
  for (c = 0; c < ncell; c++) {
    uint64_t a = g->start[c], e = g->start[c + 1], j;
    if (e - a > 32) {
      qsort(g->items + a, (size_t)(e - a), sizeof(uint32_t), ob_cmp_u32);
      continue;
    }
    for (j = a + 1; j < e; j++) { /* insertion sort: most cells hold a few ids */
      uint32_t v = g->items[j];
      uint64_t k = j;
      while (k > a && g->items[k - 1] > v) {
        g->items[k] = g->items[k - 1];
        k--;
      }
      g->items[k] = v;
    }
  }
  return g;
}

void OB_PFX(grid_free)(ob_grid* g) {
  if (!g) return;
  free(g->start);
  free(g->items);
  free(g);
}

/* Evaluates query qi; writes matching geom ids (ascending) to out when out is
 * non-NULL and adds ob_pair_mix(id, rid) of each match to *dig when dig is
 * non-NULL; returns the match count.  scratch grows as the grid path of an
 * intersects query needs for de-duplication. */
#define OB_EMIT(id)                               \
  do {                                            \
    if (out) out[cnt] = (id);                     \
    if (dig) *dig += ob_pair_mix((id), rid);      \
    cnt++;                                        \
  } while (0)
static uint64_t OB_PFX(one_query)(const ob_grid* g, const ob_box* boxes,
                                  uint64_t nb, int kind, const float* queries,
                                  uint64_t qi, uint32_t* out,
                                  uint32_t** scratch, uint64_t* scratch_cap,
                                  float k, uint64_t* dig, uint32_t rid) {
  uint64_t cnt = 0, i;
  (void)k;
  if (kind == OB_KIND_POINT) {
    float px = queries[2 * qi], py = queries[2 * qi + 1];
    if (!g) {
      for (i = 0; i < nb; i++)
        if (OB_PRED_POINT(&boxes[i], px, py)) OB_EMIT((uint32_t)i);
    } else {
      int64_t cx = ob_cell(px, g->lox, g->invx, g->gx);
      int64_t cy = ob_cell(py, g->loy, g->invy, g->gy);
      uint64_t c = (uint64_t)(cy * g->gx + cx), j;
      for (j = g->start[c]; j < g->start[c + 1]; j++) {
        uint32_t id = g->items[j];
        if (OB_PRED_POINT(&boxes[id], px, py)) OB_EMIT(id);
      }
    }
    return cnt;
  } else {
    const ob_box* q = (const ob_box*)(queries + 4 * qi);
    int inverted = !(q->minx <= q->maxx) || !(q->miny <= q->maxy);
    if (!g || (kind == OB_KIND_CONTAINS && inverted)) {
      for (i = 0; i < nb; i++) {
        int hit = (kind == OB_KIND_CONTAINS) ? OB_PRED_CONTAINS(&boxes[i], q)
                                             : OB_PRED_INTERSECTS(&boxes[i], q);
        if (hit) OB_EMIT((uint32_t)i);
      }
      return cnt;
    }
    if (kind == OB_KIND_CONTAINS) {
      int64_t cx = ob_cell(q->minx, g->lox, g->invx, g->gx);
      int64_t cy = ob_cell(q->miny, g->loy, g->invy, g->gy);
      uint64_t c = (uint64_t)(cy * g->gx + cx), j;
      for (j = g->start[c]; j < g->start[c + 1]; j++) {
        uint32_t id = g->items[j];
        if (OB_PRED_CONTAINS(&boxes[id], q)) OB_EMIT(id);
      }
      return cnt;
    } else {
      float mx = ob_fmax(g->magx, ob_fmax(ob_fabs(q->minx), ob_fabs(q->maxx)));
      float my = ob_fmax(g->magy, ob_fmax(ob_fabs(q->miny), ob_fabs(q->maxy)));
      double ex = (double)mx * (1.0 / 131072.0) + 1e-36;
      double ey = (double)my * (1.0 / 131072.0) + 1e-36;
      int64_t cx0 = ob_cell((double)ob_fmin(q->minx, q->maxx) - ex, g->lox, g->invx, g->gx);
      int64_t cx1 = ob_cell((double)ob_fmax(q->minx, q->maxx) + ex, g->lox, g->invx, g->gx);
      int64_t cy0 = ob_cell((double)ob_fmin(q->miny, q->maxy) - ey, g->loy, g->invy, g->gy);
      int64_t cy1 = ob_cell((double)ob_fmax(q->miny, q->maxy) + ey, g->loy, g->invy, g->gy);
      int64_t cx, cy;
      uint64_t n = 0, j, u;
      for (cy = cy0; cy <= cy1; cy++)
        for (cx = cx0; cx <= cx1; cx++) {
          uint64_t c = (uint64_t)(cy * g->gx + cx);
          uint64_t need = n + (g->start[c + 1] - g->start[c]);
          if (need > *scratch_cap) {
            uint64_t cap = need * 2 + 64;
            *scratch = (uint32_t*)realloc(*scratch, sizeof(uint32_t) * cap);
            *scratch_cap = cap;
          }
          for (j = g->start[c]; j < g->start[c + 1]; j++) (*scratch)[n++] = g->items[j];
        }
      if (cx1 > cx0 || cy1 > cy0) qsort(*scratch, (size_t)n, sizeof(uint32_t), ob_cmp_u32);
      for (u = 0; u < n; u++) {
        uint32_t id = (*scratch)[u];
        if (u > 0 && (*scratch)[u - 1] == id) continue;
        if (OB_PRED_INTERSECTS(&boxes[id], q)) OB_EMIT(id);
      }
      return cnt;
    }
  }
}

#undef OB_EMIT

/* Runs `kind` for all queries.  grid == NULL means brute force.
 * per_query (nullable, nq entries) receives each query's count.
 * pairs (nullable, 2*cap uint32) receives (geom_id, query_id) sorted by
 * (query_id, geom_id) when the total fits in cap.  Returns the total. */
uint64_t OB_PFX(run)(const ob_grid* g, const ob_box* boxes, uint64_t nb,
                     int kind, const float* queries, uint64_t nq,
                     uint64_t* per_query, uint32_t* pairs, uint64_t cap,
                     int n_threads) {
  uint64_t* counts = per_query;
  uint64_t total = 0, qi;
  int own = 0;
  float k = ob_slab_k();
  if (n_threads <= 0) n_threads = 1;
  if (!counts && pairs) {
    counts = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nq ? nq : 1));
    own = 1;
  }
#pragma omp parallel num_threads(n_threads) reduction(+ : total)
  {
    uint32_t* scratch = NULL;
    uint64_t scratch_cap = 0;
    int64_t q;
#pragma omp for schedule(dynamic, 64)
    for (q = 0; q < (int64_t)nq; q++) {
      uint64_t c = OB_PFX(one_query)(g, boxes, nb, kind, queries, (uint64_t)q, NULL,
                                     &scratch, &scratch_cap, k, NULL, 0);
      if (counts) counts[q] = c;
      total += c;
    }
    free(scratch);
  }
  if (pairs && total <= cap) {
    uint64_t* offs = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nq + 1));
    offs[0] = 0;
    for (qi = 0; qi < nq; qi++) offs[qi + 1] = offs[qi] + counts[qi];
#pragma omp parallel num_threads(n_threads)
    {
      uint32_t* scratch = NULL;
      uint64_t scratch_cap = 0;
      uint32_t* ids = NULL;
      uint64_t ids_cap = 0;
      int64_t q;
#pragma omp for schedule(dynamic, 64)
      for (q = 0; q < (int64_t)nq; q++) {
        uint64_t c = counts[q], j;
        if (c == 0) continue;
        if (c > ids_cap) {
          ids_cap = c * 2;
          ids = (uint32_t*)realloc(ids, sizeof(uint32_t) * ids_cap);
        }
        OB_PFX(one_query)(g, boxes, nb, kind, queries, (uint64_t)q, ids, &scratch,
                          &scratch_cap, k, NULL, 0);
        for (j = 0; j < c; j++) {
          pairs[2 * (offs[q] + j)] = ids[j];
          pairs[2 * (offs[q] + j) + 1] = (uint32_t)q;
        }
      }
      free(scratch);
      free(ids);
    }
    free(offs);
  }
  if (own) free(counts);
  return total;
}

/* Per-query counts and digests of `kind` over all queries (grid == NULL:
 * brute force).  The digest of query q is the sum modulo 2^64 of
 * ob_pair_mix(geom_id, rid[q]) over its matches (rid == NULL: rid[q] = q),
 * i.e. of the pairs a query call reporting query id rid[q] writes.  Returns
 * the total count. */
uint64_t OB_PFX(run_digest)(const ob_grid* g, const ob_box* boxes, uint64_t nb,
                            int kind, const float* queries, uint64_t nq,
                            const uint32_t* rid, uint64_t* counts,
                            uint64_t* digests, int n_threads) {
  uint64_t total = 0;
  float k = ob_slab_k();
  if (n_threads <= 0) n_threads = 1;
#pragma omp parallel num_threads(n_threads) reduction(+ : total)
  {
    uint32_t* scratch = NULL;
    uint64_t scratch_cap = 0;
    int64_t q;
#pragma omp for schedule(dynamic, 64)
    for (q = 0; q < (int64_t)nq; q++) {
      uint64_t d = 0;
      uint64_t c = OB_PFX(one_query)(g, boxes, nb, kind, queries, (uint64_t)q, NULL,
                                     &scratch, &scratch_cap, k, &d,
                                     rid ? rid[q] : (uint32_t)q);
      if (counts) counts[q] = c;
      if (digests) digests[q] = d;
      total += c;
    }
    free(scratch);
  }
  return total;
}
