/*
 * TEST INFRASTRUCTURE ONLY — generators of the reference's known-answer-test
 * inputs.  The reference's tests draw their boxes and points with libstdc++'s
 * std::mt19937 seeded by the element count and std::uniform_real_distribution
 * (test/test_commons.h:22-67); using the same standard-library engine and
 * distribution here yields the same float streams, so the KAT counts
 * (4 224 111 and 6 549 771) apply to these arrays.
 */
#include <algorithm>
#include <cstdint>
#include <random>
#include <vector>

extern "C" {

/* Boxes: x, y ~ U[0,1); w ~ U[0,max_w); h ~ U[0,max_h); max = min(min+w, 1).
 * Draw order per box: x, y, w, h (test/test_commons.h:36-47). */
void ob_fix_uniform_boxes(uint64_t n, float max_w, float max_h, float* out) {
  std::mt19937 mt(static_cast<std::mt19937::result_type>(n));
  std::uniform_real_distribution<float> dx(0.0, 1.0), dy(0.0, 1.0);
  std::uniform_real_distribution<float> dw(0.0, max_w), dh(0.0, max_h);
  for (uint64_t i = 0; i < n; i++) {
    float x = dx(mt), y = dy(mt), w = dw(mt), h = dh(mt);
    out[4 * i + 0] = x;
    out[4 * i + 1] = y;
    out[4 * i + 2] = std::min(x + w, 1.0f);
    out[4 * i + 3] = std::min(y + h, 1.0f);
  }
}

/* Points: x, y ~ U[0,1) (test/test_commons.h:51-67). */
void ob_fix_uniform_points(uint64_t n, float* out) {
  std::mt19937 mt(static_cast<std::mt19937::result_type>(n));
  std::uniform_real_distribution<float> gx(0.0, 1.0), gy(0.0, 1.0);
  for (uint64_t i = 0; i < n; i++) {
    float x = gx(mt), y = gy(mt);
    out[2 * i + 0] = x;
    out[2 * i + 1] = y;
  }
}

/* The update test's id selection (test/test_envelope_queries.h:120-134):
 * n_updates distinct ids drawn from uniform_int_distribution<size_t>(0, n1-1)
 * with std::mt19937(n_updates); ids are returned in acceptance order. */
void ob_fix_update_ids(uint64_t n1, uint64_t n_updates, uint64_t* out) {
  std::mt19937 mt(static_cast<std::mt19937::result_type>(n_updates));
  std::uniform_int_distribution<size_t> id_dist(0, n1 - 1);
  std::vector<uint8_t> seen(n1, 0);
  uint64_t k = 0;
  while (k < n_updates) {
    size_t id = id_dist(mt);
    if (!seen[id]) {
      seen[id] = 1;
      out[k++] = id;
    }
  }
}
}
