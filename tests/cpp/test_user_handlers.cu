// The reference's handler contract through the drop-in C++ API: a handler
// module compiled from a custom header (handlers/histogram_handlers.h: per
// query, the number of matches and the sum of their geom ids) the way
// RTSPATIAL_COMPILE_SHADERS compiles one, loaded by SpatialIndex::Init from
// Config::ptx_root as the reference loads its shader modules, and called once
// per pair by Query.  Inputs are the reference tests' fixtures (std::mt19937
// seeded by the element count), so the Python side rebuilds the same floats
// and checks every query's histogram against the oracle.
//
//   test_user_handlers <module dir> <output file>
//
// Output: for each of the six queries (float: point-contains, range-contains,
// range-intersects; then the same on SpatialIndex<double, 2>), the query
// count n, n uint32 counts, n uint64 id sums.
#include <thrust/device_vector.h>

#include <algorithm>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

#include "handlers/histogram_handlers.h"
#include "rtspatial/rtspatial.h"

using namespace rtspatial;

namespace {

template <typename COORD_T>
std::vector<Envelope<Point<COORD_T, 2>>> uniform_boxes(size_t n, float max_w, float max_h) {
  using point_t = Point<COORD_T, 2>;
  std::mt19937 mt(n);
  std::uniform_real_distribution<float> ux(0.0, 1.0), uy(0.0, 1.0);
  std::uniform_real_distribution<float> uw(0.0, max_w), uh(0.0, max_h);
  std::vector<Envelope<point_t>> out(n);
  for (size_t i = 0; i < n; ++i) {
    float x = ux(mt), y = uy(mt), w = uw(mt), h = uh(mt);
    out[i] = Envelope<point_t>(point_t(x, y),
                               point_t(std::min(x + w, 1.0f), std::min(y + h, 1.0f)));
  }
  return out;
}

template <typename COORD_T>
std::vector<Point<COORD_T, 2>> uniform_points(size_t n) {
  std::mt19937 mt(n);
  std::uniform_real_distribution<float> ux(0.0, 1.0), uy(0.0, 1.0);
  std::vector<Point<COORD_T, 2>> out(n);
  for (size_t i = 0; i < n; ++i) {
    float x = ux(mt), y = uy(mt);
    out[i] = Point<COORD_T, 2>(x, y);
  }
  return out;
}

template <typename INDEX, typename Q>
void histogram_query(INDEX& index, Predicate p, const std::vector<Q>& queries, Stream& s,
                     FILE* out) {
  const size_t n = queries.size();
  thrust::device_vector<Q> dq(queries.begin(), queries.end());
  thrust::device_vector<unsigned int> count(n, 0u);
  thrust::device_vector<unsigned long long> idsum(n, 0ull);
  Histogram h{thrust::raw_pointer_cast(count.data()), thrust::raw_pointer_cast(idsum.data())};
  thrust::device_vector<Histogram> dh(1, h);
  index.Query(p, ArrayView<Q>(dq), thrust::raw_pointer_cast(dh.data()), s.cuda_stream());
  s.Sync();
  std::vector<unsigned int> hc(n);
  std::vector<unsigned long long> hs(n);
  thrust::copy(count.begin(), count.end(), hc.begin());
  thrust::copy(idsum.begin(), idsum.end(), hs.begin());
  const unsigned long long nn = n;
  fwrite(&nn, sizeof(nn), 1, out);
  fwrite(hc.data(), sizeof(unsigned int), n, out);
  fwrite(hs.data(), sizeof(unsigned long long), n, out);
}

template <typename COORD_T>
void run_index(const char* module_dir, FILE* out) {
  using index_t = SpatialIndex<COORD_T, 2>;
  using envelope_t = typename index_t::envelope_t;
  index_t index;
  Config config;
  config.ptx_root = module_dir;  // the handler module's directory, as the reference's PTX root
  index.Init(config);
  Stream s;
  std::vector<envelope_t> boxes = uniform_boxes<COORD_T>(100000, 0.01f, 0.01f);
  thrust::device_vector<envelope_t> env(boxes.begin(), boxes.end());
  index.Insert(ArrayView<envelope_t>(env), s.cuda_stream());
  histogram_query(index, Predicate::kContains, uniform_points<COORD_T>(2000), s, out);
  std::vector<envelope_t> qs = uniform_boxes<COORD_T>(2000, 0.02f, 0.02f);
  histogram_query(index, Predicate::kContains, qs, s, out);
  histogram_query(index, Predicate::kIntersects, qs, s, out);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s <module dir> <output file>\n", argv[0]);
    return 2;
  }
  FILE* out = std::fopen(argv[2], "wb");
  if (!out) return 2;
  try {
    run_index<float>(argv[1], out);
    run_index<double>(argv[1], out);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "failed: %s\n", e.what());
    std::fclose(out);
    return 1;
  }
  std::fclose(out);
  std::printf("user handlers: 6 queries written\n");
  return 0;
}
