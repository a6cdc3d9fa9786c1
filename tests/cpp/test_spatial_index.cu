// The reference's unit tests (test/test_point_queries.h,
// test/test_envelope_queries.h), written against the drop-in C++ API
// (include/rtspatial/*) and run on the B200 library.  Same inputs (libstdc++
// std::mt19937 fixtures seeded by the element count), same calls, same
// expected counts.  Built with RTSPATIAL_COUNTING_HANDLERS, as the reference
// builds its test shaders with the counting handler header.
#include <thrust/device_vector.h>

#include <algorithm>
#include <cstdio>
#include <functional>
#include <random>
#include <string>
#include <unordered_set>
#include <vector>

#include "rtspatial/rtspatial.h"

namespace {

struct Case {
  std::string name;
  std::function<void()> fn;
};
std::vector<Case>& registry() {
  static std::vector<Case> r;
  return r;
}
struct Reg {
  Reg(const char* n, std::function<void()> f) { registry().push_back({n, f}); }
};
#define TEST_CASE(suite, name) \
  void suite##_##name();       \
  Reg reg_##suite##_##name(#suite "." #name, suite##_##name); \
  void suite##_##name()

struct Failure {
  std::string msg;
};
#define EXPECT_EQ_OR_FAIL(a, b)                                                      \
  do {                                                                               \
    auto _a = (a);                                                                   \
    auto _b = (b);                                                                   \
    if (!(_a == _b))                                                                 \
      throw Failure{std::string(#a " == " #b ": ") + std::to_string(_a) + " vs " +   \
                    std::to_string(_b)};                                             \
  } while (0)

using namespace rtspatial;
using index_t = SpatialIndex<float, 2>;
using point_t = index_t::point_t;
using envelope_t = index_t::envelope_t;

SharedValue<unsigned long long>& counter() {
  static SharedValue<unsigned long long> c;
  return c;
}

std::vector<envelope_t> uniform_boxes(size_t n, float max_w, float max_h) {
  std::mt19937 mt(n);
  std::uniform_real_distribution<float> ux(0.0, 1.0), uy(0.0, 1.0);
  std::uniform_real_distribution<float> uw(0.0, max_w), uh(0.0, max_h);
  std::vector<envelope_t> out(n);
  for (size_t i = 0; i < n; ++i) {
    float x = ux(mt), y = uy(mt), w = uw(mt), h = uh(mt);
    out[i] = envelope_t(point_t(x, y), point_t(std::min(x + w, 1.0f), std::min(y + h, 1.0f)));
  }
  return out;
}

std::vector<point_t> uniform_points(size_t n) {
  std::mt19937 mt(n);
  std::uniform_real_distribution<float> ux(0.0, 1.0), uy(0.0, 1.0);
  std::vector<point_t> out(n);
  for (size_t i = 0; i < n; ++i) {
    float x = ux(mt), y = uy(mt);
    out[i] = point_t(x, y);
  }
  return out;
}

template <typename Q>
unsigned long long count_query(index_t& index, Predicate p, ArrayView<Q> q, Stream& s) {
  counter().set(s.cuda_stream(), 0);
  index.Query(p, q, counter().data(), s.cuda_stream());
  return counter().get(s.cuda_stream());
}

void insert_in_batches(index_t& index, thrust::device_vector<envelope_t>& env, int n_batches,
                       Stream& s) {
  size_t avg = (env.size() + n_batches - 1) / n_batches;
  for (int b = 0; b < n_batches; ++b) {
    size_t begin = b * avg, end = std::min(begin + avg, env.size());
    index.Insert(ArrayView<envelope_t>(thrust::raw_pointer_cast(env.data()) + begin, end - begin),
                 s.cuda_stream());
  }
}

TEST_CASE(PointQueries, fp32_contains_point_large) {
  index_t index;
  thrust::device_vector<envelope_t> env = uniform_boxes(100000, 0.5, 0.5);
  thrust::device_vector<point_t> q = uniform_points(1000);
  Stream s;
  Config config;
  index.Init(config);
  index.Insert(ArrayView<envelope_t>(env), s.cuda_stream());
  EXPECT_EQ_OR_FAIL(count_query(index, Predicate::kContains, ArrayView<point_t>(q), s), 4224111ull);
}

TEST_CASE(PointQueries, fp32_contains_point_large_batch) {
  index_t index;
  thrust::device_vector<envelope_t> env = uniform_boxes(100000, 0.5, 0.5);
  thrust::device_vector<point_t> q = uniform_points(1000);
  Stream s;
  Config config;
  index.Init(config);
  insert_in_batches(index, env, 10, s);
  EXPECT_EQ_OR_FAIL(count_query(index, Predicate::kContains, ArrayView<point_t>(q), s), 4224111ull);
}

TEST_CASE(PointQueries, fp32_contains_point) {
  index_t index;
  pinned_vector<envelope_t> env;
  pinned_vector<point_t> pts;
  env.push_back(envelope_t(point_t(0, 0), point_t(1, 1)));
  env.push_back(envelope_t(point_t(0.2, 0.2), point_t(0.8, 0.8)));
  pts.push_back(point_t(0.1, 0.1));
  pts.push_back(point_t(0.5, 0.5));
  pts.push_back(point_t(0.5, 0.6));
  pts.push_back(point_t(1.0, 1.1));
  pts.push_back(point_t(2.0, 2.0));
  Stream s;
  Config config;
  index.Init(config);
  index.Insert(ArrayView<envelope_t>(env), s.cuda_stream());
  EXPECT_EQ_OR_FAIL(count_query(index, Predicate::kContains, ArrayView<point_t>(pts), s), 5ull);
}

TEST_CASE(EnvelopeQueries, fp32_intersects_envelope) {
  index_t index;
  pinned_vector<envelope_t> env, q;
  env.push_back(envelope_t(point_t(0, 0), point_t(1, 1)));
  env.push_back(envelope_t(point_t(0.5, -0.5), point_t(1.5, 0.5)));
  q.push_back(envelope_t(point_t(0.75, 0.25), point_t(1.25, 0.75)));
  Stream s;
  Config config;
  index.Init(config);
  index.Insert(ArrayView<envelope_t>(env), s.cuda_stream());
  EXPECT_EQ_OR_FAIL(count_query(index, Predicate::kIntersects, ArrayView<envelope_t>(q), s), 2ull);
}

TEST_CASE(EnvelopeQueries, fp32_intersects_envelope_big) {
  thrust::device_vector<envelope_t> env = uniform_boxes(100000, 0.5, 0.5);
  thrust::device_vector<envelope_t> q = uniform_boxes(1000, 0.1, 0.1);
  index_t index;
  Stream s;
  Config config;
  index.Init(config);
  index.Insert(ArrayView<envelope_t>(env), s.cuda_stream());
  EXPECT_EQ_OR_FAIL(count_query(index, Predicate::kIntersects, ArrayView<envelope_t>(q), s),
                    6549771ull);
}

TEST_CASE(EnvelopeQueries, fp32_intersects_envelope_batch) {
  thrust::device_vector<envelope_t> env = uniform_boxes(100000, 0.5, 0.5);
  thrust::device_vector<envelope_t> q = uniform_boxes(1000, 0.1, 0.1);
  index_t index;
  Stream s;
  Config config;
  index.Init(config);
  insert_in_batches(index, env, 10, s);
  EXPECT_EQ_OR_FAIL(count_query(index, Predicate::kIntersects, ArrayView<envelope_t>(q), s),
                    6549771ull);
}

TEST_CASE(EnvelopeQueries, fp32_intersects_envelope_batch_update) {
  size_t n1 = 100000;
  thrust::device_vector<envelope_t> env = uniform_boxes(n1, 0.5, 0.5);
  thrust::device_vector<envelope_t> q = uniform_boxes(1000, 0.1, 0.1);
  index_t index;
  Stream s;
  Config config;
  index.Init(config);
  insert_in_batches(index, env, 10, s);
  size_t n_updates = n1 * 0.05;
  std::vector<thrust::pair<size_t, envelope_t>> updates;
  auto new_boxes = uniform_boxes(n_updates, 0.5, 0.5);
  std::unordered_set<size_t> ids;
  std::uniform_int_distribution<size_t> id_dist(0, n1 - 1);
  std::mt19937 mt(n_updates);
  while (ids.size() < n_updates) {
    size_t id = id_dist(mt);
    if (ids.find(id) == ids.end()) {
      updates.push_back(thrust::make_pair(id, new_boxes[ids.size()]));
      ids.insert(id);
    }
  }
  unsigned long long answer;
  {
    index_t fresh;
    pinned_vector<envelope_t> tmp = env;
    for (auto& u : updates) tmp[u.first] = u.second;
    fresh.Init(config);
    fresh.Insert(ArrayView<envelope_t>(tmp), s.cuda_stream());
    answer = count_query(fresh, Predicate::kIntersects, ArrayView<envelope_t>(q), s);
  }
  thrust::device_vector<thrust::pair<size_t, envelope_t>> d_updates = updates;
  index.Update(ArrayView<thrust::pair<size_t, envelope_t>>(d_updates), s.cuda_stream());
  s.Sync();
  EXPECT_EQ_OR_FAIL(count_query(index, Predicate::kIntersects, ArrayView<envelope_t>(q), s),
                    answer);
}

void delete_case(bool compact) {
  index_t index;
  pinned_vector<envelope_t> env, q;
  env.push_back(envelope_t(point_t(0, 0), point_t(1, 1)));
  env.push_back(envelope_t(point_t(0.5, -0.5), point_t(1.5, 0.5)));
  q.push_back(envelope_t(point_t(0.75, 0.25), point_t(1.25, 0.75)));
  Stream s;
  Config config;
  config.compact = compact;
  index.Init(config);
  index.Insert(ArrayView<envelope_t>(env), s.cuda_stream());
  EXPECT_EQ_OR_FAIL(count_query(index, Predicate::kIntersects, ArrayView<envelope_t>(q), s), 2ull);
  thrust::device_vector<size_t> deleted;
  deleted.push_back(1);
  index.Delete(ArrayView<size_t>(deleted), s.cuda_stream());
  s.Sync();
  EXPECT_EQ_OR_FAIL(count_query(index, Predicate::kIntersects, ArrayView<envelope_t>(q), s), 1ull);
}

TEST_CASE(EnvelopeQueries, fp32_test_delete) { delete_case(false); }
TEST_CASE(EnvelopeQueries, fp32_test_delete_compact) { delete_case(true); }

// Collecting handler through rtspatial::Queue (the reference's example path,
// examples/spatial_index.cu:58-67): the queue holds exactly the counted pairs.
TEST_CASE(CollectingQueue, matches_count) {
  thrust::device_vector<envelope_t> env = uniform_boxes(100000, 0.5, 0.5);
  thrust::device_vector<point_t> q = uniform_points(1000);
  Stream s;
  Config config;
  index_t counting;
  counting.Init(config);
  counting.Insert(ArrayView<envelope_t>(env), s.cuda_stream());
  unsigned long long n = count_query(counting, Predicate::kContains, ArrayView<point_t>(q), s);
  config.handler = RTS_HANDLER_COLLECT;
  index_t collecting;
  collecting.Init(config);
  collecting.Insert(ArrayView<envelope_t>(env), s.cuda_stream());
  Queue<thrust::pair<uint32_t, uint32_t>> queue;
  queue.Init(static_cast<uint32_t>(n));
  SharedValue<dev::Queue<thrust::pair<uint32_t, uint32_t>>> dq;
  dq.set(s.cuda_stream(), queue.DeviceObject());
  queue.Clear(s.cuda_stream());
  collecting.Query(Predicate::kContains, ArrayView<point_t>(q), dq.data(), s.cuda_stream());
  EXPECT_EQ_OR_FAIL(static_cast<unsigned long long>(queue.size(s.cuda_stream())), n);
  thrust::host_vector<thrust::pair<uint32_t, uint32_t>> pairs;
  queue.CopyTo(pairs, s.cuda_stream());
  std::unordered_set<unsigned long long> seen;
  for (auto& p : pairs) seen.insert((static_cast<unsigned long long>(p.second) << 32) | p.first);
  EXPECT_EQ_OR_FAIL(static_cast<unsigned long long>(seen.size()), n);
}

// SpatialIndex<double, 2> (test_commons.h:12's spatial_index_d2d_t): the
// point KAT's float inputs widened to double give the same count, since the
// double index's contains compares float-rounded coordinates.
TEST_CASE(PointQueries, fp64_contains_point_large_batch) {
  using dindex_t = SpatialIndex<double, 2>;
  using dpoint_t = dindex_t::point_t;
  using denvelope_t = dindex_t::envelope_t;
  std::vector<envelope_t> envf = uniform_boxes(100000, 0.5, 0.5);
  std::vector<point_t> qf = uniform_points(1000);
  std::vector<denvelope_t> envd(envf.size());
  std::vector<dpoint_t> qd(qf.size());
  for (size_t i = 0; i < envf.size(); ++i)
    envd[i] = denvelope_t(dpoint_t(envf[i].get_min().get_x(), envf[i].get_min().get_y()),
                          dpoint_t(envf[i].get_max().get_x(), envf[i].get_max().get_y()));
  for (size_t i = 0; i < qf.size(); ++i) qd[i] = dpoint_t(qf[i].get_x(), qf[i].get_y());
  thrust::device_vector<denvelope_t> env = envd;
  thrust::device_vector<dpoint_t> q = qd;
  Stream s;
  Config config;
  dindex_t index;
  index.Init(config);
  size_t avg = (env.size() + 9) / 10;
  for (size_t b = 0; b < env.size(); b += avg)
    index.Insert(ArrayView<denvelope_t>(thrust::raw_pointer_cast(env.data()) + b,
                                        std::min(avg, env.size() - b)),
                 s.cuda_stream());
  counter().set(s.cuda_stream(), 0);
  index.Query(Predicate::kContains, ArrayView<dpoint_t>(q), counter().data(), s.cuda_stream());
  EXPECT_EQ_OR_FAIL(counter().get(s.cuda_stream()), 4224111ull);
}

// Line queries: the reference's kIntersects line shader reports nothing (its
// intersection body is commented out), so neither does the drop-in.
TEST_CASE(LineQueries, fp32_line_query_reports_like_the_reference) {
  using line_t = index_t::line_t;
  thrust::device_vector<envelope_t> env = uniform_boxes(10000, 0.5, 0.5);
  std::vector<line_t> lh = {line_t(point_t(0, 0), point_t(1, 1)),
                            line_t(point_t(0.5, 0), point_t(0.5, 1))};
  thrust::device_vector<line_t> lines = lh;
  Stream s;
  Config config;
  index_t index;
  index.Init(config);
  index.Insert(ArrayView<envelope_t>(env), s.cuda_stream());
  for (Predicate p : {Predicate::kIntersects, Predicate::kContains}) {
    counter().set(s.cuda_stream(), 0);
    index.Query(p, ArrayView<line_t>(lines), counter().data(), s.cuda_stream());
    EXPECT_EQ_OR_FAIL(counter().get(s.cuda_stream()), 0ull);
  }
}

}  // namespace

int main() {
  int failed = 0;
  for (auto& c : registry()) {
    try {
      c.fn();
      std::printf("[ OK ] %s\n", c.name.c_str());
    } catch (const Failure& f) {
      ++failed;
      std::printf("[FAIL] %s: %s\n", c.name.c_str(), f.msg.c_str());
    } catch (const std::exception& e) {
      ++failed;
      std::printf("[FAIL] %s: exception %s\n", c.name.c_str(), e.what());
    }
  }
  std::printf("%zu tests, %d failed\n", registry().size(), failed);
  return failed ? 1 : 0;
}
