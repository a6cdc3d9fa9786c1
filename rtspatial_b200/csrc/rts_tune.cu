// Autotuner of the query launch: times candidate (node width, traversal
// scheme, register cap, visiting order, chunk size) settings on the caller's
// batches and keeps the fastest in the index.
//
// The sample runs through the tuner's own counters and queues (a counting
// pass sizes a pair buffer, then every candidate runs with the collecting
// handler into it), so the caller's handlers and outputs are never touched.
// Node width changes the tree layout: with tune_width the index is re-sorted
// at each candidate width and left at the fastest one.
#include <algorithm>

#include "rts_index_impl.h"

namespace rts {
namespace {

struct Candidate {
  int traversal, occupancy, sort;
  uint32_t chunk;
};

int rebuild_at_width(rts_index* ix, int W, cudaStream_t s) {
  if (ix->W == W) return RTS_OK;
  ix->W = W;
  ix->cfg.node_width = W;
  return rebuild_all(ix, s);
}

// Median time (ms) of `reps` launches of the batches under the index's
// current settings.
int time_launches(rts_index* ix, const std::vector<rts_batch>& b, int reps, cudaStream_t s,
                  DevBuf& qsize, uint32_t nb, double* ms) {
  cudaEvent_t e0, e1;
  RTS_CUDA_TRY(cudaEventCreate(&e0));
  RTS_CUDA_TRY(cudaEventCreate(&e1));
  std::vector<float> t;
  int rc = RTS_OK;
  for (int r = 0; r < reps + 1 && !rc; ++r) {
    cudaMemsetAsync(qsize.ptr, 0, nb * sizeof(uint32_t), s);
    cudaEventRecord(e0, s);
    rc = rts_query_batched(ix, b.data(), static_cast<uint32_t>(b.size()), s);
    cudaEventRecord(e1, s);
    cudaError_t e = cudaEventSynchronize(e1);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "autotune launch");
    float v = 0;
    cudaEventElapsedTime(&v, e0, e1);
    if (r > 0) t.push_back(v);  // first launch warms caches and buffers
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return RTS_OK;
}

}  // namespace
}  // namespace rts

using namespace rts;

extern "C" int rts_autotune(rts_index* ix, const rts_batch* batches, uint32_t n_batches,
                            int tune_width, void* stream, rts_tune_result* out) {
  if (!ix || !out) return fail(RTS_ERR_INVALID_ARGUMENT, "index or result is null");
  std::memset(out, 0, sizeof(*out));
  if (n_batches == 0 || ix->n_ids == 0) return RTS_OK;
  if (!batches) return fail(RTS_ERR_INVALID_ARGUMENT, "batches is null");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const rts_config saved = ix->cfg;
  int rc;

  // 1. Counting pass into the tuner's counters.
  DevBuf counts, qsize, queues, pairs;
  auto cleanup = [&]() {
    buf_free(counts, s);
    buf_free(qsize, s);
    buf_free(queues, s);
    buf_free(pairs, s);
    cudaStreamSynchronize(s);
  };
  std::vector<rts_batch> b(batches, batches + n_batches);
  if ((rc = buf_reserve(counts, n_batches * sizeof(unsigned long long), s, false, 0))) return rc;
  RTS_CUDA_TRY(cudaMemsetAsync(counts.ptr, 0, n_batches * sizeof(unsigned long long), s));
  for (uint32_t i = 0; i < n_batches; ++i) {
    b[i].handler = RTS_HANDLER_COUNT;
    b[i].arg = static_cast<unsigned long long*>(counts.ptr) + i;
  }
  if ((rc = rts_query_batched(ix, b.data(), n_batches, s))) {
    cleanup();
    return rc;
  }
  std::vector<unsigned long long> hc(n_batches);
  RTS_CUDA_TRY(cudaMemcpyAsync(hc.data(), counts.ptr, n_batches * 8, cudaMemcpyDeviceToHost, s));
  RTS_CUDA_TRY(cudaStreamSynchronize(s));
  uint64_t total = 0;
  for (auto c : hc) total += c;

  // 2. Collecting queues of exact size (fall back to counting when huge).
  const bool collect = total <= (1ull << 28);
  if (collect) {
    if ((rc = buf_reserve(pairs, std::max<uint64_t>(total, 1) * sizeof(rts_pair), s, false, 0)) ||
        (rc = buf_reserve(qsize, n_batches * sizeof(uint32_t), s, false, 0)) ||
        (rc = buf_reserve(queues, n_batches * sizeof(rts_queue), s, false, 0))) {
      cleanup();
      return rc;
    }
    std::vector<rts_queue> hq(n_batches);
    uint64_t off = 0;
    for (uint32_t i = 0; i < n_batches; ++i) {
      hq[i].data = static_cast<rts_pair*>(pairs.ptr) + off;
      hq[i].capacity = hc[i];
      hq[i].size = static_cast<uint32_t*>(qsize.ptr) + i;
      off += hc[i];
      b[i].handler = RTS_HANDLER_COLLECT;
      b[i].arg = static_cast<rts_queue*>(queues.ptr) + i;
    }
    RTS_CUDA_TRY(cudaMemcpyAsync(queues.ptr, hq.data(), n_batches * sizeof(rts_queue),
                                 cudaMemcpyHostToDevice, s));
    RTS_CUDA_TRY(cudaStreamSynchronize(s));
  } else {
    if ((rc = buf_reserve(qsize, n_batches * sizeof(uint32_t), s, false, 0))) {
      cleanup();
      return rc;
    }
  }

  // 3. Candidates.
  std::vector<int> widths;
  if (tune_width) widths = {4, 8, 16, 32};
  else widths = {ix->W};
  // occupancy 1 = uncapped registers, 2 / 4 = capped for 2 / 4 CTAs per SM
  const Candidate cands[] = {
      {RTS_TRAVERSAL_THREAD, 1, 0, 32},   {RTS_TRAVERSAL_THREAD, 1, 0, 128},
      {RTS_TRAVERSAL_THREAD, 4, 0, 32},   {RTS_TRAVERSAL_THREAD, 4, 0, 64},
      {RTS_TRAVERSAL_THREAD, 4, 0, 128},  {RTS_TRAVERSAL_THREAD, 4, 0, 256},
      {RTS_TRAVERSAL_THREAD, 1, 1, 32},   {RTS_TRAVERSAL_THREAD, 1, 1, 128},
      {RTS_TRAVERSAL_THREAD, 2, 1, 64},   {RTS_TRAVERSAL_THREAD, 2, 0, 64},
      {RTS_TRAVERSAL_THREAD, 2, 1, 128},  {RTS_TRAVERSAL_THREAD, 2, 0, 128},
      {RTS_TRAVERSAL_THREAD, 4, 1, 64},   {RTS_TRAVERSAL_THREAD, 4, 1, 128},
      {RTS_TRAVERSAL_THREAD, 3, 1, 64},   {RTS_TRAVERSAL_THREAD, 3, 1, 128},
      {RTS_TRAVERSAL_TEAM, 1, 1, 64},     {RTS_TRAVERSAL_TEAM, 4, 1, 128},
      {RTS_TRAVERSAL_FRONTIER, 4, 0, 64}, {RTS_TRAVERSAL_FRONTIER, 4, 1, 64},
      {RTS_TRAVERSAL_PACKET, 1, 1, 64},   {RTS_TRAVERSAL_PACKET, 4, 1, 64},
      {RTS_TRAVERSAL_PACKET, 2, 1, 64},   {RTS_TRAVERSAL_PACKET, 4, 1, 256},
      {RTS_TRAVERSAL_PACKET, 3, 1, 64},
      // staged: the occupancy field does not apply (shared memory sets it)
      {RTS_TRAVERSAL_STAGED, 1, 1, 64},   {RTS_TRAVERSAL_STAGED, 1, 1, 128},
      {RTS_TRAVERSAL_STAGED, 1, 0, 128},  {RTS_TRAVERSAL_STAGED, 1, 1, 256},
  };
  double best = 1e300, first = -1;
  int best_w = ix->W;
  Candidate best_c = {saved.traversal, saved.query_occupancy, saved.sort_queries, saved.chunk};
  uint32_t tried = 0;
  for (int W : widths) {
    if ((rc = rebuild_at_width(ix, W, s))) break;
    for (const Candidate& c : cands) {
      if ((c.traversal == RTS_TRAVERSAL_THREAD || c.traversal == RTS_TRAVERSAL_STAGED) && W > 16)
        continue;  // W float4 per lane
      ix->cfg.traversal = c.traversal;
      ix->cfg.query_occupancy = c.occupancy;
      ix->cfg.sort_queries = c.sort;
      ix->cfg.chunk = c.chunk;
      double ms = 0;
      if ((rc = time_launches(ix, b, 3, s, qsize, n_batches, &ms))) break;
      ++tried;
      if (first < 0) first = ms;
      if (ms < best) {
        best = ms;
        best_w = W;
        best_c = c;
      }
    }
    if (rc) break;
  }
  // 4. Keep the winner; for the thread scheme, also its L1 policy of the
  //    group loads (cached or streaming), timed both ways.
  ix->cfg = saved;
  if (!rc) {
    ix->cfg.traversal = best_c.traversal;
    ix->cfg.query_occupancy = best_c.occupancy;
    ix->cfg.sort_queries = best_c.sort;
    ix->cfg.chunk = best_c.chunk;
    rc = rebuild_at_width(ix, best_w, s);
  } else {
    rebuild_at_width(ix, saved.node_width, s);
  }
  if (!rc && best_c.traversal == RTS_TRAVERSAL_THREAD) {
    double pol_ms[2] = {0, 0};
    const int pol[2] = {RTS_LOADS_CACHED, RTS_LOADS_STREAMING};
    for (int i = 0; i < 2 && !rc; ++i) {
      ix->cfg.group_loads = pol[i];
      ix->forest_dirty = true;
      rc = time_launches(ix, b, 3, s, qsize, n_batches, &pol_ms[i]);
      ++tried;
    }
    if (!rc) {
      const int k = pol_ms[1] < pol_ms[0] ? 1 : 0;
      ix->cfg.group_loads = pol[k];
      best = std::min(best, pol_ms[k]);
    }
    ix->forest_dirty = true;
  }
  cleanup();
  if (rc) return rc;
  out->node_width = ix->W;
  out->traversal = ix->cfg.traversal;
  out->query_occupancy = ix->cfg.query_occupancy;
  out->sort_queries = ix->cfg.sort_queries;
  out->chunk = ix->cfg.chunk;
  out->candidates = tried;
  out->best_ms = best;
  out->first_ms = first;
  out->collecting = collect ? 1 : 0;
  out->group_loads = group_loads_streaming(ix, collect) ? RTS_LOADS_STREAMING : RTS_LOADS_CACHED;
  return RTS_OK;
}
