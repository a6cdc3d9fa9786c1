// Prepared launches: a fixed set of batches whose descriptors are validated
// and staged once, with every scratch buffer sized up front, so that each
// launch enqueues only kernels and memsets — the sequence a CUDA graph can
// capture once and replay.  The batches' query and output buffers are fixed;
// their contents may change between launches.
//
// The captured graph holds the index's sub-tree descriptors as kernel
// arguments.  Delete and Update (refit) keep them valid; Insert, a rebuild or
// Clear change them, and the next launch re-captures.
#include "rts_index_impl.h"

struct rts_plan {
  rts_index* ix = nullptr;
  std::vector<rts::BatchDesc> descs;
  rts::DevBuf ddescs;
  rts::QueryScratch qs;
  rts::LaunchPlan plan;
  uint64_t chunks = 0, total = 0;
  bool sorted = false;
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_version = ~0ull;
};

namespace rts {
namespace {

void drop_graph(rts_plan* p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->exec = nullptr;
  p->graph = nullptr;
  p->graph_version = ~0ull;
}

// The launch sequence: [order keys + sort], work-counter reset, query kernel.
int enqueue(rts_plan* p, cudaStream_t s) {
  rts_index* ix = p->ix;
  int rc = refresh_forest(ix);
  if (rc) return rc;
  const uint32_t nd = static_cast<uint32_t>(p->descs.size());
  const BatchDesc* dd = static_cast<const BatchDesc*>(p->ddescs.ptr);
  if (p->sorted && (rc = fill_order(ix, p->qs, p->plan, p->descs.data(), nd > 1 ? dd : nullptr, nd,
                                    p->total, p->chunks, s)))
    return rc;
  return run_launch(ix, p->qs, p->plan, p->descs.data(), nd > 1 ? dd : nullptr, nd, p->total,
                    p->chunks, s);
}

}  // namespace
}  // namespace rts

using namespace rts;

extern "C" {

int rts_plan_create(rts_index* ix, const rts_batch* batches, uint32_t n_batches, rts_plan** out) {
  if (!out) return fail(RTS_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  if (n_batches && !batches) return fail(RTS_ERR_INVALID_ARGUMENT, "batches is null");
  auto* p = new (std::nothrow) rts_plan();
  if (!p) return fail(RTS_ERR_OUT_OF_MEMORY, "host allocation failed");
  p->ix = ix;
  p->plan = plan_for(ix, launch_pred(batches, n_batches),
                     n_batches ? sum_queries(batches, n_batches) : 0);
  int rc = make_descs(ix, batches, n_batches, p->plan, p->descs, p->chunks);
  if (!rc)
    rc = handler_plan(ix, p->descs.data(), static_cast<uint32_t>(p->descs.size()), p->plan);
  cudaStream_t s = 0;
  for (const auto& d : p->descs) p->total += d.n;
  if (!rc) rc = buf_reserve(p->qs.work, sizeof(uint32_t), s, false, 0);
  p->sorted = !p->descs.empty() && want_sort(ix, p->total);
  if (!rc && p->sorted) {
    p->plan.merged =
        merge_batches(p->plan, p->descs.data(), static_cast<uint32_t>(p->descs.size()));
    p->plan.chunk_order = !p->plan.merged && !p->plan.frontier && p->descs.size() > 1;
    rc = plan_order(p->qs, p->plan, p->descs.data(), static_cast<uint32_t>(p->descs.size()),
                    p->total, p->chunks, s);
    size_t need = 0;
    if (!rc) rc = query_order_temp_bytes(p->total, static_cast<uint32_t>(p->descs.size()), &need);
    if (!rc) rc = buf_reserve(p->qs.sort_temp, need, s, false, 0);
  }
  if (!rc && p->plan.frontier && !p->descs.empty()) rc = reserve_frontier(ix, p->qs, p->total, s);
  if (!rc) rc = prepare_query_kernel(p->plan);
  if (!rc && !p->descs.empty()) {
    size_t bytes = p->descs.size() * sizeof(BatchDesc);
    rc = buf_reserve(p->ddescs, bytes, s, false, 0);
    if (!rc) {
      cudaError_t e = cudaMemcpyAsync(p->ddescs.ptr, p->descs.data(), bytes,
                                      cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) rc = cuda_fail(e, "staging plan descriptors");
    }
  }
  if (rc) {
    rts_plan_destroy(p);
    return rc;
  }
  *out = p;
  return RTS_OK;
}

int rts_plan_launch(rts_plan* p, void* stream, int use_graph) {
  if (!p) return fail(RTS_ERR_INVALID_ARGUMENT, "plan is null");
  if (p->descs.empty() || p->ix->n_ids == 0) return RTS_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!use_graph) return enqueue(p, s);
  if (!p->exec || p->graph_version != p->ix->version) {
    drop_graph(p);
    if (!p->capture_stream)
      RTS_CUDA_TRY(cudaStreamCreateWithFlags(&p->capture_stream, cudaStreamNonBlocking));
    if (int rc = refresh_forest(p->ix)) return rc;
    RTS_CUDA_TRY(cudaStreamBeginCapture(p->capture_stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue(p, p->capture_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(p->capture_stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    p->graph = g;
    RTS_CUDA_TRY(cudaGraphInstantiate(&p->exec, p->graph, 0));
    p->graph_version = p->ix->version;
  }
  RTS_CUDA_TRY(cudaGraphLaunch(p->exec, s));
  return RTS_OK;
}

int rts_plan_destroy(rts_plan* p) {
  if (!p) return RTS_OK;
  drop_graph(p);
  if (p->capture_stream) cudaStreamDestroy(p->capture_stream);
  bool touched = p->ddescs.ptr || p->qs.work.ptr;
  buf_free(p->ddescs, 0);
  p->qs.release(0);
  if (touched) cudaStreamSynchronize(0);
  delete p;
  return RTS_OK;
}

}  // extern "C"
