// Serving engine: continuous batching over a resident index.
//
// Requests (query batches of any size, and update batches of deletes /
// inserts / updates) are submitted from any host thread and served in
// submission order by one worker thread:
//  - Query requests are cut into parts and packed into launches.  Each launch
//    runs on one of `slots` streams with its own device arena (query buffer,
//    pair buffer, per-part queues and counters, sort scratch); a part is
//    admitted only while the launch's arena has room for its queries and for
//    its estimated pairs (admission by memory headroom).  While one launch
//    runs, the next is packed and launched on another slot, and finished
//    launches copy their pairs back, so requests that arrive while others are
//    on the GPU are admitted as soon as a slot frees.
//  - A part whose pairs exceed its estimate is re-run alone with the exact
//    capacity its counter reported (no pair is lost or duplicated).
//  - An update request is applied on the update stream after every launch
//    issued before it and before every launch issued after it (stream
//    events), so each query sees exactly the updates submitted before it.
// Each part is one batch of the persistent query kernel with its own 0-based
// query ids, so a request's pairs are the same whether it ran alone or in a
// mix; the engine shifts ids by the part's offset in its request.
#include <chrono>
#include <condition_variable>
#include <map>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "rts_index_impl.h"

namespace rts {
namespace {

using Clock = std::chrono::steady_clock;

double now_s() {
  return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

// Pinned host memory that receives every part's pairs straight from the
// device (one DMA, no staging copy); rts_server_take copies them out and
// frees them.  First fit over a free list, 256-byte granules.  A full arena
// holds finished launches back until results are taken (back-pressure).
struct PinnedArena {
  unsigned char* base = nullptr;
  size_t bytes = 0;
  std::map<size_t, size_t> free_;  // offset -> size

  int init(size_t n) {
    n = (n + 255) & ~size_t(255);
    RTS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&base), n));
    bytes = n;
    free_.clear();
    free_[0] = n;
    return RTS_OK;
  }
  void destroy() {
    if (base) cudaFreeHost(base);
    base = nullptr;
  }
  bool alloc(size_t n, size_t* off) {
    n = (n + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *off = it->first;
      size_t rest = it->second - n;
      size_t at = it->first + n;
      free_.erase(it);
      if (rest) free_[at] = rest;
      return true;
    }
    return false;
  }
  void release(size_t off, size_t n) {
    n = (n + 255) & ~size_t(255);
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct Chunk {
  size_t off;     // byte offset in the arena, or ~0 when held in `heap`
  uint64_t n;     // pairs
  std::vector<rts_pair> heap;
};

struct Request {
  uint64_t ticket = 0;
  bool is_update = false;
  int pred = kPoint;
  uint32_t qwidth = 2;          // floats per query
  std::vector<float> q;         // queries (host copy)
  uint64_t n = 0;               // queries
  uint64_t next = 0;            // first query not yet admitted
  uint64_t parts_open = 0;      // admitted parts whose pairs are not back yet
  std::vector<Chunk> out;        // pairs, part by part
  uint64_t n_out = 0;
  std::vector<uint64_t> del;
  std::vector<float> ins;
  std::vector<rts_update_entry> upd;
  uint64_t first_new_id = 0;
  int status = RTS_OK;
  bool done = false;
  bool viewed = false;          // pairs handed out by rts_server_view until release
  double t_submit = 0, t_done = 0;
};

struct Part {
  Request* r = nullptr;
  uint64_t q0 = 0, nq = 0;      // query range of the request
  uint64_t in_off = 0;          // byte offset in the slot's query buffer
  uint64_t out_off = 0;         // pair offset in the slot's pair buffer
  uint64_t cap = 0;             // pairs reserved
  uint32_t count = 0;           // pairs reported
  size_t host_off = 0;          // arena offset of the pairs once copied
  bool heap = false;            // too large for the arena: copied to the heap
};

struct Retry {
  Request* r;
  uint64_t q0, nq, cap;
};

struct Slot {
  cudaStream_t stream = nullptr;
  DevBuf d_in, d_pairs, d_counts, d_queues, d_descs;
  unsigned char* h_in = nullptr;
  rts_pair* h_pairs = nullptr;
  uint32_t* h_counts = nullptr;
  DevQueue* h_queues = nullptr;
  BatchDesc* h_descs = nullptr;
  uint64_t in_cap = 0, pair_cap = 0;
  uint32_t max_parts = 0;
  QueryScratch qs;
  cudaEvent_t ev_counts = nullptr, ev_pairs = nullptr;
  cudaEvent_t ev_start = nullptr, ev_copy0 = nullptr;  // timing: launch start, pair copies start
  cudaGraphExec_t gexec = nullptr;  // replayed launch sequence of an unsorted launch
  std::vector<Part> parts;
  int state = 0;  // 0 free, 1 launched, 2 copying pairs
  bool overflowed = false;  // state 2: some part must run again with its exact size
  bool waited_update = true;
};

}  // namespace
}  // namespace rts

using namespace rts;

struct rts_server {
  rts_index* ix = nullptr;
  rts_server_config cfg{};
  int device = 0;
  std::vector<std::unique_ptr<Slot>> slots;
  PinnedArena arena;
  cudaStream_t update_stream = nullptr;
  cudaEvent_t ev_update = nullptr;
  // pinned staging of update batches, two buffers used in turn; ev_staged[k]
  // is recorded after the copies that read buffer k
  unsigned char* upd_host[2] = {nullptr, nullptr};
  size_t upd_host_bytes[2] = {0, 0};
  cudaEvent_t ev_staged[2] = {nullptr, nullptr};
  bool staged[2] = {false, false};
  int upd_flip = 0;
  bool update_pending_event = false;  // ev_update recorded; slots must wait on it once
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::deque<Retry> retries;
  std::deque<Request*> updates_in_flight;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::thread worker;
  double rate[kNumPreds] = {4.0, 4.0, 4.0, 4.0, 4.0, 4.0};  // pairs per query, per PredKind
  // statistics
  std::vector<double> lat;
  uint64_t queries_done = 0, pairs_done = 0, launches = 0, retried = 0, updates_done = 0;
  uint64_t parts = 0, graph_launches = 0;
  double pack_s = 0, launch_s = 0, copy_s = 0, take_s = 0, update_s = 0, issue_s = 0;
  double t_first = 0, t_last = 0;
  int fatal = RTS_OK;
};

namespace rts {
namespace {

uint64_t qbytes(const Request* r) { return r->qwidth * sizeof(float); }

int slot_init(rts_server* sv, Slot& sl, uint64_t in_bytes, uint64_t pairs, uint32_t max_parts) {
  RTS_CUDA_TRY(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
  cudaStream_t s = sl.stream;
  int rc;
  if ((rc = buf_reserve(sl.d_in, in_bytes, s, false, 0))) return rc;
  if ((rc = buf_reserve(sl.d_pairs, pairs * sizeof(rts_pair), s, false, 0))) return rc;
  if ((rc = buf_reserve(sl.d_counts, max_parts * sizeof(uint32_t), s, false, 0))) return rc;
  if ((rc = buf_reserve(sl.d_queues, max_parts * sizeof(DevQueue), s, false, 0))) return rc;
  if ((rc = buf_reserve(sl.d_descs, max_parts * sizeof(BatchDesc), s, false, 0))) return rc;
  RTS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&sl.h_in), in_bytes));
  RTS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&sl.h_pairs), pairs * sizeof(rts_pair)));
  RTS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&sl.h_counts), max_parts * sizeof(uint32_t)));
  RTS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&sl.h_queues), max_parts * sizeof(DevQueue)));
  RTS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&sl.h_descs), max_parts * sizeof(BatchDesc)));
  RTS_CUDA_TRY(cudaEventCreate(&sl.ev_counts));
  RTS_CUDA_TRY(cudaEventCreate(&sl.ev_pairs));
  RTS_CUDA_TRY(cudaEventCreate(&sl.ev_start));
  RTS_CUDA_TRY(cudaEventCreate(&sl.ev_copy0));
  if ((rc = buf_reserve(sl.qs.work, sizeof(uint32_t), s, false, 0))) return rc;
  // Order scratch for a full slot (so no launch allocates).
  const uint64_t maxq = in_bytes / (2 * sizeof(float));
  if ((rc = buf_reserve(sl.qs.keys_a, maxq * 8, s, false, 0))) return rc;
  if ((rc = buf_reserve(sl.qs.keys_b, maxq * 8, s, false, 0))) return rc;
  if ((rc = buf_reserve(sl.qs.vals, maxq * 4, s, false, 0))) return rc;
  if ((rc = buf_reserve(sl.qs.order, maxq * 4, s, false, 0))) return rc;
  size_t tb = 0;
  if ((rc = query_order_temp_bytes(maxq, max_parts, &tb))) return rc;
  if ((rc = buf_reserve(sl.qs.sort_temp, tb, s, false, 0))) return rc;
  RTS_CUDA_TRY(cudaStreamSynchronize(s));
  sl.in_cap = in_bytes;
  sl.pair_cap = pairs;
  sl.max_parts = max_parts;
  (void)sv;
  return RTS_OK;
}

void slot_free(Slot& sl) {
  if (sl.stream) cudaStreamSynchronize(sl.stream);
  cudaStream_t s = sl.stream;
  buf_free(sl.d_in, s);
  buf_free(sl.d_pairs, s);
  buf_free(sl.d_counts, s);
  buf_free(sl.d_queues, s);
  buf_free(sl.d_descs, s);
  sl.qs.release(s);
  if (s) cudaStreamSynchronize(s);
  if (sl.h_in) cudaFreeHost(sl.h_in);
  if (sl.h_pairs) cudaFreeHost(sl.h_pairs);
  if (sl.h_counts) cudaFreeHost(sl.h_counts);
  if (sl.h_queues) cudaFreeHost(sl.h_queues);
  if (sl.h_descs) cudaFreeHost(sl.h_descs);
  if (sl.ev_counts) cudaEventDestroy(sl.ev_counts);
  if (sl.ev_pairs) cudaEventDestroy(sl.ev_pairs);
  if (sl.gexec) cudaGraphExecDestroy(sl.gexec);
  if (sl.ev_start) cudaEventDestroy(sl.ev_start);
  if (sl.ev_copy0) cudaEventDestroy(sl.ev_copy0);
  if (s) cudaStreamDestroy(s);
}

void finish_request(rts_server* sv, Request* r) {
  r->done = true;
  r->t_done = now_s();
  sv->t_last = r->t_done;
  if (!r->is_update) {
    sv->lat.push_back(r->t_done - r->t_submit);
    sv->queries_done += r->n;
  }
  sv->cv_done.notify_all();
}

// Packs parts into a free slot and launches them.  Returns true if launched.
bool admit_and_launch(rts_server* sv, Slot& sl) {
  rts_index* ix = sv->ix;
  sl.parts.clear();
  uint64_t in_used = 0, pair_used = 0;
  auto add_part = [&](Request* r, uint64_t q0, uint64_t nq, uint64_t cap) {
    Part p;
    p.r = r;
    p.q0 = q0;
    p.nq = nq;
    p.in_off = in_used;
    p.out_off = pair_used;
    p.cap = cap;
    in_used += (nq * qbytes(r) + 15) & ~uint64_t(15);
    pair_used += cap;
    r->parts_open++;
    sl.parts.push_back(p);
  };
  // Overflowed parts first, each with its exact capacity.
  while (!sv->retries.empty() && sl.parts.size() < sl.max_parts) {
    Retry& t = sv->retries.front();
    uint64_t need_in = (t.nq * qbytes(t.r) + 15) & ~uint64_t(15);
    if (in_used + need_in > sl.in_cap || pair_used + t.cap > sl.pair_cap) {
      if (!sl.parts.empty()) break;
      if (t.cap > sl.pair_cap || need_in > sl.in_cap) {
        // Cannot fit even alone: split the query range.
        if (t.nq > 1) {
          Retry a{t.r, t.q0, t.nq / 2, 0}, b{t.r, t.q0 + t.nq / 2, t.nq - t.nq / 2, 0};
          a.cap = std::min<uint64_t>(sl.pair_cap, t.cap);
          b.cap = std::min<uint64_t>(sl.pair_cap, t.cap);
          sv->retries.pop_front();
          sv->retries.push_front(b);
          sv->retries.push_front(a);
          continue;
        }
        t.r->status = RTS_ERR_CAPACITY;  // one query with more pairs than a slot holds
        sv->retries.pop_front();
        if (t.r->parts_open == 0 && t.r->next == t.r->n) finish_request(sv, t.r);
        continue;
      }
    }
    add_part(t.r, t.q0, t.nq, t.cap);
    sv->retries.pop_front();
  }
  // Then requests in submission order, up to the next update.
  while (!sv->pending.empty() && sl.parts.size() < sl.max_parts) {
    Request* r = sv->pending.front();
    if (r->is_update) break;
    uint64_t room_q = (sl.in_cap - in_used) / qbytes(r);
    if (room_q == 0) break;
    uint64_t take = std::min<uint64_t>(r->n - r->next, room_q);
    double rate = sv->rate[r->pred];
    uint64_t room_p = sl.pair_cap - pair_used;
    uint64_t est = static_cast<uint64_t>(static_cast<double>(take) * rate * 1.5) + 64;
    if (est > room_p) {
      // shrink the part to what the pair room supports
      uint64_t t2 = static_cast<uint64_t>(static_cast<double>(room_p > 64 ? room_p - 64 : 0) /
                                          std::max(rate * 1.5, 1e-9));
      if (t2 == 0 && !sl.parts.empty()) break;
      take = std::max<uint64_t>(1, std::min(take, t2));
      est = std::min<uint64_t>(room_p, static_cast<uint64_t>(take * rate * 1.5) + 64);
      if (est == 0) break;
    }
    add_part(r, r->next, take, est);
    r->next += take;
    if (r->next == r->n) sv->pending.pop_front();
  }
  if (sl.parts.empty()) return false;

  cudaStream_t s = sl.stream;
  if (sv->update_pending_event && !sl.waited_update) {
    cudaStreamWaitEvent(s, sv->ev_update, 0);
    sl.waited_update = true;
  }
  const uint32_t np = static_cast<uint32_t>(sl.parts.size());
  const double t_pack0 = now_s();
  auto* d_in = static_cast<unsigned char*>(sl.d_in.ptr);
  auto* d_pairs = static_cast<DevPair*>(sl.d_pairs.ptr);
  auto* d_counts = static_cast<uint32_t*>(sl.d_counts.ptr);
  auto* d_queues = static_cast<DevQueue*>(sl.d_queues.ptr);
  uint64_t total_q = 0;
  for (const Part& p : sl.parts) total_q += p.nq;
  LaunchPlan plan = plan_for(ix, kContains, total_q);
  uint64_t chunks = 0, total = 0;
  for (uint32_t i = 0; i < np; ++i) {
    const Part& p = sl.parts[i];
    std::memcpy(sl.h_in + p.in_off, p.r->q.data() + p.q0 * p.r->qwidth, p.nq * qbytes(p.r));
    sl.h_queues[i] = DevQueue{d_pairs + p.out_off, p.cap, d_counts + i};
    BatchDesc d{};
    d.queries = reinterpret_cast<const float*>(d_in + p.in_off);
    d.arg = d_queues + i;
    d.n = static_cast<uint32_t>(p.nq);
    d.pred = p.r->pred;
    d.mode = kCollect;
    d.chunk_begin = static_cast<uint32_t>(chunks);
    d.order = nullptr;
    d.qbase = 0;
    d.id_offset = static_cast<uint32_t>(p.q0);  // ids relative to the request
    chunks += (p.nq + plan.chunk - 1) / plan.chunk;
    total += p.nq;
    sl.h_descs[i] = d;
  }
  int rc = RTS_OK;
  sv->pack_s += now_s() - t_pack0;
  sv->parts += np;
  const double t_issue0 = now_s();
  const bool sorted = want_sort(ix, total);
  if (sorted) rc = plan_order(sl.qs, plan, sl.h_descs, np, total, chunks, s);
  if (!rc) rc = refresh_forest(ix);
  if (!rc) rc = prepare_query_kernel(plan);  // outside any capture
  cudaEventRecord(sl.ev_start, s);
  const BatchDesc* dd = static_cast<const BatchDesc*>(sl.d_descs.ptr);
  // The launch sequence: inputs in, counters cleared, (visiting order,) the
  // persistent kernel, counts out.
  auto issue = [&]() -> int {
    cudaError_t e = cudaMemcpyAsync(sl.d_in.ptr, sl.h_in, in_used, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sl.d_queues.ptr, sl.h_queues, np * sizeof(DevQueue),
                          cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sl.d_descs.ptr, sl.h_descs, np * sizeof(BatchDesc),
                          cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_counts, 0, np * sizeof(uint32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "server launch staging");
    int r = RTS_OK;
    if (sorted)
      r = fill_order(ix, sl.qs, plan, sl.h_descs, np > 1 ? dd : nullptr, np, total, chunks, s);
    if (!r)
      r = launch_queries(ix->forest, plan, sl.h_descs, np > 1 ? dd : nullptr, np,
                         static_cast<uint32_t>(chunks), static_cast<uint32_t*>(sl.qs.work.ptr), s);
    if (!r) {
      e = cudaMemcpyAsync(sl.h_counts, d_counts, np * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) r = cuda_fail(e, "server launch");
    }
    return r;
  };
  if (!rc && sv->cfg.use_graphs) {
    // CUDA-graph replay: the slot keeps one executable graph of the sequence;
    // each launch records the sequence with its own sizes and arguments and
    // updates the executable graph in place (re-instantiating it only when the
    // sequence's shape changed, e.g. a sort of another number of passes),
    // then replays it.
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) rc = cuda_fail(e, "server graph capture");
    if (!rc) {
      const int r = issue();
      e = cudaStreamEndCapture(s, &g);
      rc = r ? r : (e != cudaSuccess ? cuda_fail(e, "server graph capture") : RTS_OK);
    }
    if (!rc) {
      bool fresh = !sl.gexec;
      if (!fresh) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(sl.gexec, g, &info) != cudaSuccess) {
          cudaGetLastError();
          cudaGraphExecDestroy(sl.gexec);
          sl.gexec = nullptr;
          fresh = true;
        }
      }
      if (fresh && (e = cudaGraphInstantiate(&sl.gexec, g, 0)) != cudaSuccess) {
        sl.gexec = nullptr;
        rc = cuda_fail(e, "server graph instantiate");
      }
      if (!rc && (e = cudaGraphLaunch(sl.gexec, s)) != cudaSuccess)
        rc = cuda_fail(e, "server graph launch");
      if (!rc) sv->graph_launches++;
    }
    if (g) cudaGraphDestroy(g);
  } else if (!rc) {
    rc = issue();
  }
  if (!rc) {
    cudaError_t e = cudaEventRecord(sl.ev_counts, s);
    if (e != cudaSuccess) rc = cuda_fail(e, "server launch");
  }
  sv->issue_s += now_s() - t_issue0;
  if (rc) sv->fatal = rc;
  sl.state = 1;
  sv->launches++;
  return true;
}

// Moves finished launches forward; returns true if anything progressed.
bool poll_slot(rts_server* sv, Slot& sl) {
  if (sl.state == 1) {
    if (cudaEventQuery(sl.ev_counts) != cudaSuccess) return false;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, sl.ev_start, sl.ev_counts) == cudaSuccess) sv->launch_s += 1e-3 * ms;
    // Reserve arena space for every part that fits its capacity; if the arena
    // is full, try again later (results not yet taken hold it).
    std::vector<size_t> got;
    bool ok = true;
    sl.overflowed = false;
    for (size_t i = 0; i < sl.parts.size(); ++i) {
      Part& p = sl.parts[i];
      p.count = sl.h_counts[i];
      p.heap = false;
      sl.overflowed |= p.count > p.cap;
      if (p.count > p.cap || p.count == 0) continue;
      const size_t bytes = p.count * sizeof(rts_pair);
      if (bytes > sv->arena.bytes) {
        p.heap = true;
        continue;
      }
      if (!sv->arena.alloc(bytes, &p.host_off)) {
        ok = false;
        break;
      }
      got.push_back(i);
    }
    if (!ok) {
      for (size_t i : got)
        sv->arena.release(sl.parts[i].host_off, sl.parts[i].count * sizeof(rts_pair));
      return false;
    }
    auto* d_pairs = static_cast<rts_pair*>(sl.d_pairs.ptr);
    cudaEventRecord(sl.ev_copy0, sl.stream);
    for (auto& p : sl.parts) {
      if (p.count > p.cap || p.count == 0 || p.heap) continue;
      cudaMemcpyAsync(sv->arena.base + p.host_off, d_pairs + p.out_off,
                      p.count * sizeof(rts_pair), cudaMemcpyDeviceToHost, sl.stream);
    }
    cudaEventRecord(sl.ev_pairs, sl.stream);
    sl.state = 2;
    return true;
  }
  if (sl.state == 2) {
    if (cudaEventQuery(sl.ev_pairs) != cudaSuccess) return false;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, sl.ev_copy0, sl.ev_pairs) == cudaSuccess) sv->copy_s += 1e-3 * ms;
    auto* d_pairs = static_cast<rts_pair*>(sl.d_pairs.ptr);
    for (auto& p : sl.parts) {
      Request* r = p.r;
      r->parts_open--;
      if (p.count > p.cap) {  // overflow: run this part again with its exact size
        sv->retries.push_back(Retry{r, p.q0, p.nq, p.count});
        sv->retried++;
        continue;
      }
      if (p.count) {
        Chunk c;
        c.n = p.count;
        if (p.heap) {
          c.off = ~size_t(0);
          c.heap.resize(p.count);
          cudaMemcpy(c.heap.data(), d_pairs + p.out_off, p.count * sizeof(rts_pair),
                     cudaMemcpyDeviceToHost);
        } else {
          c.off = p.host_off;
        }
        r->out.push_back(std::move(c));
        r->n_out += p.count;
      }
      sv->pairs_done += p.count;
      if (p.nq) {
        double observed = static_cast<double>(p.count) / static_cast<double>(p.nq);
        double& est = sv->rate[r->pred];
        est = 0.8 * est + 0.2 * std::max(observed, 0.01);
      }
      if (r->parts_open == 0 && r->next == r->n) {
        bool waiting_retry = false;
        for (const Retry& t : sv->retries) waiting_retry |= (t.r == r);
        if (!waiting_retry) finish_request(sv, r);
      }
    }
    sl.parts.clear();
    sl.state = 0;
    return true;
  }
  return false;
}

void release_chunks(rts_server* sv, Request* r) {
  for (auto& c : r->out)
    if (c.off != ~size_t(0)) sv->arena.release(c.off, c.n * sizeof(rts_pair));
  r->out.clear();
}

// The parts of an update batch go through a pinned buffer of the server: a
// copy from the request's pageable vectors would block the worker until the
// driver had staged it, behind whatever pair copies of earlier launches are
// still running.  Two buffers in turn, so an update only waits for the
// copies of the one before the previous.
int stage_update(rts_server* sv, const Request* r, void** d_del, void** d_upd, void** d_ins) {
  cudaStream_t us = sv->update_stream;
  const size_t b_del = r->del.size() * sizeof(uint64_t);
  const size_t b_upd = r->upd.size() * sizeof(rts_update_entry);
  const size_t b_ins = r->ins.size() * sizeof(float);
  const auto al = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  const size_t o_upd = al(b_del), o_ins = o_upd + al(b_upd), total = o_ins + b_ins;
  const int k = sv->upd_flip;
  sv->upd_flip ^= 1;
  if (sv->staged[k]) RTS_CUDA_TRY(cudaEventSynchronize(sv->ev_staged[k]));
  if (total > sv->upd_host_bytes[k]) {
    if (sv->upd_host[k]) cudaFreeHost(sv->upd_host[k]);
    sv->upd_host[k] = nullptr;
    sv->upd_host_bytes[k] = 0;
    const size_t cap = std::max(total, 2 * sv->upd_host_bytes[k ^ 1]);
    RTS_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&sv->upd_host[k]), cap));
    sv->upd_host_bytes[k] = cap;
  }
  unsigned char* h = sv->upd_host[k];
  const struct {
    const void* src;
    size_t bytes, off;
    void** dev;
  } parts[3] = {{r->del.data(), b_del, 0, d_del},
                {r->upd.data(), b_upd, o_upd, d_upd},
                {r->ins.data(), b_ins, o_ins, d_ins}};
  for (const auto& p : parts) {
    *p.dev = nullptr;
    if (!p.bytes) continue;
    std::memcpy(h + p.off, p.src, p.bytes);
    if (int rc = dev_alloc(p.dev, p.bytes, us)) return rc;
    cudaError_t e = cudaMemcpyAsync(*p.dev, h + p.off, p.bytes, cudaMemcpyHostToDevice, us);
    if (e != cudaSuccess) return cuda_fail(e, "staging an update batch");
  }
  RTS_CUDA_TRY(cudaEventRecord(sv->ev_staged[k], us));
  sv->staged[k] = true;
  return RTS_OK;
}

void release_update_staging(rts_server* sv) {
  for (int k = 0; k < 2; ++k) {
    if (sv->ev_staged[k]) {
      if (sv->staged[k]) cudaEventSynchronize(sv->ev_staged[k]);
      cudaEventDestroy(sv->ev_staged[k]);
      sv->ev_staged[k] = nullptr;
    }
    if (sv->upd_host[k]) cudaFreeHost(sv->upd_host[k]);
    sv->upd_host[k] = nullptr;
    sv->upd_host_bytes[k] = 0;
    sv->staged[k] = false;
  }
}

// Applies the update request at the head of the queue.  Called only when no
// launch is in flight and no part waits for a re-run, so every query
// submitted before the update has its final pairs and every later query
// launches after it (its stream waits on ev_update).
void apply_update(rts_server* sv, Request* r) {
  cudaStream_t us = sv->update_stream;
  const double t0 = now_s();
  void *d_del = nullptr, *d_upd = nullptr, *d_ins = nullptr;
  int rc = stage_update(sv, r, &d_del, &d_upd, &d_ins);
  if (!rc && d_del)
    rc = rts_delete(sv->ix, static_cast<const uint64_t*>(d_del), r->del.size(), us);
  if (!rc && d_upd)
    rc = rts_update(sv->ix, static_cast<const rts_update_entry*>(d_upd), r->upd.size(), us);
  r->first_new_id = rts_size(sv->ix);
  if (!rc && d_ins) rc = rts_insert(sv->ix, static_cast<const float*>(d_ins), r->ins.size() / 4, us);
  dev_free(d_del, us);
  dev_free(d_upd, us);
  dev_free(d_ins, us);
  r->status = rc;
  sv->update_s += now_s() - t0;
  cudaEventRecord(sv->ev_update, us);
  sv->update_pending_event = true;
  for (auto& sl : sv->slots) sl->waited_update = false;
  sv->updates_in_flight.push_back(r);
}

void worker_loop(rts_server* sv) {
  cudaSetDevice(sv->device);
  std::unique_lock<std::mutex> lock(sv->mu);
  for (;;) {
    bool progress = false;
    for (auto& sl : sv->slots) progress |= poll_slot(sv, *sl);
    while (!sv->updates_in_flight.empty() &&
           cudaEventQuery(sv->ev_update) == cudaSuccess) {
      Request* r = sv->updates_in_flight.front();
      sv->updates_in_flight.pop_front();
      sv->updates_done++;
      finish_request(sv, r);
      progress = true;
    }
    // An update at the head waits until every earlier launch has finished its
    // kernel and reported its counts (so no part of an earlier query can need
    // a re-run after it); copies of their pairs may still be in flight, as
    // they read the launch's own buffers, not the index.
    bool drained = sv->retries.empty();
    for (auto& sl : sv->slots) drained &= sl->state == 0 || (sl->state == 2 && !sl->overflowed);
    if (!sv->pending.empty() && sv->pending.front()->is_update && drained) {
      Request* r = sv->pending.front();
      sv->pending.pop_front();
      apply_update(sv, r);
      progress = true;
    }
    for (auto& sl : sv->slots)
      if (sl->state == 0 && (!sv->pending.empty() || !sv->retries.empty()) &&
          !(sv->retries.empty() && sv->pending.front()->is_update))
        progress |= admit_and_launch(sv, *sl);
    bool busy = !sv->pending.empty() || !sv->retries.empty() || !sv->updates_in_flight.empty();
    for (auto& sl : sv->slots) busy |= sl->state != 0;
    if (sv->stop && !busy) break;
    if (!progress) {
      if (busy) {
        lock.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lock.lock();
      } else {
        sv->cv_work.wait_for(lock, std::chrono::milliseconds(5));
      }
    }
  }
}

}  // namespace
}  // namespace rts

extern "C" {

int rts_server_config_default(rts_server_config* c) {
  if (!c) return fail(RTS_ERR_INVALID_ARGUMENT, "cfg is null");
  std::memset(c, 0, sizeof(*c));
  c->slots = 3;
  c->max_parts_per_launch = 1024;
  c->max_queries_per_launch = 1u << 20;
  c->pairs_per_launch = 32ull << 20;
  c->hbm_budget_bytes = 0;
  c->host_result_bytes = 1ull << 30;
  c->use_graphs = 1;
  return RTS_OK;
}

int rts_server_create(rts_index* ix, const rts_server_config* cfg, rts_server** out) {
  if (!out) return fail(RTS_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  if (!ix) return fail(RTS_ERR_INVALID_ARGUMENT, "index is null");
  rts_server_config c;
  if (cfg) c = *cfg; else rts_server_config_default(&c);
  if (c.slots < 1 || c.slots > 8) return fail(RTS_ERR_INVALID_ARGUMENT, "slots must be 1..8");
  if (c.max_parts_per_launch < 1 || c.max_queries_per_launch < 1 || c.pairs_per_launch < 1)
    return fail(RTS_ERR_INVALID_ARGUMENT, "launch limits must be positive");
  // Memory budget: every slot's arena must fit in the budget (default: half
  // of the free HBM at creation).
  size_t free_b = 0, total_b = 0;
  RTS_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  uint64_t budget = c.hbm_budget_bytes ? c.hbm_budget_bytes : free_b / 2;
  uint64_t per_slot = c.max_queries_per_launch * 16ull + c.pairs_per_launch * 8ull +
                      c.max_queries_per_launch * 24ull + c.max_parts_per_launch * 96ull;
  if (per_slot * c.slots > budget)
    return fail(RTS_ERR_OUT_OF_MEMORY, "server arenas exceed the HBM budget");
  // The index will take update batches from the request stream: its first
  // ones would grow its slot arrays and reserve its re-sort buffers, an
  // allocation of the index's size inside a request's latency.  Do it now.
  int rc = reserve_for_updates(ix, 0);
  if (rc) return rc;
  RTS_CUDA_TRY(cudaStreamSynchronize(0));
  auto sv = std::make_unique<rts_server>();
  sv->ix = ix;
  sv->cfg = c;
  RTS_CUDA_TRY(cudaGetDevice(&sv->device));
  for (uint32_t i = 0; i < c.slots && !rc; ++i) {
    sv->slots.push_back(std::make_unique<Slot>());
    rc = slot_init(sv.get(), *sv->slots.back(), c.max_queries_per_launch * 16ull,
                   c.pairs_per_launch, c.max_parts_per_launch);
  }
  if (!rc) rc = sv->arena.init(c.host_result_bytes ? c.host_result_bytes : (1ull << 30));
  if (!rc) {
    cudaError_t e = cudaStreamCreateWithFlags(&sv->update_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sv->ev_update, cudaEventDisableTiming);
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
      e = cudaEventCreateWithFlags(&sv->ev_staged[k], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&sv->upd_host[k]), 8u << 20);
      if (e == cudaSuccess) sv->upd_host_bytes[k] = 8u << 20;
    }
    if (e != cudaSuccess) rc = cuda_fail(e, "server streams");
  }
  if (rc) {
    for (auto& sl : sv->slots) slot_free(*sl);
    release_update_staging(sv.get());
    if (sv->ev_update) cudaEventDestroy(sv->ev_update);
    if (sv->update_stream) cudaStreamDestroy(sv->update_stream);
    sv->arena.destroy();
    return rc;
  }
  rts_server* raw = sv.release();
  raw->worker = std::thread(worker_loop, raw);
  *out = raw;
  return RTS_OK;
}

int rts_server_destroy(rts_server* sv) {
  if (!sv) return RTS_OK;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  for (auto& sl : sv->slots) slot_free(*sl);
  if (sv->update_stream) {
    cudaStreamSynchronize(sv->update_stream);
    cudaStreamDestroy(sv->update_stream);
  }
  if (sv->ev_update) cudaEventDestroy(sv->ev_update);
  release_update_staging(sv);
  sv->reqs.clear();
  sv->arena.destroy();
  delete sv;
  return RTS_OK;
}

int rts_server_submit_query(rts_server* sv, int query_kind, int predicate, const float* queries,
                            uint64_t n, uint64_t* ticket) {
  if (!sv || !ticket) return fail(RTS_ERR_INVALID_ARGUMENT, "server or ticket is null");
  if (n && !queries) return fail(RTS_ERR_INVALID_ARGUMENT, "queries is null");
  int pred;
  uint32_t w;  // 4-byte words per query (a double counts as two)
  const bool f64 = query_kind == RTS_QUERY_POINTS_F64 || query_kind == RTS_QUERY_ENVELOPES_F64;
  const bool points = query_kind == RTS_QUERY_POINTS || query_kind == RTS_QUERY_POINTS_F64;
  const bool boxes = query_kind == RTS_QUERY_ENVELOPES || query_kind == RTS_QUERY_ENVELOPES_F64;
  if (points && predicate == RTS_PREDICATE_CONTAINS) {
    pred = f64 ? kPoint64 : kPoint;
    w = f64 ? 4 : 2;
  } else if (boxes && predicate == RTS_PREDICATE_CONTAINS) {
    pred = f64 ? kContains64 : kContains;
    w = f64 ? 8 : 4;
  } else if (boxes && predicate == RTS_PREDICATE_INTERSECTS) {
    pred = f64 ? kIntersects64 : kIntersects;
    w = f64 ? 8 : 4;
  } else {
    return fail(RTS_ERR_INVALID_ARGUMENT, "unsupported query kind / predicate");
  }
  if (f64 != is_f64(sv->ix))
    return fail(RTS_ERR_INVALID_ARGUMENT, f64 ? "double queries on a float index"
                                              : "float queries on a double index");
  if (n > 0xffffffffull) return fail(RTS_ERR_CAPACITY, "more than 2^32-1 queries in a request");
  auto r = std::make_unique<Request>();
  r->pred = pred;
  r->qwidth = w;
  r->n = n;
  r->q.resize(n * w);
  if (n) std::memcpy(r->q.data(), queries, n * w * sizeof(float));
  r->t_submit = now_s();
  std::lock_guard<std::mutex> lock(sv->mu);
  if (sv->fatal) return fail(sv->fatal, "server stopped after an error");
  r->ticket = sv->next_ticket++;
  *ticket = r->ticket;
  if (sv->t_first == 0) sv->t_first = r->t_submit;
  Request* raw = r.get();
  sv->reqs[r->ticket] = std::move(r);
  if (n == 0) {
    finish_request(sv, raw);
  } else {
    sv->pending.push_back(raw);
    sv->cv_work.notify_one();
  }
  return RTS_OK;
}

int rts_server_submit_update(rts_server* sv, const uint64_t* delete_ids, uint64_t n_delete,
                             const float* insert_envelopes, uint64_t n_insert,
                             const rts_update_entry* updates, uint64_t n_update,
                             uint64_t* ticket) {
  if (!sv || !ticket) return fail(RTS_ERR_INVALID_ARGUMENT, "server or ticket is null");
  if ((n_delete && !delete_ids) || (n_insert && !insert_envelopes) || (n_update && !updates))
    return fail(RTS_ERR_INVALID_ARGUMENT, "null update array");
  if (is_f64(sv->ix) && (n_insert || n_update))
    return fail(RTS_ERR_INVALID_ARGUMENT,
                "a served double index takes deletes only; insert and update it before serving");
  auto r = std::make_unique<Request>();
  r->is_update = true;
  r->del.assign(delete_ids, delete_ids + n_delete);
  r->ins.assign(insert_envelopes, insert_envelopes + n_insert * 4);
  r->upd.assign(updates, updates + n_update);
  r->t_submit = now_s();
  std::lock_guard<std::mutex> lock(sv->mu);
  if (sv->fatal) return fail(sv->fatal, "server stopped after an error");
  r->ticket = sv->next_ticket++;
  *ticket = r->ticket;
  if (sv->t_first == 0) sv->t_first = r->t_submit;
  sv->pending.push_back(r.get());
  sv->reqs[r->ticket] = std::move(r);
  sv->cv_work.notify_one();
  return RTS_OK;
}

int rts_server_wait(rts_server* sv, uint64_t ticket, double timeout_s) {
  if (!sv) return fail(RTS_ERR_INVALID_ARGUMENT, "server is null");
  std::unique_lock<std::mutex> lock(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return fail(RTS_ERR_INVALID_ARGUMENT, "unknown ticket");
  Request* r = it->second.get();
  auto until = Clock::now() + std::chrono::duration<double>(timeout_s < 0 ? 1e9 : timeout_s);
  while (!r->done && !sv->fatal) {
    if (sv->cv_done.wait_until(lock, until) == std::cv_status::timeout && !r->done)
      return fail(RTS_ERR_TIMEOUT, "request not done before the timeout");
  }
  if (sv->fatal && !r->done) return fail(sv->fatal, "server stopped after an error");
  return r->status;
}

int rts_server_take(rts_server* sv, uint64_t ticket, rts_pair* out, uint64_t capacity,
                    uint64_t* n_pairs) {
  if (!sv || !n_pairs) return fail(RTS_ERR_INVALID_ARGUMENT, "server or n_pairs is null");
  std::unique_ptr<Request> owned;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return fail(RTS_ERR_INVALID_ARGUMENT, "unknown ticket");
    Request* r = it->second.get();
    if (!r->done) return fail(RTS_ERR_INVALID_ARGUMENT, "request not done");
    if (r->viewed) return fail(RTS_ERR_INVALID_ARGUMENT, "request is viewed: release it");
    *n_pairs = r->is_update ? r->first_new_id : r->n_out;
    if (r->is_update) {
      int st = r->status;
      sv->reqs.erase(it);
      return st;
    }
    if (capacity < r->n_out || (!out && r->n_out))
      return fail(RTS_ERR_QUEUE_FULL, "output capacity smaller than the result");
    owned = std::move(it->second);  // off the ticket table: its arena chunks stay reserved
    sv->reqs.erase(it);
  }
  // The copy runs without the server lock, so the worker keeps launching.
  const double t0 = now_s();
  uint64_t at = 0;
  for (auto& c : owned->out) {
    const rts_pair* src = (c.off == ~size_t(0))
                              ? c.heap.data()
                              : reinterpret_cast<const rts_pair*>(sv->arena.base + c.off);
    std::memcpy(out + at, src, c.n * sizeof(rts_pair));
    at += c.n;
  }
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->take_s += now_s() - t0;
  release_chunks(sv, owned.get());
  return owned->status;
}

int rts_server_view(rts_server* sv, uint64_t ticket, const rts_pair** segments,
                    uint64_t* segment_pairs, uint32_t max_segments, uint32_t* n_segments,
                    uint64_t* n_pairs) {
  if (!sv || !n_segments || !n_pairs)
    return fail(RTS_ERR_INVALID_ARGUMENT, "server, n_segments or n_pairs is null");
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return fail(RTS_ERR_INVALID_ARGUMENT, "unknown ticket");
  Request* r = it->second.get();
  if (!r->done) return fail(RTS_ERR_INVALID_ARGUMENT, "request not done");
  if (r->is_update) return fail(RTS_ERR_INVALID_ARGUMENT, "an update ticket has no pairs");
  *n_pairs = r->n_out;
  *n_segments = static_cast<uint32_t>(r->out.size());
  if (r->out.size() > max_segments)
    return fail(RTS_ERR_QUEUE_FULL, "more segments than max_segments");
  if (!r->out.empty() && (!segments || !segment_pairs))
    return fail(RTS_ERR_INVALID_ARGUMENT, "segments or segment_pairs is null");
  for (size_t i = 0; i < r->out.size(); ++i) {
    const Chunk& c = r->out[i];
    segments[i] = (c.off == ~size_t(0))
                      ? c.heap.data()
                      : reinterpret_cast<const rts_pair*>(sv->arena.base + c.off);
    segment_pairs[i] = c.n;
  }
  r->viewed = true;
  return r->status;
}

int rts_server_release(rts_server* sv, uint64_t ticket) {
  if (!sv) return fail(RTS_ERR_INVALID_ARGUMENT, "server is null");
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return fail(RTS_ERR_INVALID_ARGUMENT, "unknown ticket");
  Request* r = it->second.get();
  if (!r->done) return fail(RTS_ERR_INVALID_ARGUMENT, "request not done");
  release_chunks(sv, r);
  sv->reqs.erase(it);
  return RTS_OK;
}

int rts_server_get_stats(rts_server* sv, rts_server_stats* st) {
  if (!sv || !st) return fail(RTS_ERR_INVALID_ARGUMENT, "server or stats is null");
  std::lock_guard<std::mutex> lock(sv->mu);
  std::memset(st, 0, sizeof(*st));
  std::vector<double> l = sv->lat;
  std::sort(l.begin(), l.end());
  auto pct = [&](double q) {
    if (l.empty()) return 0.0;
    size_t i = static_cast<size_t>(q * static_cast<double>(l.size() - 1) + 0.5);
    return l[std::min(i, l.size() - 1)];
  };
  st->requests_done = l.size();
  st->queries_done = sv->queries_done;
  st->pairs_done = sv->pairs_done;
  st->launches = sv->launches;
  st->retried_parts = sv->retried;
  st->updates_done = sv->updates_done;
  st->latency_p50_s = pct(0.50);
  st->latency_p99_s = pct(0.99);
  st->latency_max_s = l.empty() ? 0.0 : l.back();
  st->elapsed_s = (sv->t_last > sv->t_first) ? sv->t_last - sv->t_first : 0.0;
  st->pack_s = sv->pack_s;
  st->launch_s = sv->launch_s;
  st->copy_s = sv->copy_s;
  st->take_s = sv->take_s;
  st->update_s = sv->update_s;
  st->parts = sv->parts;
  st->graph_launches = sv->graph_launches;
  st->issue_s = sv->issue_s;
  return RTS_OK;
}

int rts_server_reset_stats(rts_server* sv) {
  if (!sv) return fail(RTS_ERR_INVALID_ARGUMENT, "server is null");
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->lat.clear();
  sv->queries_done = sv->pairs_done = sv->launches = sv->retried = sv->updates_done = 0;
  sv->parts = sv->graph_launches = 0;
  sv->pack_s = sv->launch_s = sv->copy_s = sv->take_s = sv->update_s = sv->issue_s = 0;
  sv->t_first = sv->t_last = 0;
  return RTS_OK;
}

}  // extern "C"
