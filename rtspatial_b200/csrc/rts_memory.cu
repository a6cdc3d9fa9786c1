// Device memory of the library: a caching allocator over cudaMalloc, one heap
// per device (the scheme of PyTorch's caching allocator).
//
// Freed blocks are kept.  A request takes the smallest kept block that holds
// it and is at most a quarter (plus 2 MB) larger, else it calls cudaMalloc
// (with an eighth of headroom below 1 GB).
// A block freed on one stream and handed out on another is first waited for
// (cudaStreamWaitEvent on an event recorded at the free), so a buffer is never
// reused before the work queued on it has finished, as with stream-ordered
// allocation.  Memory goes back to the driver only in rts_trim_memory (and
// rts_destroy), after a device synchronisation.
//
// Why not the stream-ordered pools (cudaMallocAsync): measured on B200 under a
// 20M-box index's rounds of deletes, updates and inserts, they were slow and
// erratic exactly on the rounds that merge or re-sort, where the slot arrays
// are swapped or grown: pool growth steps took 6 ms to 1.1 s, and allocations
// that a pool served from memory it already held took up to 0.24 s (free
// memory in pieces is remapped into one range).  cudaMalloc of 10 x 300 MB
// took 3.6 ms, and the re-sorts' swapped arrays come back from the cache.
// cudaMalloc itself still stalls at random (30-110 ms for blocks of 0.3-30 MB
// in the same runs, others of 1.2 GB in 1.4 ms), which is why the index
// reserves what its re-sorts need up front and a warm index allocates nothing.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "rts_internal.h"

namespace rts {

namespace {

constexpr int kMaxDevices = 64;

struct Block {
  void* ptr = nullptr;
  size_t bytes = 0;
  int dev = 0;
  cudaStream_t stream = nullptr;  // the stream of the last allocation or free
  cudaEvent_t freed = nullptr;    // recorded on `stream` at the free
};

struct Heap {
  std::multimap<size_t, Block> free;  // by size
  std::vector<Block> retired;         // freed inside a stream capture
  uint64_t reserved = 0, used = 0;
};

std::mutex g_mu;
Heap g_heap[kMaxDevices];
std::unordered_map<void*, Block> g_live;

size_t round_request(size_t b) {
  const size_t g = b < (1u << 20) ? 512 : (2u << 20);
  return (b + g - 1) / g * g;
}

bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return st != cudaStreamCaptureStatusNone;
}

void release_block(Block& b) {
  cudaFree(b.ptr);
  if (b.freed) cudaEventDestroy(b.freed);
}

// With g_mu held: returns the device's kept blocks to the driver.
int trim_locked(int dev) {
  Heap& h = g_heap[dev];
  if (h.free.empty() && h.retired.empty()) return RTS_OK;
  int cur = 0;
  RTS_CUDA_TRY(cudaGetDevice(&cur));
  if (cur != dev) RTS_CUDA_TRY(cudaSetDevice(dev));
  const cudaError_t e = cudaDeviceSynchronize();  // retired blocks: their graphs may run
  if (e == cudaSuccess) {
    for (auto& kv : h.free) {
      release_block(kv.second);
      h.reserved -= kv.second.bytes;
    }
    for (auto& b : h.retired) {
      release_block(b);
      h.reserved -= b.bytes;
    }
    h.free.clear();
    h.retired.clear();
  }
  if (cur != dev) cudaSetDevice(cur);
  return e == cudaSuccess ? RTS_OK : cuda_fail(e, "cudaDeviceSynchronize (trim)");
}

}  // namespace

int dev_alloc(void** p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  if (bytes == 0) return RTS_OK;
  if (capturing(s)) return fail(RTS_ERR_CUDA, "device allocation inside a stream capture");
  int dev = 0;
  RTS_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(RTS_ERR_INVALID_ARGUMENT, "device out of range");
  const size_t need = round_request(bytes);
  std::lock_guard<std::mutex> lock(g_mu);
  Heap& h = g_heap[dev];
  auto it = h.free.lower_bound(need);
  if (it != h.free.end() && it->first <= need + need / 4 + (2u << 20)) {
    Block b = it->second;
    h.free.erase(it);
    if (b.stream != s) {
      const cudaError_t e = cudaStreamWaitEvent(s, b.freed, 0);
      if (e != cudaSuccess) {
        h.free.emplace(b.bytes, b);
        return cuda_fail(e, "cudaStreamWaitEvent (cached block)");
      }
      b.stream = s;
    }
    h.used += b.bytes;
    g_live[b.ptr] = b;
    *p = b.ptr;
    return RTS_OK;
  }
  // A new block below 1 GB gets an eighth more than asked: buffers that come
  // back a little larger each time (the node buffer of a full re-sort as ids
  // grow, sub-trees of moved updates) then find their freed block big enough.
  const size_t take = need < (1ull << 30) ? round_request(need + need / 8) : need;
  Block b;
  b.bytes = take;
  b.dev = dev;
  b.stream = s;
  cudaError_t e = cudaMalloc(&b.ptr, take);
  if (e == cudaErrorMemoryAllocation) {  // give the kept blocks back and try once more
    cudaGetLastError();
    if (trim_locked(dev) == RTS_OK) {
      b.bytes = need;
      e = cudaMalloc(&b.ptr, need);
    }
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  e = cudaEventCreateWithFlags(&b.freed, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cudaFree(b.ptr);
    return cuda_fail(e, "cudaEventCreate");
  }
  h.reserved += b.bytes;
  h.used += b.bytes;
  g_live[b.ptr] = b;
  *p = b.ptr;
  return RTS_OK;
}

void dev_free(void* p, cudaStream_t s) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_live.find(p);
  if (it == g_live.end()) return;
  Block b = it->second;
  g_live.erase(it);
  Heap& h = g_heap[b.dev];
  h.used -= b.bytes;
  if (capturing(s)) {  // the free is part of a graph: no reuse before a trim
    h.retired.push_back(b);
    return;
  }
  if (cudaEventRecord(b.freed, s) != cudaSuccess) {
    cudaGetLastError();
    h.retired.push_back(b);
    return;
  }
  b.stream = s;
  h.free.emplace(b.bytes, b);
}

int buf_reserve(DevBuf& b, size_t bytes, cudaStream_t s, bool keep, size_t used) {
  if (bytes <= b.bytes && b.ptr) return RTS_OK;
  size_t cap = std::max(bytes, b.bytes + b.bytes / 2);
  cap = (cap + 255) & ~static_cast<size_t>(255);
  void* p = nullptr;
  if (int rc = dev_alloc(&p, cap, s)) return rc;
  if (keep && b.ptr && used) {
    cudaError_t e = cudaMemcpyAsync(p, b.ptr, std::min(used, b.bytes), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) {
      dev_free(p, s);
      return cuda_fail(e, "cudaMemcpyAsync(grow)");
    }
  }
  dev_free(b.ptr, s);
  b.ptr = p;
  b.bytes = cap;
  return RTS_OK;
}

void buf_free(DevBuf& b, cudaStream_t s) {
  dev_free(b.ptr, s);
  b.ptr = nullptr;
  b.bytes = 0;
}

}  // namespace rts

extern "C" {

int rts_memory_pool_stats(int device, uint64_t* reserved, uint64_t* used) {
  if (!reserved || !used) return rts::fail(RTS_ERR_INVALID_ARGUMENT, "null output");
  *reserved = *used = 0;
  if (device < 0 || device >= rts::kMaxDevices)
    return rts::fail(RTS_ERR_INVALID_ARGUMENT, "device out of range");
  std::lock_guard<std::mutex> lock(rts::g_mu);
  *reserved = rts::g_heap[device].reserved;
  *used = rts::g_heap[device].used;
  return RTS_OK;
}

int rts_trim_memory(int device) {
  if (device < 0 || device >= rts::kMaxDevices)
    return rts::fail(RTS_ERR_INVALID_ARGUMENT, "device out of range");
  std::lock_guard<std::mutex> lock(rts::g_mu);
  return rts::trim_locked(device);
}

}  // extern "C"
