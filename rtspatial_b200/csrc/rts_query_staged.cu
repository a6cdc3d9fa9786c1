// Query kernels of the staged scheme (groups moved into shared memory by bulk
// copies), node widths 4, 8 and 16.
#include "rts_query_kernels.cuh"

namespace rts {

QueryKernel query_kernel_staged(const LaunchPlan& p, bool routed) {
  switch (p.width) {
    case 4: return routed ? k_query_staged<4, true> : k_query_staged<4, false>;
    case 8: return routed ? k_query_staged<8, true> : k_query_staged<8, false>;
    case 16: return routed ? k_query_staged<16, true> : k_query_staged<16, false>;
  }
  return nullptr;
}

size_t staged_smem_bytes(int width) {
  switch (width) {
    case 4: return staged_stride<4>() * (kQueryThreads / 32);
    case 8: return staged_stride<8>() * (kQueryThreads / 32);
    case 16: return staged_stride<16>() * (kQueryThreads / 32);
  }
  return 0;
}

}  // namespace rts
