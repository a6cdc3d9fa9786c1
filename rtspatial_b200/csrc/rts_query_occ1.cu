// Query kernels for at least 1 resident block of kQueryThreads per SM.
#include "rts_query_kernels.cuh"

namespace rts {

QueryKernel query_kernel_occ1(const LaunchPlan& p, bool routed) {
  return routed ? pick_kernel_occ<1, true>(p) : pick_kernel_occ<1, false>(p);
}

}  // namespace rts
