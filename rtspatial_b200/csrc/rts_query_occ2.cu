// Query kernels for at least 2 resident blocks of kQueryThreads per SM.
#include "rts_query_kernels.cuh"

namespace rts {

QueryKernel query_kernel_occ2(const LaunchPlan& p, bool routed) {
  return routed ? pick_kernel_occ<2, true>(p) : pick_kernel_occ<2, false>(p);
}

}  // namespace rts
