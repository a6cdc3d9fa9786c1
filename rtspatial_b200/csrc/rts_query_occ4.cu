// Query kernels for at least 4 resident blocks of kQueryThreads per SM.
#include "rts_query_kernels.cuh"

namespace rts {

QueryKernel query_kernel_occ4(const LaunchPlan& p, bool routed) {
  return routed ? pick_kernel_occ<4, true>(p) : pick_kernel_occ<4, false>(p);
}

}  // namespace rts
