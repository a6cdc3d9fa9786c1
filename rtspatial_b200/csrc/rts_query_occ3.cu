// Query kernels for at least 3 resident blocks of kQueryThreads per SM.
#include "rts_query_kernels.cuh"

namespace rts {

QueryKernel query_kernel_occ3(const LaunchPlan& p, bool routed) {
  return routed ? pick_kernel_occ<3, true>(p) : pick_kernel_occ<3, false>(p);
}

}  // namespace rts
