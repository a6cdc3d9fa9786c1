// Errors of the rtspatial C++ API: every failing call of the B200 library is
// raised as rtspatial::Exception carrying the library's message.
#ifndef RTSPATIAL_B200_UTILS_EXCEPTION_H
#define RTSPATIAL_B200_UTILS_EXCEPTION_H

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "rtspatial_b200.h"

namespace rtspatial {

class Exception : public std::runtime_error {
 public:
  explicit Exception(const std::string& what) : std::runtime_error(what) {}
};

inline void check_rts(int rc, const char* call) {
  if (rc != RTS_OK)
    throw Exception(std::string(call) + " failed (" + std::to_string(rc) + "): " +
                    rts_last_error());
}

inline void check_cuda(cudaError_t e, const char* call) {
  if (e != cudaSuccess) throw Exception(std::string(call) + ": " + cudaGetErrorString(e));
}

}  // namespace rtspatial

#define RTS_CHECK(call) ::rtspatial::check_rts((call), #call)
#define CUDA_CHECK(call) ::rtspatial::check_cuda((call), #call)
#endif
