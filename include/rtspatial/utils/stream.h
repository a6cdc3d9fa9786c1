// RAII CUDA stream (the reference's utils/stream.h interface).
#ifndef RTSPATIAL_B200_UTILS_STREAM_H
#define RTSPATIAL_B200_UTILS_STREAM_H

#include <cuda_runtime.h>

#include "rtspatial/utils/exception.h"

namespace rtspatial {

class Stream {
 public:
  Stream() { CUDA_CHECK(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking)); }
  Stream(const Stream&) = delete;
  Stream& operator=(const Stream&) = delete;
  ~Stream() {
    if (s_) cudaStreamDestroy(s_);
  }
  cudaStream_t cuda_stream() const { return s_; }
  void Sync() const { CUDA_CHECK(cudaStreamSynchronize(s_)); }

 private:
  cudaStream_t s_ = nullptr;
};

}  // namespace rtspatial
#endif
