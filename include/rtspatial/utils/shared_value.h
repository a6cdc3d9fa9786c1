// One value mirrored in device and pinned host memory (the reference's
// utils/shared_value.h interface); the counting handler's argument is
// SharedValue<unsigned long long>::data().
#ifndef RTSPATIAL_B200_UTILS_SHARED_VALUE_H
#define RTSPATIAL_B200_UTILS_SHARED_VALUE_H

#include "rtspatial/utils/exception.h"
#include "rtspatial/utils/util.h"

namespace rtspatial {

template <typename T>
class SharedValue {
 public:
  SharedValue() : d_(1), h_(1) {}

  void set(const T& t) { d_[0] = t; }
  void set(cudaStream_t stream, const T& t) {
    h_[0] = t;
    CUDA_CHECK(cudaMemcpyAsync(data(), thrust::raw_pointer_cast(h_.data()), sizeof(T),
                               cudaMemcpyHostToDevice, stream));
  }
  T get(cudaStream_t stream) const {
    T* h = const_cast<T*>(thrust::raw_pointer_cast(h_.data()));
    CUDA_CHECK(cudaMemcpyAsync(h, data(), sizeof(T), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    return *h;
  }
  T get() const { return d_[0]; }
  T* data() { return thrust::raw_pointer_cast(d_.data()); }
  const T* data() const { return thrust::raw_pointer_cast(d_.data()); }

 private:
  thrust::device_vector<T> d_;
  pinned_vector<T> h_;
};

}  // namespace rtspatial
#endif
