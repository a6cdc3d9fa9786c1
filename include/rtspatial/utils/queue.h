// Output queue of the collecting handler (the reference's utils/queue.h
// interface).  dev::Queue<T> has the member layout the B200 library writes
// through (rts_queue in rtspatial_b200.h): {T* data; size_t capacity;
// uint32_t* size}.  A query never writes past the capacity; its counter still
// counts every pair, so size() > capacity() after a query means the queue was
// too small and size() is the capacity needed.
#ifndef RTSPATIAL_B200_UTILS_QUEUE_H
#define RTSPATIAL_B200_UTILS_QUEUE_H

#include <cstdint>

#include "rtspatial/utils/array_view.h"
#include "rtspatial/utils/shared_value.h"

namespace rtspatial {
namespace dev {

template <typename T>
class Queue {
 public:
  using value_type = T;
  Queue() = default;
  DEV_HOST Queue(const ArrayView<T>& data, uint32_t* last_pos) : data_(data), last_pos_(last_pos) {}

  // Appends one item; items past the capacity are counted but not stored.
  DEV_INLINE uint32_t Append(const T& item) {
    uint32_t at = atomicAdd(last_pos_, 1u);
    if (at < data_.size()) data_[at] = item;
    return at;
  }
  DEV_INLINE T& operator[](uint32_t i) { return data_[i]; }
  DEV_INLINE const T& operator[](uint32_t i) const { return data_[i]; }
  DEV_INLINE uint32_t size() const { return *last_pos_; }
  DEV_INLINE T* data() { return data_.data(); }

 private:
  ArrayView<T> data_;
  uint32_t* last_pos_ = nullptr;
};

}  // namespace dev

template <typename T>
class Queue {
 public:
  using value_type = T;
  using device_t = dev::Queue<T>;

  void Init(uint32_t capacity) {
    data_.resize(capacity);
    counter_.set(0);
  }
  void Clear() { counter_.set(0); }
  void Clear(cudaStream_t stream) { counter_.set(stream, 0); }
  void set_size(cudaStream_t stream, size_t n) { counter_.set(stream, static_cast<uint32_t>(n)); }
  size_t size() const { return counter_.get(); }
  size_t size(cudaStream_t stream) const { return counter_.get(stream); }
  size_t capacity() const { return data_.size(); }
  bool overflowed(cudaStream_t stream) const { return size(stream) > capacity(); }
  T* data() { return thrust::raw_pointer_cast(data_.data()); }
  const T* data() const { return thrust::raw_pointer_cast(data_.data()); }

  // Copies the stored items (at most capacity()) into `out`.
  template <typename VECTOR_T>
  void CopyTo(VECTOR_T& out, cudaStream_t stream) {
    size_t s = size(stream);
    if (s > data_.size()) s = data_.size();
    out.resize(s);
    thrust::copy(data_.begin(), data_.begin() + s, out.begin());
  }

  device_t DeviceObject() { return device_t(ArrayView<T>(data_), counter_.data()); }

 private:
  thrust::device_vector<T> data_;
  SharedValue<uint32_t> counter_;
};

}  // namespace rtspatial
#endif
