// Non-owning (pointer, size) view, the argument type of every SpatialIndex
// call (the reference's utils/array_view.h interface).
#ifndef RTSPATIAL_B200_UTILS_ARRAY_VIEW_H
#define RTSPATIAL_B200_UTILS_ARRAY_VIEW_H

#include <cstddef>

#include "rtspatial/utils/util.h"

namespace rtspatial {

template <typename T>
class ArrayView {
 public:
  ArrayView() = default;
  template <typename ALLOC_T>
  ArrayView(const thrust::device_vector<T, ALLOC_T>& v)
      : data_(const_cast<T*>(thrust::raw_pointer_cast(v.data()))), size_(v.size()) {}
  template <typename ALLOC_T>
  ArrayView(const thrust::host_vector<T, ALLOC_T>& v)
      : data_(const_cast<T*>(thrust::raw_pointer_cast(v.data()))), size_(v.size()) {}
  DEV_HOST ArrayView(T* data, size_t size) : data_(data), size_(size) {}

  DEV_HOST_INLINE T* data() { return data_; }
  DEV_HOST_INLINE const T* data() const { return data_; }
  DEV_HOST_INLINE size_t size() const { return size_; }
  DEV_HOST_INLINE bool empty() const { return size_ == 0; }
  DEV_HOST_INLINE T& operator[](size_t i) { return data_[i]; }
  DEV_HOST_INLINE const T& operator[](size_t i) const { return data_[i]; }
  DEV_HOST_INLINE T* begin() { return data_; }
  DEV_HOST_INLINE T* end() { return data_ + size_; }
  DEV_HOST_INLINE const T* begin() const { return data_; }
  DEV_HOST_INLINE const T* end() const { return data_ + size_; }

 private:
  T* data_ = nullptr;
  size_t size_ = 0;
};

}  // namespace rtspatial
#endif
