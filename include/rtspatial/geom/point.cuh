// Point<float, 2> of the rtspatial C++ API: an 8-byte float2, the layout the
// B200 library reads for point queries.
#ifndef RTSPATIAL_B200_GEOM_POINT_CUH
#define RTSPATIAL_B200_GEOM_POINT_CUH

#include <vector_types.h>

#include "rtspatial/utils/util.h"

namespace rtspatial {

template <typename COORD_T, int N_DIMS>
class Point;

template <>
class Point<float, 2> {
 public:
  using coord_t = float;
  static constexpr int n_dims = 2;

  Point() = default;
  DEV_HOST Point(const float2& p) : p_(p) {}
  DEV_HOST Point(float x, float y) : p_{x, y} {}

  DEV_HOST_INLINE float get_x() const { return p_.x; }
  DEV_HOST_INLINE float get_y() const { return p_.y; }
  DEV_HOST_INLINE void set_x(float x) { p_.x = x; }
  DEV_HOST_INLINE void set_y(float y) { p_.y = y; }
  DEV_HOST_INLINE int get_n_dims() const { return n_dims; }
  DEV_HOST_INLINE float get_coordinate(int dim) const { return dim == 0 ? p_.x : p_.y; }

 private:
  float2 p_;
};

static_assert(sizeof(Point<float, 2>) == 8, "Point<float,2> must be two packed floats");

}  // namespace rtspatial
#endif
