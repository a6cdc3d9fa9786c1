// Point<float, 2> and Point<double, 2> of the rtspatial C++ API: a float2 /
// double2, the layouts the B200 library reads for point queries.
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

// As in the reference (geom/point.cuh:44-75), get_coordinate of a double
// point returns float: the Envelope predicates compare float-rounded
// coordinates, while get_x / get_y keep the doubles.
template <>
class Point<double, 2> {
 public:
  using coord_t = double;
  static constexpr int n_dims = 2;

  Point() = default;
  DEV_HOST Point(const double2& p) : p_(p) {}
  DEV_HOST Point(double x, double y) : p_{x, y} {}

  DEV_HOST_INLINE double get_x() const { return p_.x; }
  DEV_HOST_INLINE double get_y() const { return p_.y; }
  DEV_HOST_INLINE void set_x(double x) { p_.x = x; }
  DEV_HOST_INLINE void set_y(double y) { p_.y = y; }
  DEV_HOST_INLINE int get_n_dims() const { return n_dims; }
  DEV_HOST_INLINE float get_coordinate(int dim) const {
    return static_cast<float>(dim == 0 ? p_.x : p_.y);
  }

 private:
  double2 p_;
};

static_assert(sizeof(Point<float, 2>) == 8, "Point<float,2> must be two packed floats");
static_assert(sizeof(Point<double, 2>) == 16, "Point<double,2> must be two packed doubles");

}  // namespace rtspatial
#endif
