// Line (segment) of the rtspatial C++ API: two points, the query type of
// SpatialIndex::Query(Predicate, ArrayView<line_t>, ...).
#ifndef RTSPATIAL_B200_GEOM_LINE_CUH
#define RTSPATIAL_B200_GEOM_LINE_CUH

#include "rtspatial/geom/point.cuh"

namespace rtspatial {

template <typename POINT_T>
class Line {
 public:
  using point_t = POINT_T;
  using coord_t = typename point_t::coord_t;

  Line() = default;
  DEV_HOST Line(const point_t& p1, const point_t& p2) : p1_(p1), p2_(p2) {}

  DEV_HOST_INLINE const point_t& get_p1() const { return p1_; }
  DEV_HOST_INLINE const point_t& get_p2() const { return p2_; }

 private:
  point_t p1_, p2_;
};

}  // namespace rtspatial
#endif
