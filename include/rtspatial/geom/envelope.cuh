// Envelope (axis-aligned box) of the rtspatial C++ API: {min, max} points,
// 16 bytes for float 2-D, the layout the B200 library indexes.  The member
// predicates are closed-interval comparisons; the index's range-intersects
// result set is the reference's ray-slab formulation (see rtspatial_b200.h),
// which Intersects() below only approximates to within float rounding.
#ifndef RTSPATIAL_B200_GEOM_ENVELOPE_CUH
#define RTSPATIAL_B200_GEOM_ENVELOPE_CUH

#include "rtspatial/geom/point.cuh"

namespace rtspatial {

template <typename POINT_T>
class Envelope {
 public:
  using point_t = POINT_T;
  using coord_t = typename point_t::coord_t;
  static constexpr int n_dims = point_t::n_dims;

  Envelope() = default;
  DEV_HOST Envelope(const point_t& min, const point_t& max) : min_(min), max_(max) {}

  DEV_HOST_INLINE const point_t& get_min() const { return min_; }
  DEV_HOST_INLINE const point_t& get_max() const { return max_; }

  DEV_HOST_INLINE bool Contains(const point_t& p) const {
    bool in = true;
    for (int d = 0; d < n_dims; ++d)
      in &= p.get_coordinate(d) >= min_.get_coordinate(d) &&
            p.get_coordinate(d) <= max_.get_coordinate(d);
    return in;
  }
  DEV_HOST_INLINE bool Contains(const Envelope& o) const {
    bool in = true;
    for (int d = 0; d < n_dims; ++d)
      in &= o.min_.get_coordinate(d) >= min_.get_coordinate(d) &&
            o.max_.get_coordinate(d) <= max_.get_coordinate(d);
    return in;
  }
  DEV_HOST_INLINE bool Intersects(const Envelope& o) const {
    bool hit = true;
    for (int d = 0; d < n_dims; ++d)
      hit &= o.min_.get_coordinate(d) <= max_.get_coordinate(d) &&
             o.max_.get_coordinate(d) >= min_.get_coordinate(d);
    return hit;
  }
  // Deletion marker: the box collapses onto its min corner.
  DEV_HOST_INLINE void Invalid() { max_ = min_; }
  DEV_HOST_INLINE bool IsValid() const {
    return min_.get_x() < max_.get_x() && min_.get_y() < max_.get_y();
  }

 private:
  point_t min_, max_;
};

static_assert(sizeof(Envelope<Point<float, 2>>) == 16, "envelopes are 4 packed floats");

}  // namespace rtspatial
#endif
