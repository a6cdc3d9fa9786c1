// Query predicates; the values are the B200 library's RTS_PREDICATE_*.
#ifndef RTSPATIAL_B200_GEOM_PREDICATES_H
#define RTSPATIAL_B200_GEOM_PREDICATES_H

#include "rtspatial_b200.h"

namespace rtspatial {

enum class Predicate {
  kIntersects = RTS_PREDICATE_INTERSECTS,
  kContains = RTS_PREDICATE_CONTAINS,
};

}  // namespace rtspatial
#endif
