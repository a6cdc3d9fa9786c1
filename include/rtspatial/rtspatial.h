// Umbrella header of the rtspatial C++ API on the B200 library.
#ifndef RTSPATIAL_B200_RTSPATIAL_H
#define RTSPATIAL_B200_RTSPATIAL_H
#include "rtspatial/geom/envelope.cuh"
#include "rtspatial/geom/line.cuh"
#include "rtspatial/geom/point.cuh"
#include "rtspatial/spatial_index.cuh"
#include "rtspatial/utils/queue.h"
#include "rtspatial/utils/shared_value.h"
#include "rtspatial/utils/stream.h"
#include "rtspatial/utils/util.h"
#endif
