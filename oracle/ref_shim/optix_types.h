/* TEST INFRASTRUCTURE ONLY — stand-in for the two OptiX 8 POD types that the
 * reference's predicate headers name, so those headers compile on the host
 * without the OptiX SDK.  Layout of OptixAabb: six floats minX, minY, minZ,
 * maxX, maxY, maxZ (the OptiX 8 public header's field order). */
#ifndef RTS_ORACLE_SHIM_OPTIX_TYPES_H
#define RTS_ORACLE_SHIM_OPTIX_TYPES_H
typedef struct OptixAabb {
  float minX, minY, minZ, maxX, maxY, maxZ;
} OptixAabb;
typedef unsigned long long OptixTraversableHandle;
#endif
