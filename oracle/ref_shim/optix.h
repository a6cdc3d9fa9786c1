/* TEST INFRASTRUCTURE ONLY — see optix_types.h in this folder. */
#ifndef RTS_ORACLE_SHIM_OPTIX_H
#define RTS_ORACLE_SHIM_OPTIX_H
#include "optix_types.h"
#endif
