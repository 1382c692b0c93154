/* Stand-in declarations for the OptiX types named by the reference headers
 * compiled on the host (test infrastructure; nothing here is called). */
#ifndef R2_REFSHIM_OPTIX_TYPES_H
#define R2_REFSHIM_OPTIX_TYPES_H
#include <cstdint>
typedef unsigned long long OptixTraversableHandle;
typedef unsigned long long CUdeviceptr;
typedef unsigned int OptixVisibilityMask;
typedef struct OptixProgramGroup_t* OptixProgramGroup;
typedef struct { float minX, minY, minZ, maxX, maxY, maxZ; } OptixAabb;
typedef struct { int dummy; } OptixBuildInput;
typedef int OptixResult;
#define OPTIX_SUCCESS 0
#define OPTIX_SBT_RECORD_ALIGNMENT 16
#define OPTIX_SBT_RECORD_HEADER_SIZE 32
#endif
