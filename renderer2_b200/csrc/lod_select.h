// Screen-space LOD selection of many-instance scenes (see lod_select.cu).
#pragma once
#include <cuda_runtime.h>

#include "r2.h"

namespace r2 {

// Chooses a LOD per tree (index into lods, -1: the mesh); host arrays, the
// selection runs on stream s.
void select_lods(const r2_lod_camera& cam, const r2_lod_volume* lods, uint32_t nlods, const uint32_t* modelFirst,
                 const uint32_t* modelCount, uint32_t nmodels, const double* treePos, const double* treeScaling,
                 const uint32_t* treeModel, uint32_t ntrees, double minLod, double coveredPixels, int32_t* out,
                 cudaStream_t s);

}  // namespace r2
