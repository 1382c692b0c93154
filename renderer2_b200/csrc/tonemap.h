// Frame output stage (see tonemap.cu).
#pragma once
#include <stdint.h>

#include <algorithm>

#include "runtime.h"

namespace r2 {

// d_rgb: W*H*3 linear floats on the device.  d_out (W*H*3 floats) and d_bytes
// (W*H*3 bytes) are optional outputs; d_scratch holds W + 1 floats.
void tonemap_device(const float* d_rgb, uint32_t W, uint32_t H, float gamma, float* d_out, uint8_t* d_bytes,
                    float* d_scratch, cudaStream_t s);

}  // namespace r2
