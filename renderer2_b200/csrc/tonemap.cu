// Output stage of a frame: Raytracer::renderFrame's global tonemapping,
// gamma correction and byte conversion (raytracer/raytracer.cu:33-127, called
// from renderFrame 161-210).
//
// The log-average keeps the reference's summation structure: one thread per
// column accumulates log(r + g + b + FLT_MIN) / (W H 3) over the rows in
// order, then one thread adds the column sums in order and takes
// exp(sum) - W H FLT_MIN.  A frame is then mapped per channel to
// c / (c + L), raised to 1/gamma and rounded to bytes.  The two reduction
// kernels are O(H) + O(W) serial steps, a few microseconds at 1080p.
#include <float.h>

#include "tonemap.h"

namespace r2 {
namespace {

__global__ void k_tm_columns(const float* __restrict__ rgb, int W, int H, float* __restrict__ colSum) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= W) return;
  const float divisor = (float)(H * W * 3);
  float acc = 0.0f;
  for (int y = 0; y < H; ++y) {
    const float* p = rgb + 3 * ((size_t)y * W + x);
    acc += logf(p[0] + p[1] + p[2] + FLT_MIN) / divisor;
  }
  colSum[x] = acc;
}

__global__ void k_tm_total(const float* __restrict__ colSum, int W, int H, float* __restrict__ factor) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  float r = 0.0f;
  for (int i = 0; i < W; ++i) r += colSum[i];
  *factor = expf(r) - (float)(W * H) * FLT_MIN;
}

__global__ void k_tm_apply(const float* __restrict__ in, size_t n, const float* __restrict__ factor, float invGamma,
                           float* __restrict__ out, uint8_t* __restrict__ bytes) {
  const float L = *factor;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float c = in[i];
    const float t = powf(c / (c + L), invGamma);
    if (out) out[i] = t;
    if (bytes) bytes[i] = (uint8_t)roundf(t * 255.0f);  // glm::round: halves away from zero
  }
}

}  // namespace

void tonemap_device(const float* d_rgb, uint32_t W, uint32_t H, float gamma, float* d_out, uint8_t* d_bytes,
                    float* d_scratch, cudaStream_t s) {
  R2_REQUIRE(W > 0 && H > 0, R2_ERR_INVALID_ARGUMENT, "empty frame");
  R2_REQUIRE((uint64_t)W * H * 3 < (1ull << 31), R2_ERR_UNSUPPORTED, "frame too large for the tonemapper");
  R2_REQUIRE(gamma > 0.0f, R2_ERR_INVALID_ARGUMENT, "gamma must be positive");
  k_tm_columns<<<(W + 127) / 128, 128, 0, s>>>(d_rgb, (int)W, (int)H, d_scratch);
  k_tm_total<<<1, 32, 0, s>>>(d_scratch, (int)W, (int)H, d_scratch + W);
  const size_t n = (size_t)W * H * 3;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 16);
  k_tm_apply<<<blocks, 256, 0, s>>>(d_rgb, n, d_scratch + W, 1.0f / gamma, d_out, d_bytes);
  R2_CUDA(cudaGetLastError());
}

}  // namespace r2
