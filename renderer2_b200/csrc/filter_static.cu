// Filter entry point for callers that may not allocate device memory.
//
// Some host programs cannot call cudaMalloc at the moment they run the filter:
// a renderer's frame loop that runs under a fixed memory budget with no
// allocation allowed after start-up, an embedding application that owns every
// device allocation through its own pool, or a latency-bound caller that
// cannot afford the device-wide synchronisation an allocation may imply.  For
// them, r2_filter_scene_run_static filters one LOD with the voxel work list
// and queue counters placed in a fixed scratch array that lives in this
// library's device image instead of a buffer allocated per call.  The scene
// (BVH, shading data) is created beforehand, when allocation is allowed.
//
// The scratch holds at most kStaticMaxVoxels voxel ids (4 MiB) plus two
// counters; every GPU that loads the library keeps it until the process ends.
// Larger grids are rejected with R2_ERR_UNSUPPORTED.  All calls share the one
// array: calls that overlap on the GPU (different streams, or different host
// threads without ordering) race on it and must not be issued concurrently.
// A NULL stream means the device's legacy default stream, so calls given NULL
// run one after another whatever scene they filter.  The array keeps the
// previous call's contents: the counters are cleared by every call before use;
// the work list needs no clearing (each call writes the entries it reads).
// The first call on a device resolves the array's device address with
// cudaGetSymbolAddress (once per device, with that device current); make that
// first call before any stream capture.  The device current at the call, and
// the device of a given stream, must be the scene's device.
#include <mutex>

#include "capi_util.h"
#include "filter.cuh"
#include "filter_host.h"

namespace r2 {
constexpr size_t kStaticMaxVoxels = (size_t)1 << 20;
constexpr int kStaticMaxDevices = 64;
}  // namespace r2

// Work list followed by the two queue counters.
static __device__ __align__(256) uint32_t g_filterScratch[r2::kStaticMaxVoxels + 64];

namespace r2 {

// Device address of g_filterScratch on device `dev`, resolved once per device
// with that device current (the host-side symbol g_filterScratch is not a
// device address).  The lookup table is shared by all host threads.
static uint32_t* scratch_address(int dev) {
  static std::mutex mu;
  static uint32_t* addr[kStaticMaxDevices] = {nullptr};
  R2_REQUIRE(dev >= 0 && dev < kStaticMaxDevices, R2_ERR_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    R2_CUDA(cudaGetSymbolAddress(&p, g_filterScratch));
    addr[dev] = (uint32_t*)p;
  }
  return addr[dev];
}

}  // namespace r2

struct r2_filter_scene;  // defined in capi_filter.cu
r2::FilterScene* r2_filter_scene_impl(r2_filter_scene* scene);

extern "C" r2_status r2_filter_scene_run_static(r2_filter_scene* scene, const r2_filter_grid* grid,
                                                const r2_filter_params* params, r2_voxel* d_out, float* d_wide,
                                                uint16_t* d_fp16, void* stream) {
  R2_API_BEGIN
  R2_REQUIRE(scene && grid && params && d_out, R2_ERR_INVALID_ARGUMENT, "null argument");
  const size_t nvox = (size_t)grid->num_voxels[0] * grid->num_voxels[1] * grid->num_voxels[2];
  R2_REQUIRE(nvox <= r2::kStaticMaxVoxels, R2_ERR_UNSUPPORTED,
             "grid of " + std::to_string(nvox) + " voxels exceeds the static scratch limit of " +
                 std::to_string(r2::kStaticMaxVoxels) + " voxels");
  r2::FilterScene* sc = r2_filter_scene_impl(scene);
  int dev = -1;
  R2_CUDA(cudaGetDevice(&dev));
  R2_REQUIRE(dev == sc->device(), R2_ERR_INVALID_ARGUMENT,
             "current device " + std::to_string(dev) + " is not the scene's device " +
                 std::to_string(sc->device()));
  cudaStream_t s = stream ? (cudaStream_t)stream : cudaStreamLegacy;
  if (stream) {
    int sdev = -1;
    R2_CUDA(cudaStreamGetDevice(s, &sdev));
    R2_REQUIRE(sdev == dev, R2_ERR_INVALID_ARGUMENT,
               "stream of device " + std::to_string(sdev) + " given for a scene on device " + std::to_string(dev));
  }
  uint32_t* work = r2::scratch_address(dev);
  uint32_t* counters = work + r2::kStaticMaxVoxels;
  sc->run(*grid, *params, 0, d_out, d_wide, d_fp16, s, nullptr, work, counters);
  R2_API_END
}
