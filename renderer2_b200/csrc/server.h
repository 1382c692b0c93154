// Request loop for render and filter jobs on one GPU (continuous batching).
//
// Jobs arrive on any host thread (submit) and wait in a FIFO queue.  A
// scheduler thread admits the queue head as soon as a slot is free and the
// job's device memory fits in what the HBM budget leaves; each slot owns a
// CUDA stream, a render context (wave buffers grown on demand), the filter's
// work list, a device output buffer and a pinned staging buffer, so admitted
// jobs overlap on the device.  Scenes stay resident: jobs reference committed
// render scenes and filter scenes that the caller keeps alive and unmodified
// while its jobs run.  A render is one captured wave replayed once per sample;
// a filter job is one LOD of a filter scene.  Results are written to the
// caller's host buffer before the job reports completion.
//
// The reference renders one frame at a time (raytracer/pipeline.cu:24-90);
// this loop has no counterpart there.
#pragma once
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "filter_host.h"
#include "render_host.h"

namespace r2 {

struct ServerJob {
  uint64_t id = 0;
  int kind = 0;  // 0 render, 1 filter
  // render
  RenderScene* scene = nullptr;
  r2_camera cam;
  r2_render_params rp;
  float* rgbOut = nullptr;
  // filter
  FilterScene* fscene = nullptr;
  r2_filter_grid grid;
  r2_filter_params fp;
  uint32_t lod = 0;
  r2_voxel* voxOut = nullptr;
  // accounting
  size_t bytes = 0;        // device memory the job holds while admitted
  size_t outBytes = 0;
  double tSubmit = 0, tStart = 0, tEnd = 0;  // seconds on the server's clock
  bool done = false;
  r2_status status = R2_OK;
  std::string error;
};

class Server {
 public:
  Server(uint32_t slots, uint64_t hbmBudget);
  // Device bytes a render job is admitted with (its slot's wave buffers and frame).
  static size_t render_bytes(const RenderScene& scene, const r2_camera& cam, const r2_render_params& rp);
  ~Server();  // finishes the admitted and queued jobs, then stops
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  uint64_t submit(std::unique_ptr<ServerJob> job);
  // Waits up to timeout seconds (< 0: forever); false on timeout.  The job's
  // record stays until it is waited for successfully.
  bool wait(uint64_t id, double timeout, ServerJob* out);
  // [0] jobs done, [1] jobs queued, [2] jobs running, [3] device bytes admitted,
  // [4] seconds since start
  void stats(double* out);
  double now() const;

 private:
  struct Slot;
  void loop();
  bool start(Slot& s, ServerJob* j);
  void complete(Slot& s);
  uint32_t nslots_;
  uint64_t budget_;
  std::vector<std::unique_ptr<Slot>> slots_;
  std::mutex mu_;
  std::condition_variable cv_;      // scheduler wake-up
  std::condition_variable doneCv_;  // job completion
  std::deque<ServerJob*> queue_;
  std::map<uint64_t, std::unique_ptr<ServerJob>> jobs_;
  uint64_t nextId_ = 1;
  uint64_t admitted_ = 0;
  uint64_t doneCount_ = 0;
  bool stop_ = false;
  int device_ = 0;
  double t0_ = 0;
  std::thread thread_;
};

}  // namespace r2
