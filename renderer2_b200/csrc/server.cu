// Request loop for render and filter jobs (see server.h).
#include "server.h"

#include <string.h>

#include <chrono>

namespace r2 {

// Paths per wave of a render job: 0 keeps the scene's tuning.  A wave of a
// few million paths fills the GPU by itself (capping waves at 1M paths so that
// concurrent jobs would share the GPU made single jobs 1.7x slower), so slots
// mainly overlap one job's host work and copies with another's kernels.
constexpr uint32_t kServeWavePaths = 0;

// Bytes of a buffer grown to a power of two (DBuf::reserve_grow).
static size_t grow_bytes(size_t n) {
  size_t c = 1;
  while (c < n) c <<= 1;
  return c;
}

struct Server::Slot {
  RenderContext ctx;  // wave buffers + the slot's stream
  DBuf<float> frame;
  DBuf<r2_voxel> vox;
  DBuf<uint32_t> work, counters;
  void* pinned = nullptr;
  size_t pinnedBytes = 0;
  uint32_t* pinnedBound = nullptr;
  cudaEvent_t done = nullptr;
  ServerJob* job = nullptr;
  bool busy = false;

  Slot() {
    R2_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    R2_CUDA(cudaHostAlloc((void**)&pinnedBound, sizeof(uint32_t), cudaHostAllocDefault));
  }
  ~Slot() {
    if (ctx.stream) cudaStreamSynchronize(ctx.stream);
    if (pinned) cudaFreeHost(pinned);
    if (pinnedBound) cudaFreeHost(pinnedBound);
    if (done) cudaEventDestroy(done);
  }
  void* staging(size_t bytes) {
    if (bytes > pinnedBytes) {  // grown to a power of two: pinned allocation is slow and synchronous
      if (pinned) cudaFreeHost(pinned);
      pinned = nullptr;
      pinnedBytes = 0;
      size_t c = 1 << 16;
      while (c < bytes) c <<= 1;
      R2_CUDA(cudaHostAlloc(&pinned, c, cudaHostAllocDefault));
      pinnedBytes = c;
    }
    return pinned;
  }
};

Server::Server(uint32_t slots, uint64_t hbmBudget) : nslots_(slots), budget_(hbmBudget) {
  R2_REQUIRE(slots >= 1 && slots <= 64, R2_ERR_INVALID_ARGUMENT, "slots must be in [1, 64]");
  R2_REQUIRE(hbmBudget > 0, R2_ERR_INVALID_ARGUMENT, "empty HBM budget");
  R2_CUDA(cudaGetDevice(&device_));
  for (uint32_t i = 0; i < slots; ++i) slots_.emplace_back(new Slot());
  t0_ = 0.0;
  t0_ = now();
  thread_ = std::thread([this] { loop(); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  if (thread_.joinable()) thread_.join();
}

double Server::now() const {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count() - t0_;
}

size_t Server::render_bytes(const RenderScene& scene, const r2_camera& cam, const r2_render_params& rp) {
  const uint32_t npix = cam.width * cam.height;
  return RenderContext::bytes_for(npix * scene.wave_spp(npix, rp.spp, kServeWavePaths), scene.has_media()) +
         grow_bytes((size_t)npix * 12);
}

uint64_t Server::submit(std::unique_ptr<ServerJob> job) {
  ServerJob* j = job.get();
  if (j->kind == 0) {
    R2_REQUIRE(j->scene && j->scene->committed(), R2_ERR_INVALID_ARGUMENT, "render job needs a committed scene");
    const uint32_t npix = j->cam.width * j->cam.height;
    R2_REQUIRE(npix > 0 && j->rp.spp > 0 && j->rp.max_depth > 0 && j->rp.max_depth <= 60, R2_ERR_INVALID_ARGUMENT,
               "bad render job");
    j->bytes = render_bytes(*j->scene, j->cam, j->rp);
    j->outBytes = (size_t)npix * 12;
  } else {
    R2_REQUIRE(j->fscene, R2_ERR_INVALID_ARGUMENT, "filter job needs a filter scene");
    const size_t nvox = (size_t)j->grid.num_voxels[0] * j->grid.num_voxels[1] * j->grid.num_voxels[2];
    R2_REQUIRE(nvox > 0 && nvox < (1ull << 32), R2_ERR_INVALID_ARGUMENT, "bad filter grid");
    j->outBytes = nvox * sizeof(r2_voxel);
    j->bytes = grow_bytes(nvox * sizeof(r2_voxel)) + grow_bytes(nvox * 4) + 64;
  }
  R2_REQUIRE(j->bytes <= budget_, R2_ERR_ADMISSION_REJECTED, "job needs more device memory than the HBM budget");
  uint64_t id;
  {
    std::lock_guard<std::mutex> lk(mu_);
    R2_REQUIRE(!stop_, R2_ERR_INVALID_ARGUMENT, "server is stopping");
    id = nextId_++;
    j->id = id;
    j->tSubmit = now();
    queue_.push_back(j);
    jobs_[id] = std::move(job);
  }
  cv_.notify_all();
  return id;
}

bool Server::wait(uint64_t id, double timeout, ServerJob* out) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = jobs_.find(id);
  R2_REQUIRE(it != jobs_.end(), R2_ERR_INVALID_ARGUMENT, "unknown job id");
  ServerJob* j = it->second.get();
  auto ready = [j] { return j->done; };
  if (timeout < 0) {
    doneCv_.wait(lk, ready);
  } else if (!doneCv_.wait_for(lk, std::chrono::duration<double>(timeout), ready)) {
    return false;
  }
  if (out) *out = *j;
  jobs_.erase(it);
  return true;
}

void Server::stats(double* out) {
  std::lock_guard<std::mutex> lk(mu_);
  uint32_t running = 0;
  for (auto& s : slots_) running += s->busy ? 1u : 0u;
  out[0] = (double)doneCount_;
  out[1] = (double)queue_.size();
  out[2] = (double)running;
  out[3] = (double)admitted_;
  out[4] = now();
}

// Issues the job's device work on the slot's stream; false if it failed to start.
bool Server::start(Slot& s, ServerJob* j) {
  try {
    cudaStream_t st = s.ctx.stream;
    if (j->kind == 0) {
      const uint32_t npix = j->cam.width * j->cam.height;
      s.frame.reserve_grow((size_t)npix * 3);
      j->scene->render_graph(s.ctx, j->cam, j->rp, s.frame.get(), st, kServeWavePaths);
      R2_CUDA(cudaMemcpyAsync(s.staging(j->outBytes), s.frame.get(), j->outBytes, cudaMemcpyDeviceToHost, st));
      R2_CUDA(cudaMemcpyAsync(s.pinnedBound, s.ctx.bound.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    } else {
      const size_t nvox = (size_t)j->grid.num_voxels[0] * j->grid.num_voxels[1] * j->grid.num_voxels[2];
      s.vox.reserve_grow(nvox);
      s.work.reserve_grow(nvox);
      s.counters.reserve(2);
      j->fscene->run(j->grid, j->fp, j->lod, s.vox.get(), nullptr, nullptr, st, nullptr, s.work.get(),
                     s.counters.get());
      R2_CUDA(cudaMemcpyAsync(s.staging(j->outBytes), s.vox.get(), j->outBytes, cudaMemcpyDeviceToHost, st));
      *s.pinnedBound = 0;
    }
    R2_CUDA(cudaEventRecord(s.done, st));
    return true;
  } catch (const Error& e) {
    j->status = e.code;
    j->error = e.msg;
  } catch (const std::exception& e) {
    j->status = R2_ERR_DEVICE;
    j->error = e.what();
  }
  return false;
}

void Server::complete(Slot& s) {
  ServerJob* j = s.job;
  if (j->status == R2_OK) {
    memcpy(j->kind == 0 ? (void*)j->rgbOut : (void*)j->voxOut, s.pinned, j->outBytes);
    if (*s.pinnedBound != 0) {
      j->status = R2_ERR_DEVICE_TIMEOUT;
      j->error = std::to_string(*s.pinnedBound) + " paths or shadow rays ended by a loop bound";
    }
  }
  std::lock_guard<std::mutex> lk(mu_);
  j->tEnd = now();
  j->done = true;
  admitted_ -= j->bytes;
  ++doneCount_;
  s.job = nullptr;
  s.busy = false;
  doneCv_.notify_all();
}

void Server::loop() {
  cudaSetDevice(device_);
  for (;;) {
    std::vector<std::pair<Slot*, ServerJob*>> starts;
    {
      std::unique_lock<std::mutex> lk(mu_);
      // admit the queue head while a slot is free and its memory fits
      for (auto& s : slots_) {
        if (s->busy || queue_.empty()) continue;
        ServerJob* j = queue_.front();
        if (admitted_ > 0 && admitted_ + j->bytes > budget_) break;
        queue_.pop_front();
        admitted_ += j->bytes;
        j->tStart = now();
        s->busy = true;
        s->job = j;
        starts.emplace_back(s.get(), j);
      }
      bool anyBusy = false;
      for (auto& s : slots_) anyBusy = anyBusy || s->busy;
      if (stop_ && queue_.empty() && !anyBusy) return;
      if (starts.empty() && !anyBusy) {
        cv_.wait(lk, [this] { return stop_ || !queue_.empty(); });
        continue;
      }
    }
    for (auto& sj : starts)
      if (!start(*sj.first, sj.second)) complete(*sj.first);
    bool progressed = !starts.empty();
    for (auto& s : slots_) {
      if (!s->busy) continue;
      const cudaError_t q = cudaEventQuery(s->done);
      if (q == cudaSuccess) {
        complete(*s);
        progressed = true;
      } else if (q != cudaErrorNotReady) {
        s->job->status = R2_ERR_DEVICE;
        s->job->error = cudaGetErrorString(q);
        cudaGetLastError();
        complete(*s);
        progressed = true;
      }
    }
    if (!progressed) {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait_for(lk, std::chrono::microseconds(50));
    }
  }
}

}  // namespace r2
