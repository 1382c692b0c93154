// Host runtime pieces shared by the filter and the path tracer: status codes
// (the C ABI returns them; no exception crosses it), an owning device buffer,
// and CUDA error plumbing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <utility>
#include <vector>

#include "../../include/r2.h"

namespace r2 {

// Error carried inside the C++ runtime; the C ABI converts it to r2_status and
// records the message for r2_last_error().
struct Error {
  r2_status code;
  std::string msg;
};

void set_last_error(const std::string& msg);

#define R2_CUDA(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      throw ::r2::Error{e_ == cudaErrorMemoryAllocation ? R2_ERR_OUT_OF_MEMORY            \
                                                         : R2_ERR_DEVICE,                \
                        std::string(#call) + ": " + cudaGetErrorString(e_)};             \
    }                                                                                    \
  } while (0)

#define R2_REQUIRE(cond, code, text)                       \
  do {                                                     \
    if (!(cond)) throw ::r2::Error{(code), std::string(text)}; \
  } while (0)

// Owning device allocation (cudaMalloc / cudaFree).
template <typename T>
class DBuf {
 public:
  DBuf() = default;
  explicit DBuf(size_t n) { alloc(n); }
  ~DBuf() { release(); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
    return *this;
  }
  void alloc(size_t n) {
    release();
    if (n == 0) return;
    R2_CUDA(cudaMalloc((void**)&p_, n * sizeof(T)));
    n_ = n;
  }
  // Grow-only reallocation (contents are not preserved).
  void reserve(size_t n) { if (n > n_) alloc(n); }
  // Grows to a power of two at least n, so that buffers reused for jobs of
  // varying size reallocate rarely (each cudaFree/cudaMalloc waits for the device).
  void reserve_grow(size_t n) {
    if (n <= n_) return;
    size_t c = 1;
    while (c < n) c <<= 1;
    alloc(c);
  }
  void release() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }
  void upload(const T* h, size_t n, cudaStream_t s) {
    reserve(n);
    if (n) R2_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void download(T* h, size_t n, cudaStream_t s) const {
    if (n) R2_CUDA(cudaMemcpyAsync(h, p_, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  size_t bytes() const { return n_ * sizeof(T); }

 private:
  T* p_ = nullptr;
  size_t n_ = 0;
};

inline int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

}  // namespace r2
