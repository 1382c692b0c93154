// Exception-to-status conversion for the C ABI.
#pragma once
#include <new>

#include "runtime.h"

namespace r2 {
const char* last_error();

// Throws R2_ERR_NO_DEVICE when no CUDA device is visible.
inline void require_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    throw Error{R2_ERR_NO_DEVICE, "no CUDA device available"};
  }
}
}  // namespace r2

#define R2_API_BEGIN          \
  ::r2::set_last_error("");   \
  try {
#define R2_API_END                                      \
  }                                                     \
  catch (const ::r2::Error& e) {                        \
    ::r2::set_last_error(e.msg);                        \
    return e.code;                                      \
  }                                                     \
  catch (const std::bad_alloc&) {                       \
    ::r2::set_last_error("host allocation failed");     \
    return R2_ERR_OUT_OF_MEMORY;                        \
  }                                                     \
  catch (const std::exception& e) {                     \
    ::r2::set_last_error(e.what());                     \
    return R2_ERR_INVALID_ARGUMENT;                     \
  }                                                     \
  catch (...) {                                         \
    ::r2::set_last_error("unknown error");              \
    return R2_ERR_DEVICE;                               \
  }                                                     \
  return R2_OK;
