// Makes a device current for the duration of one library call and gives the
// caller's thread its previous current device back on every return path, so
// that no entry point leaves the host thread on another device.
#pragma once

#include <cuda_runtime.h>

namespace ap {

class DeviceScope {
 public:
  explicit DeviceScope(int device) {
    if (cudaGetDevice(&prev_) != cudaSuccess) {
      cudaGetLastError();
      prev_ = -1;
    }
    if (prev_ != device) {
      err_ = cudaSetDevice(device);
      switched_ = err_ == cudaSuccess;
    }
  }
  ~DeviceScope() {
    if (switched_ && prev_ >= 0) cudaSetDevice(prev_);
  }
  cudaError_t status() const { return err_; }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;

 private:
  int prev_ = -1;
  bool switched_ = false;
  cudaError_t err_ = cudaSuccess;
};

}  // namespace ap
