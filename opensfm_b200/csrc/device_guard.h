// Restores the calling thread's current CUDA device when an entry point
// returns.  The library's objects live on the device that was current when
// they were created and make it current while they work; a host
// application that runs on another device keeps its own current device
// across every dn_* call (dn_set_device excepted: its job is to change it).
#pragma once

#include <cuda_runtime.h>

namespace dn {

class DeviceRestore {
 public:
  DeviceRestore() { ok_ = cudaGetDevice(&device_) == cudaSuccess; }
  ~DeviceRestore() {
    int now = -1;
    if (ok_ && cudaGetDevice(&now) == cudaSuccess && now != device_) cudaSetDevice(device_);
  }
  DeviceRestore(const DeviceRestore&) = delete;
  DeviceRestore& operator=(const DeviceRestore&) = delete;

 private:
  int device_ = 0;
  bool ok_ = false;
};

}  // namespace dn
