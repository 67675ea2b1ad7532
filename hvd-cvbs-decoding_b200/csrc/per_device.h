// per_device.h -- one-time setup per CUDA device.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <set>

namespace hvdg {

// Calls fn() the first time it is reached on the calling thread's current
// CUDA device; thread-safe. Kernel attributes (cudaFuncSetAttribute) and
// __constant__ tables belong to one device, so a process that decodes on two
// GPUs (one context each) needs them set on both.
struct PerDeviceOnce {
  std::mutex mu;
  std::set<int> done;
  template <typename F>
  void operator()(F&& fn) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (done.insert(dev).second) fn();
  }
};

}  // namespace hvdg
