// per_device.h — one-time set-up of kernel attributes and occupancy figures, per device.
#pragma once

#include <cuda_runtime.h>

#include <mutex>

namespace shg {

// Kernel attributes (cudaFuncSetAttribute) and occupancy figures belong to one device. A
// process may drive several devices in turn, so PerDevice<V> runs a launcher's set-up once
// for every device ordinal the process uses, with that device current, and keeps the result
// (an error code and a value of type V) per device.
template <typename V>
class PerDevice {
  public:
    static constexpr int kMaxDevices = 64;

    // setup: cudaError_t(int device, V& value).  Returns the set-up's error code for the
    // current device; *out receives its value.
    template <class F>
    cudaError_t get(F&& setup, V* out = nullptr) {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
        std::lock_guard<std::mutex> lock(mu_);
        if (!done_[dev]) {
            err_[dev] = setup(dev, val_[dev]);
            done_[dev] = true;
        }
        if (out) *out = val_[dev];
        return err_[dev];
    }

  private:
    std::mutex mu_;
    bool done_[kMaxDevices] = {};
    cudaError_t err_[kMaxDevices] = {};
    V val_[kMaxDevices] = {};
};

}  // namespace shg
