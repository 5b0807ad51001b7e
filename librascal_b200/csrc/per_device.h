// Per-device state of the library: one slot per CUDA device ordinal.
//
// Device-side objects that the host sets up once (the __constant__ tables of
// the spherical harmonics, the tcgen05 GEMM's status word, the addresses of
// static device arrays) exist separately on every device a process uses. A
// process-wide "done" flag or pointer would leave a second device with
// zeroed constants or make it write into the first device's memory, so each
// of them is kept in a PerDevice table indexed by the device that is current
// when the state is needed.
//
// Plain C++ (no CUDA headers): the bookkeeping is unit-tested on the host.
#pragma once

#include <mutex>
#include <stdexcept>
#include <string>

namespace rgpu {

constexpr int kMaxDevices = 64;

template <class T>
class PerDevice {
 public:
  // Slot of device `dev`; throws std::out_of_range for an ordinal outside
  // [0, kMaxDevices).
  T & at(int dev) {
    if (dev < 0 || dev >= kMaxDevices)
      throw std::out_of_range("device ordinal " + std::to_string(dev) + " outside [0, " +
                              std::to_string(kMaxDevices) + ")");
    return slot_[dev];
  }
  // Runs init(slot) the first time device `dev` asks, under a lock, and
  // returns the slot. A failing init leaves the slot uninitialised, so the
  // next call retries it.
  template <class F>
  T & once(int dev, F && init) {
    T & s = at(dev);
    std::lock_guard<std::mutex> lock(mutex_);
    if (!ready_[dev]) {
      init(s);
      ready_[dev] = true;
    }
    return s;
  }
  bool ready(int dev) { return at(dev), ready_[dev]; }

 private:
  T slot_[kMaxDevices]{};
  bool ready_[kMaxDevices]{};
  std::mutex mutex_;
};

}  // namespace rgpu
