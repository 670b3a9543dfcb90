// Per-device one-time set-up, for CUDA state that belongs to one device.
//
// cudaFuncSetAttribute (for example the dynamic shared-memory limit of a
// kernel) applies to the device that is current when it is called.  A process
// that opens contexts on several devices (fdb_open takes a device ordinal)
// must therefore run such set-up once per device, not once per process, and
// two threads (the serving scheduler and a caller, say) may reach the same
// launch site together.  PerDeviceOnce keeps one "done" bit per device
// ordinal behind a mutex; the fast path is one atomic load.
//
// Ordinals at or above kTracked are not remembered: their set-up runs on every
// call, which is correct, only slower.
//
// The header has no CUDA dependency so that a host-only test can exercise the
// bookkeeping.
#pragma once
#include <atomic>
#include <cstdint>
#include <mutex>

namespace fdb {

class PerDeviceOnce {
 public:
  static constexpr int kTracked = 64;

  // Run f() unless it has already succeeded for `device`.  When f() throws,
  // the device is not marked done and the exception propagates, so a later
  // call retries.
  template <class F>
  void operator()(int device, F&& f) {
    if (done(device)) return;
    std::lock_guard<std::mutex> g(mu_);
    if (done(device)) return;
    f();
    if (device >= 0 && device < kTracked) bits_.fetch_or(1ull << device, std::memory_order_release);
  }

  bool done(int device) const {
    if (device < 0 || device >= kTracked) return false;
    return (bits_.load(std::memory_order_acquire) >> device) & 1ull;
  }

 private:
  std::atomic<uint64_t> bits_{0};
  std::mutex mu_;
};

}  // namespace fdb
