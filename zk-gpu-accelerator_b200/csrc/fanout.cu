// fanout.cu — per-device side streams and events for Fanout.
#include "fanout.h"

#include "common.cuh"

namespace zkb {

namespace {

constexpr int kMaxDevices = 64;

struct DeviceSides {
  bool ready = false;
  int next = 0;  // first side stream of the next fork: calls rotate over them
  cudaStream_t streams[Fanout::kMaxSides] = {};
  cudaEvent_t fork_event = nullptr;
  cudaEvent_t join_events[Fanout::kMaxSides] = {};
};

std::mutex g_fanout_mutex;
DeviceSides g_sides[kMaxDevices];

int ensure_sides(int dev) {
  DeviceSides& d = g_sides[dev];
  if (d.ready) return ZKB_OK;
  for (int i = 0; i < Fanout::kMaxSides; ++i) {
    ZKB_TRY(check_cuda(cudaStreamCreateWithFlags(&d.streams[i], cudaStreamNonBlocking),
                       "side stream"));
    ZKB_TRY(check_cuda(cudaEventCreateWithFlags(&d.join_events[i], cudaEventDisableTiming),
                       "join event"));
  }
  ZKB_TRY(check_cuda(cudaEventCreateWithFlags(&d.fork_event, cudaEventDisableTiming),
                     "fork event"));
  d.ready = true;
  return ZKB_OK;
}

}  // namespace

Fanout::Fanout() : lock_(g_fanout_mutex) {}

Fanout::~Fanout() = default;

int Fanout::fork(cudaStream_t s, int k) {
  ZKB_TRY(check_cuda(cudaGetDevice(&dev_), "cudaGetDevice"));
  if (dev_ < 0 || dev_ >= kMaxDevices) return fail(ZKB_EINVAL, "device index %d out of range", dev_);
  if (k < 0 || k > kMaxSides) return fail(ZKB_EINVAL, "fan-out of %d streams", k);
  ZKB_TRY(ensure_sides(dev_));
  k_ = k;
  DeviceSides& d = g_sides[dev_];
  base_ = d.next;
  d.next = (d.next + k) % kMaxSides;
  ZKB_TRY(check_cuda(cudaEventRecord(d.fork_event, s), "fork record"));
  for (int i = 0; i < k; ++i) {
    ZKB_TRY(check_cuda(cudaStreamWaitEvent(side(i), d.fork_event, 0), "fork wait"));
  }
  return ZKB_OK;
}

cudaStream_t Fanout::side(int i) const {
  return g_sides[dev_].streams[(base_ + i % k_) % kMaxSides];
}

int Fanout::join(cudaStream_t s) {
  DeviceSides& d = g_sides[dev_];
  for (int i = 0; i < k_; ++i) {
    const int idx = (base_ + i) % kMaxSides;
    ZKB_TRY(check_cuda(cudaEventRecord(d.join_events[idx], d.streams[idx]), "join record"));
    ZKB_TRY(check_cuda(cudaStreamWaitEvent(s, d.join_events[idx], 0), "join wait"));
  }
  k_ = 0;
  return ZKB_OK;
}

}  // namespace zkb
