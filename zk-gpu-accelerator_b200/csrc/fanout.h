// fanout.h — run independent pieces of one call concurrently on side streams.
//
// Fanout f; f.fork(s, k) makes k side streams of the current device wait for
// all work queued on s so far; work queued on f.side(i) then runs beside
// each other; f.join(s) makes s wait for all of it. The side streams are
// created once per device (non-blocking) and shared by every call; each
// fork starts where the previous one ended, so that concurrent calls from
// different caller streams spread over all of them. Every call
// holds a lock from construction to destruction so that the fork and join
// events of two host threads never mix. Inside a stream capture the side
// streams join the capture through the events and leave it at join().
#pragma once

#include <cuda_runtime.h>

#include <mutex>

namespace zkb {

class Fanout {
 public:
  static constexpr int kMaxSides = 8;
  Fanout();
  ~Fanout();
  Fanout(const Fanout&) = delete;
  Fanout& operator=(const Fanout&) = delete;

  int fork(cudaStream_t s, int k);  // k <= kMaxSides
  cudaStream_t side(int i) const;
  int join(cudaStream_t s);

 private:
  std::unique_lock<std::mutex> lock_;
  int dev_ = 0;
  int k_ = 0;
  int base_ = 0;  // this fork's first side stream
};

}  // namespace zkb
