// profile.h — optional per-stage timing with CUDA events on the launching stream.
//
// Off by default (no events, no overhead). zkb_profile_enable(1) clears the
// record and starts recording: every ProfSpan then puts a start and an end
// event on its stream around the launches it covers, and
// zkb_profile_report() waits for those events and sums the elapsed time of
// each stage name. Used by the benchmark to time the dominant kernel inside a
// step without a profiler attached.
#pragma once
#include <cuda_runtime.h>

namespace zkb {

bool prof_enabled();
int prof_begin(const char* name, cudaStream_t s);  // returns a span id, or -1 when off
void prof_end(int id, cudaStream_t s);

struct ProfSpan {
  int id;
  cudaStream_t s;
  ProfSpan(const char* name, cudaStream_t stream) : id(prof_begin(name, stream)), s(stream) {}
  ~ProfSpan() { prof_end(id, s); }
};

}  // namespace zkb
