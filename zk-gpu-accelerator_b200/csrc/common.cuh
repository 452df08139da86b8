// common.cuh — status codes, the thread-local error message, launch helpers.
//
// Every C-ABI entry point returns an int status and leaves a message for
// zkb_last_error(). The Python layer maps the codes onto the reference's
// exception types (ValueError, TypeError, RuntimeError;
// zkgpu/field256_gpu.py:250-266, zkgpu/msm_gpu.py:426-427).
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/zkb200.h"

namespace zkb {

void set_error(const char* fmt, ...);

inline int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  set_error("%s", buf);
  return code;
}

// Turns a CUDA error from the last launch (or call) into ZKB_ECUDA.
inline int check_cuda(cudaError_t err, const char* what) {
  if (err == cudaSuccess) return ZKB_OK;
  return fail(ZKB_ECUDA, "%s: %s", what, cudaGetErrorString(err));
}

// Counts this library's own kernel launches (one call per launch).
void count_launch();

// Tuning knobs read when a call plans its work (zkb_tune_set / zkb_tune_get).
int tune_get(const char* key);

// Per-size tuning tables (zkb_tune_set_sized): the entry for log2 size log_n,
// or 0 when the table has none.
constexpr int kMaxSizedLog = 32;
int tune_get_sized(const char* key, int log_n);

inline int check_launch(const char* what) {
  count_launch();
  return check_cuda(cudaGetLastError(), what);
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Row buffers are read and written as 16-byte vectors: a buffer that is not
// aligned is refused instead of faulting on the device. Null passes (callers
// check for null separately where a buffer is required).
inline int check_align(const void* p, unsigned align, const char* name) {
  if (p && (reinterpret_cast<uintptr_t>(p) & (align - 1)) != 0) {
    return fail(ZKB_EINVAL, "%s must be %u-byte aligned", name, align);
  }
  return ZKB_OK;
}

// Grid sizes: grid-stride loops over n items, at most `cap` blocks. The cap
// is a multiple of the B200's 148 SMs.
inline unsigned grid_for(int64_t n, int threads, int64_t cap = 148 * 64) {
  int64_t blocks = (n + threads - 1) / threads;
  if (blocks < 1) blocks = 1;
  if (blocks > cap) blocks = cap;
  return static_cast<unsigned>(blocks);
}

}  // namespace zkb

#define ZKB_TRY(expr)              \
  do {                             \
    int zkb_status_ = (expr);      \
    if (zkb_status_ != ZKB_OK) return zkb_status_; \
  } while (0)
