// field_ops.cu — element-wise Montgomery arithmetic kernels and their C ABI.
//
// One thread per row in a grid-stride loop; each row is read as two 16-byte
// vectors, so a warp reads 1 KiB of consecutive rows (full sectors). These
// kernels are HBM-bound: 96 bytes per row for mul/add/sub (two reads, one
// write). A step of 0 broadcasts a single-row operand
// (zkgpu/field256_gpu.py:171-191, :260-266).
#include "field_host.h"

namespace zkb {

enum : int { OP_MUL = 0, OP_ADD = 1, OP_SUB = 2 };

template <class F, int OP>
__global__ void __launch_bounds__(256) k_field_binary(F f, const uint64_t* a, int64_t a_step,
                                                      const uint64_t* b, int64_t b_step,
                                                      uint64_t* out, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t x[8], y[8], r[8];
    fe_load(x, a + 4 * i * a_step);
    fe_load(y, b + 4 * i * b_step);
    if (OP == OP_MUL && a == b && a_step == b_step) {
      fe_sqr(r, x, f);  // the same rows on both sides: the squaring's 36-product form
    } else if (OP == OP_MUL) {
      fe_mul(r, x, y, f);
    } else if (OP == OP_ADD) {
      fe_add(r, x, y, f);
    } else {
      fe_sub(r, x, y, f);
    }
    fe_store(out + 4 * i, r);
  }
}

// reduce_subs: how many conditional subtractions bring any 256-bit value
// below p (0 when the caller guarantees canonical input).
template <class F>
__global__ void __launch_bounds__(256) k_to_mont(F f, const uint64_t* in, uint64_t* out, int64_t n,
                                                 int reduce_subs) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t x[8], r[8];
    fe_load(x, in + 4 * i);
    fe_reduce_full(x, f, reduce_subs);
    fe_to_mont(r, x, f);
    fe_store(out + 4 * i, r);
  }
}

template <class F>
__global__ void __launch_bounds__(256) k_from_mont(F f, const uint64_t* in, uint64_t* out,
                                                   int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t x[8], r[8];
    fe_load(x, in + 4 * i);
    fe_from_mont(r, x, f);
    fe_store(out + 4 * i, r);
  }
}

template <int OP>
static int field_binary(const zkb_field* f, const uint64_t* a, int64_t a_step, const uint64_t* b,
                        int64_t b_step, uint64_t* out, int64_t n, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_field(f));
  if (n < 0) return fail(ZKB_EINVAL, "negative row count %lld", (long long)n);
  if ((a_step != 0 && a_step != 1) || (b_step != 0 && b_step != 1)) {
    return fail(ZKB_EINVAL, "steps must be 0 (broadcast) or 1");
  }
  if (n == 0) return ZKB_OK;
  if (!a || !b || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(a, 16, "a"));
  ZKB_TRY(check_align(b, 16, "b"));
  ZKB_TRY(check_align(out, 16, "out"));
  const int threads = 256;
  const unsigned grid = grid_for(n, threads);
  cudaStream_t s = as_stream(stream);
  return with_field(f, [&](auto fp) {
    k_field_binary<decltype(fp), OP><<<grid, threads, 0, s>>>(fp, a, a_step, b, b_step, out, n);
    return check_launch("field kernel launch");
  });
}

}  // namespace zkb

using namespace zkb;

extern "C" {

int zkb_field_mul(const zkb_field* f, const uint64_t* a, int64_t a_step, const uint64_t* b,
                  int64_t b_step, uint64_t* out, int64_t n, void* stream) {
  return field_binary<OP_MUL>(f, a, a_step, b, b_step, out, n, stream);
}

int zkb_field_add(const zkb_field* f, const uint64_t* a, int64_t a_step, const uint64_t* b,
                  int64_t b_step, uint64_t* out, int64_t n, void* stream) {
  return field_binary<OP_ADD>(f, a, a_step, b, b_step, out, n, stream);
}

int zkb_field_sub(const zkb_field* f, const uint64_t* a, int64_t a_step, const uint64_t* b,
                  int64_t b_step, uint64_t* out, int64_t n, void* stream) {
  return field_binary<OP_SUB>(f, a, a_step, b, b_step, out, n, stream);
}

int zkb_field_to_mont(const zkb_field* f, const uint64_t* in, uint64_t* out, int64_t n,
                      void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_field(f));
  if (n < 0) return fail(ZKB_EINVAL, "negative row count");
  if (n == 0) return ZKB_OK;
  if (!in || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(in, 16, "in"));
  ZKB_TRY(check_align(out, 16, "out"));
  // BN254's moduli exceed 2^253, so five subtractions reduce any 256-bit value.
  const int subs = f->kind == ZKB_FIELD_GENERIC ? 0 : 5;
  const unsigned grid = grid_for(n, 256);
  cudaStream_t s = as_stream(stream);
  return with_field(f, [&](auto fp) {
    k_to_mont<<<grid, 256, 0, s>>>(fp, in, out, n, subs);
    return check_launch("to_mont launch");
  });
}

int zkb_field_from_mont(const zkb_field* f, const uint64_t* in, uint64_t* out, int64_t n,
                        void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_field(f));
  if (n < 0) return fail(ZKB_EINVAL, "negative row count");
  if (n == 0) return ZKB_OK;
  if (!in || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(in, 16, "in"));
  ZKB_TRY(check_align(out, 16, "out"));
  const unsigned grid = grid_for(n, 256);
  cudaStream_t s = as_stream(stream);
  return with_field(f, [&](auto fp) {
    k_from_mont<<<grid, 256, 0, s>>>(fp, in, out, n);
    return check_launch("from_mont launch");
  });
}

}  // extern "C"
