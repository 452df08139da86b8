// curve_ops.cu — element-wise BN254 G1 kernels and their C ABI.
//
// One thread per point, grid-stride, with the reference's single-point
// broadcast (zkgpu/curve_gpu.py:234-274, :442-462). The point formulas are
// __noinline__ device functions (curve.cuh), as in the reference, which keeps
// these utility kernels small; the MSM inlines its own XYZZ formulas.
#include "curve.cuh"
#include "field_host.h"

namespace zkb {

__global__ void __launch_bounds__(128) k_g1_add(const uint64_t* a, int64_t a_step,
                                                const uint64_t* b, int64_t b_step, uint64_t* out,
                                                int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    Jac p, q, r;
    jac_load(p, a + 12 * i * a_step);
    jac_load(q, b + 12 * i * b_step);
    jac_add(r, p, q);
    jac_store(out + 12 * i, r);
  }
}

__global__ void __launch_bounds__(128) k_g1_add_affine(const uint64_t* a, int64_t a_step,
                                                       const uint64_t* b, int64_t b_step,
                                                       uint64_t* out, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    Jac p, r;
    Aff q;
    jac_load(p, a + 12 * i * a_step);
    aff_load(q, b + 8 * i * b_step);
    jac_add_affine(r, p, q);
    jac_store(out + 12 * i, r);
  }
}

__global__ void __launch_bounds__(128) k_g1_double(const uint64_t* a, uint64_t* out, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    Jac p, r;
    jac_load(p, a + 12 * i);
    jac_double(r, p);
    jac_store(out + 12 * i, r);
  }
}

// x = X / Z^2, y = Y / Z^3 with one inversion per point (zkgpu/curve.py:221-233),
// written as plain (non-Montgomery) canonical values; the identity gives (0, 0).
__global__ void __launch_bounds__(128) k_g1_to_affine(const uint64_t* jac, uint64_t* out,
                                                      int64_t n) {
  G1F f;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    Jac p;
    jac_load(p, jac + 12 * i);
    uint32_t x[8], y[8];
    if (fe_is_zero(p.z)) {
      fe_zero(x);
      fe_zero(y);
    } else {
      uint32_t zi[8], zi2[8];
      fe_inv(zi, p.z, f);
      fe_sqr(zi2, zi, f);
      fe_mul(x, p.x, zi2, f);
      fe_mul(zi2, zi2, zi, f);
      fe_mul(y, p.y, zi2, f);
      fe_from_mont(x, x, f);
      fe_from_mont(y, y, f);
    }
    fe_store(out + 8 * i, x);
    fe_store(out + 8 * i + 4, y);
  }
}

__global__ void __launch_bounds__(256) k_g1_check_affine(const uint64_t* pts, int64_t n,
                                                         unsigned long long* first_bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    Aff q;
    aff_load_nc(q, pts + 8 * i);
    if (!aff_on_curve(q)) atomicMin(first_bad, (unsigned long long)i);
  }
}

__global__ void k_set_u64(unsigned long long* p, unsigned long long v) { *p = v; }

// k G for the generator G = (1, 2): left-to-right double-and-add over the
// plain scalar's bits in XYZZ (the reference's Point.__mul__,
// zkgpu/curve.py:153-159 / :306-324, computes the same point), then affine
// Montgomery rows with one inversion. k must not be 0 mod r.
__global__ void __launch_bounds__(128) k_g1_mul_generator(const uint64_t* k, uint64_t* out,
                                                          int64_t n) {
  G1F f;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t s[8];
    fe_load(s, k + 4 * i);
    Aff g;
    uint32_t t[8] = {1, 0, 0, 0, 0, 0, 0, 0};
    fe_to_mont(g.x, t, f);
    t[0] = 2;
    fe_to_mont(g.y, t, f);
    Xyzz acc;
    xyzz_set_identity(acc);
    for (int bit = 255; bit >= 0; --bit) {
      xyzz_dbl(acc, acc);
      if ((s[bit >> 5] >> (bit & 31)) & 1u) xyzz_add_affine(acc, g);
    }
    Aff r;
    if (xyzz_is_identity(acc)) {
      fe_zero(r.x);
      fe_zero(r.y);
    } else {
      uint32_t prod[8], inv[8];
      fe_mul(prod, acc.zz, acc.zzz, f);
      fe_inv(inv, prod, f);
      fe_mul(t, inv, acc.zzz, f);
      fe_mul(r.x, acc.x, t, f);
      fe_mul(t, inv, acc.zz, f);
      fe_mul(r.y, acc.y, t, f);
    }
    fe_store(out + 8 * i, r.x);
    fe_store(out + 8 * i + 4, r.y);
  }
}

static int check_steps(int64_t n, int64_t a_step, int64_t b_step) {
  if (n < 0) return fail(ZKB_EINVAL, "negative point count %lld", (long long)n);
  if ((a_step != 0 && a_step != 1) || (b_step != 0 && b_step != 1)) {
    return fail(ZKB_EINVAL, "steps must be 0 (broadcast) or 1");
  }
  return ZKB_OK;
}

}  // namespace zkb

using namespace zkb;

extern "C" {

int zkb_g1_add(const uint64_t* a, int64_t a_step, const uint64_t* b, int64_t b_step,
               uint64_t* out, int64_t n, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_steps(n, a_step, b_step));
  if (n == 0) return ZKB_OK;
  if (!a || !b || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(a, 16, "a"));
  ZKB_TRY(check_align(b, 16, "b"));
  ZKB_TRY(check_align(out, 16, "out"));
  k_g1_add<<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(a, a_step, b, b_step, out, n);
  return check_launch("g1_add launch");
}

int zkb_g1_add_affine(const uint64_t* a, int64_t a_step, const uint64_t* b, int64_t b_step,
                      uint64_t* out, int64_t n, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_steps(n, a_step, b_step));
  if (n == 0) return ZKB_OK;
  if (!a || !b || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(a, 16, "a"));
  ZKB_TRY(check_align(b, 16, "b"));
  ZKB_TRY(check_align(out, 16, "out"));
  k_g1_add_affine<<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(a, a_step, b, b_step, out, n);
  return check_launch("g1_add_affine launch");
}

int zkb_g1_double(const uint64_t* a, uint64_t* out, int64_t n, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_steps(n, 1, 1));
  if (n == 0) return ZKB_OK;
  if (!a || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(a, 16, "a"));
  ZKB_TRY(check_align(out, 16, "out"));
  k_g1_double<<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(a, out, n);
  return check_launch("g1_double launch");
}

int zkb_g1_to_affine(const uint64_t* jac, uint64_t* out, int64_t n, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_steps(n, 1, 1));
  if (n == 0) return ZKB_OK;
  if (!jac || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(jac, 16, "jac"));
  ZKB_TRY(check_align(out, 16, "out"));
  k_g1_to_affine<<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(jac, out, n);
  return check_launch("g1_to_affine launch");
}

int zkb_g1_mul_generator(const uint64_t* k, uint64_t* out, int64_t n, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_steps(n, 1, 1));
  if (n == 0) return ZKB_OK;
  if (!k || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(k, 16, "k"));
  ZKB_TRY(check_align(out, 16, "out"));
  k_g1_mul_generator<<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(k, out, n);
  return check_launch("g1_mul_generator launch");
}

int zkb_g1_check_affine(const uint64_t* points, int64_t n, int64_t* first_bad, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_steps(n, 1, 1));
  if (!first_bad) return fail(ZKB_EINVAL, "null result pointer");
  ZKB_TRY(check_align(first_bad, 8, "first_bad"));
  ZKB_TRY(check_align(points, 16, "points"));
  cudaStream_t s = as_stream(stream);
  unsigned long long* fb = reinterpret_cast<unsigned long long*>(first_bad);
  // all ones reads back as -1 when no point fails
  k_set_u64<<<1, 1, 0, s>>>(fb, ~0ull);
  ZKB_TRY(check_launch("check_affine init"));
  if (n == 0) return ZKB_OK;
  if (!points) return fail(ZKB_EINVAL, "null buffer");
  k_g1_check_affine<<<grid_for(n, 256), 256, 0, s>>>(points, n, fb);
  return check_launch("g1_check_affine launch");
}

}  // extern "C"
