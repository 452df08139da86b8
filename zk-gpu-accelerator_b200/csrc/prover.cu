// prover.cu — the Groth16 quotient's pointwise step on the coset, fused into
// one kernel, and its C ABI.
//
// A Groth16 prover (demo/prover_simulation.py:1-25, :137-150) evaluates A, B
// and C on the coset g H and forms h(g w^i) = (A B - C)(g w^i) / Z_H(g) with
// the constant Z_H(g) = g^n - 1. The reference does it with three separate
// element-wise launches (Fr.mul, Fr.sub, Fr.mul by a one-row z_inv,
// prover_simulation.py:148); here one pass reads the three rows and writes
// one: 128 bytes per element, HBM-bound.
#include "field_host.h"

namespace zkb {

__global__ void __launch_bounds__(256) k_quotient_pointwise(const uint64_t* a, const uint64_t* b,
                                                            const uint64_t* c,
                                                            const uint64_t* z_plain, uint64_t* out,
                                                            int64_t n) {
  FrP f;
  uint32_t z[8], t[8];
  fe_load(t, z_plain);
  fe_reduce_full(t, f, 5);
  fe_to_mont(z, t, f);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t x[8], y[8], w[8];
    fe_load_nc(x, a + 4 * i);
    fe_load_nc(y, b + 4 * i);
    fe_load_nc(w, c + 4 * i);
    fe_mul(x, x, y, f);
    fe_sub(x, x, w, f);
    fe_mul(x, x, z, f);
    fe_store(out + 4 * i, x);
  }
}

}  // namespace zkb

using namespace zkb;

extern "C" {

int zkb_quotient_pointwise(const uint64_t* a, const uint64_t* b, const uint64_t* c,
                           const uint64_t* z, uint64_t* out, int64_t n, void* stream) {
  set_error("%s", "");
  if (n < 0) return fail(ZKB_EINVAL, "negative row count");
  if (n == 0) return ZKB_OK;
  if (!a || !b || !c || !z || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(a, 16, "a"));
  ZKB_TRY(check_align(b, 16, "b"));
  ZKB_TRY(check_align(c, 16, "c"));
  ZKB_TRY(check_align(z, 16, "z"));
  ZKB_TRY(check_align(out, 16, "out"));
  cudaStream_t s = as_stream(stream);
  k_quotient_pointwise<<<grid_for(n, 256), 256, 0, s>>>(a, b, c, z, out, n);
  return check_launch("quotient pointwise");
}

}  // extern "C"
