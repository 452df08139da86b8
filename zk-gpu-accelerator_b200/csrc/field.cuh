// field.cuh — 256-bit Montgomery arithmetic for sm_100a, 8 x 32-bit limbs.
//
// An element is the Montgomery form a*R mod p with R = 2^256, held as eight
// little-endian 32-bit limbs. In memory one element is 32 bytes, so its bytes
// are identical to the reference's (n, 4) uint64 rows (zkgpu/field256_gpu.py:12-20):
// a row written by this code reads back as the same four 64-bit limbs.
//
// Contract (zkgpu/field256_gpu.py:22-30): the modulus is odd and below 2^255,
// inputs are canonical (< p), and every function returns canonical output, so
// results are bit-identical to any other correct Montgomery implementation with
// R = 2^256 (the canonical representative of a*b*R^-1 mod p is unique).
//
// Multiplication is CIOS (Koc, Acar, Kaliski 1996) over 32-bit words. Each of
// the eight outer steps adds a*b[i], then m*p with m = t[0] * (-p^-1 mod 2^32),
// and drops the zero low word. Between steps t < 2p; during a step the running
// total is below 2^32 * 2p < 2^288, so nine words of state suffice and the top
// word never carries out. Each row is two carry chains written as inline PTX
// (mad.lo.cc / madc.lo.cc for the low halves of the partial products, then
// mad.hi.cc / madc.hi.cc for the high halves one word up), so the compiler
// never has to materialise a 64-bit product or a carry in a general register.
#pragma once
#include <cstdint>

namespace zkb {

// ---------------------------------------------------------------------------
// Field policies: p(i), one(i) (= R mod p), r2(i) (= R^2 mod p), ninv
// (= -p^-1 mod 2^32). Compile-time policies fold into immediates.
// ---------------------------------------------------------------------------

// BN254 scalar field r (zkgpu/field.py:17 FIELD_MODULUS).
struct FrP {
  __host__ __device__ __forceinline__ static constexpr uint32_t p(int i) {
    constexpr uint32_t v[8] = {0xf0000001u, 0x43e1f593u, 0x79b97091u, 0x2833e848u,
                               0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
    return v[i];
  }
  __host__ __device__ __forceinline__ static constexpr uint32_t one(int i) {
    constexpr uint32_t v[8] = {0x4ffffffbu, 0xac96341cu, 0x9f60cd29u, 0x36fc7695u,
                               0x7879462eu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u};
    return v[i];
  }
  __host__ __device__ __forceinline__ static constexpr uint32_t r2(int i) {
    constexpr uint32_t v[8] = {0xae216da7u, 0x1bb8e645u, 0xe35c59e3u, 0x53fe3ab1u,
                               0x53bb8085u, 0x8c49833du, 0x7f4e44a5u, 0x0216d0b1u};
    return v[i];
  }
  __host__ __device__ __forceinline__ static constexpr uint32_t ninv() { return 0xefffffffu; }
};

// BN254 base field p (zkgpu/curve.py:29 P): curve coordinates.
struct FqP {
  __host__ __device__ __forceinline__ static constexpr uint32_t p(int i) {
    constexpr uint32_t v[8] = {0xd87cfd47u, 0x3c208c16u, 0x6871ca8du, 0x97816a91u,
                               0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
    return v[i];
  }
  __host__ __device__ __forceinline__ static constexpr uint32_t one(int i) {
    constexpr uint32_t v[8] = {0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u,
                               0x7879462cu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u};
    return v[i];
  }
  __host__ __device__ __forceinline__ static constexpr uint32_t r2(int i) {
    constexpr uint32_t v[8] = {0x538afa89u, 0xf32cfc5bu, 0xd44501fbu, 0xb5e71911u,
                               0x0a417ff6u, 0x47ab1effu, 0xcab8351fu, 0x06d89f71u};
    return v[i];
  }
  __host__ __device__ __forceinline__ static constexpr uint32_t ninv() { return 0xe4866389u; }
};

// Any odd modulus in [3, 2^255), passed by value in kernel parameters
// (Field256(modulus) for moduli other than BN254's, zkgpu/field256_gpu.py:277-288).
struct FieldRT {
  uint32_t P[8];
  uint32_t ONE[8];
  uint32_t R2[8];
  uint32_t NINV;
  __host__ __device__ __forceinline__ uint32_t p(int i) const { return P[i]; }
  __host__ __device__ __forceinline__ uint32_t one(int i) const { return ONE[i]; }
  __host__ __device__ __forceinline__ uint32_t r2(int i) const { return R2[i]; }
  __host__ __device__ __forceinline__ uint32_t ninv() const { return NINV; }
};

// ---------------------------------------------------------------------------
// Loads and stores: one element is two 16-byte vectors.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void fe_load(uint32_t r[8], const void* src) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4 lo = s[0], hi = s[1];
  r[0] = lo.x; r[1] = lo.y; r[2] = lo.z; r[3] = lo.w;
  r[4] = hi.x; r[5] = hi.y; r[6] = hi.z; r[7] = hi.w;
}

// Read-only, streamed once: bypass L1 allocation.
__device__ __forceinline__ void fe_load_nc(uint32_t r[8], const void* src) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4 lo = __ldg(s), hi = __ldg(s + 1);
  r[0] = lo.x; r[1] = lo.y; r[2] = lo.z; r[3] = lo.w;
  r[4] = hi.x; r[5] = hi.y; r[6] = hi.z; r[7] = hi.w;
}

// Data written earlier in the same kernel by other CTAs: cached in L2 only,
// so that no stale L1 line of this SM is read.
__device__ __forceinline__ void fe_load_cg(uint32_t r[8], const void* src) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4 lo = __ldcg(s), hi = __ldcg(s + 1);
  r[0] = lo.x; r[1] = lo.y; r[2] = lo.z; r[3] = lo.w;
  r[4] = hi.x; r[5] = hi.y; r[6] = hi.z; r[7] = hi.w;
}

__device__ __forceinline__ void fe_store(void* dst, const uint32_t a[8]) {
  uint4* d = reinterpret_cast<uint4*>(dst);
  d[0] = make_uint4(a[0], a[1], a[2], a[3]);
  d[1] = make_uint4(a[4], a[5], a[6], a[7]);
}

__device__ __forceinline__ void fe_copy(uint32_t r[8], const uint32_t a[8]) {
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = a[j];
}

__device__ __forceinline__ void fe_zero(uint32_t r[8]) {
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = 0;
}

template <class F>
__device__ __forceinline__ void fe_one(uint32_t r[8], const F& f) {
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = f.one(j);
}

// Rows are canonical, so zero is all-zero limbs (zkgpu/curve_gpu.py:67-69).
__device__ __forceinline__ bool fe_is_zero(const uint32_t a[8]) {
  return (a[0] | a[1] | a[2] | a[3] | a[4] | a[5] | a[6] | a[7]) == 0;
}

__device__ __forceinline__ bool fe_eq(const uint32_t a[8], const uint32_t b[8]) {
  uint32_t d = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) d |= a[j] ^ b[j];
  return d == 0;
}

// ---------------------------------------------------------------------------
// t := t - p if t >= p, for t < 2p (branch-free; zkgpu/field256_gpu.py:76-94).
// ---------------------------------------------------------------------------
template <class F>
__device__ __forceinline__ void fe_reduce_once(uint32_t t[8], const F& f) {
  uint32_t d0, d1, d2, d3, d4, d5, d6, d7, bw;
  asm("sub.cc.u32 %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32 %8, 0, 0;"
      : "=r"(d0), "=r"(d1), "=r"(d2), "=r"(d3), "=r"(d4), "=r"(d5), "=r"(d6), "=r"(d7), "=r"(bw)
      : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
        "r"(f.p(0)), "r"(f.p(1)), "r"(f.p(2)), "r"(f.p(3)), "r"(f.p(4)), "r"(f.p(5)), "r"(f.p(6)),
        "r"(f.p(7)));
  // bw is all ones when t < p (the subtraction borrowed): keep t then.
  t[0] = bw ? t[0] : d0;
  t[1] = bw ? t[1] : d1;
  t[2] = bw ? t[2] : d2;
  t[3] = bw ? t[3] : d3;
  t[4] = bw ? t[4] : d4;
  t[5] = bw ? t[5] : d5;
  t[6] = bw ? t[6] : d6;
  t[7] = bw ? t[7] : d7;
}

// r = a + b mod p. a, b < p < 2^255, so a + b < 2^256 never carries out.
// r may alias a or b (every input limb is read before any output is written).
template <class F>
__device__ __forceinline__ void fe_add(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                       const F& f) {
  uint32_t s[8];
  asm("add.cc.u32 %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32 %7, %15, %23;"
      : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
        "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
  fe_reduce_once(s, f);
  fe_copy(r, s);
}

// r = a - b mod p: subtract, then add p back under the borrow mask
// (zkgpu/field256_gpu.py:148-169). r may alias a or b.
template <class F>
__device__ __forceinline__ void fe_sub(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                       const F& f) {
  uint32_t s[8], bw;
  asm("sub.cc.u32 %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32 %8, 0, 0;"
      : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7]),
        "=r"(bw)
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
        "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
  asm("add.cc.u32 %0, %0, %8;\n\t"
      "addc.cc.u32 %1, %1, %9;\n\t"
      "addc.cc.u32 %2, %2, %10;\n\t"
      "addc.cc.u32 %3, %3, %11;\n\t"
      "addc.cc.u32 %4, %4, %12;\n\t"
      "addc.cc.u32 %5, %5, %13;\n\t"
      "addc.cc.u32 %6, %6, %14;\n\t"
      "addc.u32 %7, %7, %15;"
      : "+r"(s[0]), "+r"(s[1]), "+r"(s[2]), "+r"(s[3]), "+r"(s[4]), "+r"(s[5]), "+r"(s[6]), "+r"(s[7])
      : "r"(f.p(0) & bw), "r"(f.p(1) & bw), "r"(f.p(2) & bw), "r"(f.p(3) & bw), "r"(f.p(4) & bw),
        "r"(f.p(5) & bw), "r"(f.p(6) & bw), "r"(f.p(7) & bw));
  fe_copy(r, s);
}

// r = -a mod p (0 stays 0).
template <class F>
__device__ __forceinline__ void fe_neg(uint32_t r[8], const uint32_t a[8], const F& f) {
  uint32_t z[8];
  fe_zero(z);
  fe_sub(r, z, a, f);
}

// r = a * b * 2^-256 mod p, canonical. r may alias a and/or b.
//
// CIOS (coarsely integrated operand scanning): for each word b_i, a row
// t += a b_i, then a row t = (t + m p) / 2^32 with m = t_0 (-p^-1) mod 2^32.
// Each word step is one 32 x 32 -> 64-bit multiply-add whose high half is the
// next step's carry (t_j + a_j b_i + c <= 2^64 - 1 never overflows). The
// compiler maps a step onto a single wide multiply-add, so the carry travels
// in a register instead of the condition code, and the two rows of a step can
// overlap: measured on B200, 30 % lower latency than the same rows written as
// PTX carry-flag chains (mad.lo.cc / madc.hi.cc) and 3 % more throughput, with
// bit-identical results.
template <class F>
__device__ __forceinline__ void fe_mul(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                       const F& f) {
  uint32_t x[8], y[8], t[9];
  fe_copy(x, a);
  fe_copy(y, b);
#pragma unroll
  for (int j = 0; j < 9; ++j) t[j] = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    uint64_t c = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint64_t p = (uint64_t)x[j] * y[i] + t[j] + c;
      t[j] = (uint32_t)p;
      c = p >> 32;
    }
    // t < 2p before the step and the step total stays below 2^288, so t[8] + c fits 32 bits
    t[8] += (uint32_t)c;
    const uint32_t m = t[0] * f.ninv();
    uint64_t q = (uint64_t)m * f.p(0) + t[0];
    c = q >> 32;
#pragma unroll
    for (int j = 1; j < 8; ++j) {
      q = (uint64_t)m * f.p(j) + t[j] + c;
      t[j - 1] = (uint32_t)q;
      c = q >> 32;
    }
    t[7] = t[8] + (uint32_t)c;
    t[8] = 0;
  }
  fe_reduce_once(t, f);
  fe_copy(r, t);
}

// r = a^2 * 2^-256 mod p, canonical; r may alias a.
//
// SOS (separated operand scanning): the 512-bit square first, each
// off-diagonal product a_i a_j (i < j) computed once and the sum doubled,
// then the diagonal a_i^2: 36 word products instead of 64. Then eight
// Montgomery rows t = t + m p 2^(32 i), m = t_i (-p^-1) mod 2^32, as in fe_mul
// (64 products). With a < p < 2^255 every partial sum stays below 2^512, so
// 16 words hold it, and the result (t / 2^256 < 2p) needs one conditional
// subtraction. A row's carry out of word i + 8 (0 or 1) is added one word
// higher by the next row.
template <class F>
__device__ __forceinline__ void fe_sqr(uint32_t r[8], const uint32_t a[8], const F& f) {
  uint32_t x[8], t[16];
  fe_copy(x, a);
#pragma unroll
  for (int k = 0; k < 16; ++k) t[k] = 0;
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    uint64_t c = 0;
#pragma unroll
    for (int j = i + 1; j < 8; ++j) {
      const uint64_t q = (uint64_t)x[i] * x[j] + t[i + j] + c;
      t[i + j] = (uint32_t)q;
      c = q >> 32;
    }
    t[i + 8] = (uint32_t)c;  // no earlier row reached word i + 8
  }
  // double the off-diagonal sum (words 1..14 -> 1..15)
  t[15] = t[14] >> 31;
#pragma unroll
  for (int k = 14; k >= 1; --k) t[k] = __funnelshift_l(t[k - 1], t[k], 1);
  uint64_t c = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    uint64_t q = (uint64_t)x[i] * x[i] + t[2 * i] + c;
    t[2 * i] = (uint32_t)q;
    q = (uint64_t)t[2 * i + 1] + (q >> 32);
    t[2 * i + 1] = (uint32_t)q;
    c = q >> 32;
  }
  uint32_t hc = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const uint32_t m = t[i] * f.ninv();
    uint64_t q = (uint64_t)m * f.p(0) + t[i];
    c = q >> 32;
#pragma unroll
    for (int j = 1; j < 8; ++j) {
      q = (uint64_t)m * f.p(j) + t[i + j] + c;
      t[i + j] = (uint32_t)q;
      c = q >> 32;
    }
    q = (uint64_t)t[i + 8] + c + hc;
    t[i + 8] = (uint32_t)q;
    hc = (uint32_t)(q >> 32);
  }
  uint32_t out[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) out[j] = t[8 + j];
  fe_reduce_once(out, f);
  fe_copy(r, out);
}

// ---- one shared copy of the product ----------------------------------------
// Kernels whose loop bodies hold many products (the bucket additions, the NTT
// butterflies) outgrow the SM's instruction cache when every product is
// expanded in place, and their warps then stall on instruction fetch.
// fe_mul_shared calls one out-of-line copy of the product per field instead;
// the operands travel by value in registers (no stack frame), so a call adds
// a few register moves to the ~470 instructions of the product. Fields with
// a modulus known only at run time keep the inline product.
struct Fe8 {
  uint32_t w[8];
};

template <class F>
static __device__ __noinline__ Fe8 fe_mul_outlined(const Fe8 a, const Fe8 b) {
  Fe8 r;
  fe_mul(r.w, a.w, b.w, F{});
  return r;
}

template <class F>
static __device__ __noinline__ Fe8 fe_sqr_outlined(const Fe8 a) {
  Fe8 r;
  fe_sqr(r.w, a.w, F{});
  return r;
}

// the squaring's shared copy, as fe_mul_shared
template <class F>
__device__ __forceinline__ void fe_sqr_shared(uint32_t r[8], const uint32_t a[8], const F&) {
  Fe8 x;
#pragma unroll
  for (int j = 0; j < 8; ++j) x.w[j] = a[j];
  const Fe8 z = fe_sqr_outlined<F>(x);
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = z.w[j];
}

__device__ __forceinline__ void fe_sqr_shared(uint32_t r[8], const uint32_t a[8], const FieldRT& f) {
  fe_sqr(r, a, f);
}

template <class F>
__device__ __forceinline__ void fe_mul_shared(uint32_t r[8], const uint32_t a[8],
                                              const uint32_t b[8], const F&) {
  Fe8 x, y;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    x.w[j] = a[j];
    y.w[j] = b[j];
  }
  const Fe8 z = fe_mul_outlined<F>(x, y);
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = z.w[j];
}

__device__ __forceinline__ void fe_mul_shared(uint32_t r[8], const uint32_t a[8],
                                              const uint32_t b[8], const FieldRT& f) {
  fe_mul(r, a, b, f);
}

// r = 2a, 3a, 4a, 8a mod p.
template <class F>
__device__ __forceinline__ void fe_dbl(uint32_t r[8], const uint32_t a[8], const F& f) {
  fe_add(r, a, a, f);
}

// Montgomery form of a plain canonical value: a * R^2 * R^-1 = aR
// (zkgpu/field256_gpu.py:307-310).
template <class F>
__device__ __forceinline__ void fe_to_mont(uint32_t r[8], const uint32_t a[8], const F& f) {
  uint32_t r2[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) r2[j] = f.r2(j);
  fe_mul(r, a, r2, f);
}

// Plain value of a Montgomery-form element: aR * 1 * R^-1 = a
// (zkgpu/field256_gpu.py:318-319).
template <class F>
__device__ __forceinline__ void fe_from_mont(uint32_t r[8], const uint32_t a[8], const F& f) {
  uint32_t one[8] = {1, 0, 0, 0, 0, 0, 0, 0};
  fe_mul(r, a, one, f);
}

// r = a^e for a 256-bit exponent e (little-endian limbs), left to right.
template <class F>
__device__ __noinline__ void fe_pow(uint32_t r[8], const uint32_t a[8], const uint32_t e[8],
                                    const F& f) {
  uint32_t acc[8], base[8];
  fe_one(acc, f);
  fe_copy(base, a);
  for (int w = 7; w >= 0; --w) {
    for (int bit = 31; bit >= 0; --bit) {
      fe_sqr(acc, acc, f);
      if ((e[w] >> bit) & 1u) fe_mul(acc, acc, base, f);
    }
  }
  fe_copy(r, acc);
}

// r = a^-1 = a^(p-2) (Fermat); a must be non-zero.
template <class F>
__device__ __forceinline__ void fe_inv(uint32_t r[8], const uint32_t a[8], const F& f) {
  uint32_t e[8];
  // e = p - 2, borrowing through the limbs (a low limb of 0 or 1 borrows)
  uint32_t borrow = 2;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t pj = f.p(j);
    e[j] = pj - borrow;
    borrow = pj < borrow ? 1u : 0u;
  }
  fe_pow(r, a, e, f);
}

// Compare a plain 256-bit value with p: true when a < p.
template <class F>
__device__ __forceinline__ bool fe_lt_p(const uint32_t a[8], const F& f) {
  uint32_t d, bw;
  asm("sub.cc.u32 %0, %2, %10;\n\t"
      "subc.cc.u32 %0, %3, %11;\n\t"
      "subc.cc.u32 %0, %4, %12;\n\t"
      "subc.cc.u32 %0, %5, %13;\n\t"
      "subc.cc.u32 %0, %6, %14;\n\t"
      "subc.cc.u32 %0, %7, %15;\n\t"
      "subc.cc.u32 %0, %8, %16;\n\t"
      "subc.cc.u32 %0, %9, %17;\n\t"
      "subc.u32 %1, 0, 0;"
      : "=r"(d), "=r"(bw)
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
        "r"(f.p(0)), "r"(f.p(1)), "r"(f.p(2)), "r"(f.p(3)), "r"(f.p(4)), "r"(f.p(5)), "r"(f.p(6)),
        "r"(f.p(7)));
  return bw != 0;
}

// a := a - p (no check; the caller knows a >= p).
template <class F>
__device__ __forceinline__ void fe_sub_p(uint32_t a[8], const F& f) {
  asm("sub.cc.u32 %0, %0, %8;\n\t"
      "subc.cc.u32 %1, %1, %9;\n\t"
      "subc.cc.u32 %2, %2, %10;\n\t"
      "subc.cc.u32 %3, %3, %11;\n\t"
      "subc.cc.u32 %4, %4, %12;\n\t"
      "subc.cc.u32 %5, %5, %13;\n\t"
      "subc.cc.u32 %6, %6, %14;\n\t"
      "subc.u32 %7, %7, %15;"
      : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7])
      : "r"(f.p(0)), "r"(f.p(1)), "r"(f.p(2)), "r"(f.p(3)), "r"(f.p(4)), "r"(f.p(5)), "r"(f.p(6)),
        "r"(f.p(7)));
}

// Reduce any 256-bit value into [0, p) by repeated subtraction. For BN254
// (p > 2^253) at most five subtractions are needed; for a general modulus the
// caller reduces on the host instead.
template <class F>
__device__ __forceinline__ void fe_reduce_full(uint32_t a[8], const F& f, int max_sub) {
  for (int k = 0; k < max_sub; ++k) {
    if (fe_lt_p(a, f)) break;
    fe_sub_p(a, f);
  }
}

}  // namespace zkb
