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
// total is below 2^32 * 2p < 2^288. fe_mul adds each row as two carry-flag
// chains of multiply-adds (even and odd words of a); fe_mul2 and the squaring
// use rows of eight independent 32 x 32 -> 64-bit multiply-adds recombined by
// one add chain. Both are inline PTX; fe_mul has the measurements.
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
// The two 32-bit halves of a 64-bit value (a register pair: no instruction).
__device__ __forceinline__ void split64(uint64_t v, uint32_t& lo, uint32_t& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(v));
}

// t[1..8] := lo[1..7] + hi[0..7] one word up, plus t[8] at the top:
// word k (k = 1..7) takes lo[k] + hi[k-1], word 8 takes T8 + hi[7], one
// carry-flag chain. O0..O7 name the eight output words.
#define ZKB_ROW_CHAIN(O0, O1, O2, O3, O4, O5, O6, O7, T8, lo, hi)                                  \
  asm("add.cc.u32 %0, %9, %16;\n\t"                                                                \
      "addc.cc.u32 %1, %10, %17;\n\t"                                                              \
      "addc.cc.u32 %2, %11, %18;\n\t"                                                              \
      "addc.cc.u32 %3, %12, %19;\n\t"                                                              \
      "addc.cc.u32 %4, %13, %20;\n\t"                                                              \
      "addc.cc.u32 %5, %14, %21;\n\t"                                                              \
      "addc.cc.u32 %6, %15, %22;\n\t"                                                              \
      "addc.u32 %7, %8, %23;"                                                                      \
      : "=r"(O0), "=r"(O1), "=r"(O2), "=r"(O3), "=r"(O4), "=r"(O5), "=r"(O6), "=r"(O7)             \
      : "r"(T8), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]),           \
        "r"(lo[7]), "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]), "r"(hi[4]), "r"(hi[5]),        \
        "r"(hi[6]), "r"(hi[7]))

// t[0..9] += (a0, a2, a4, a6) b at words 0, 2, 4, 6: each product's low half
// lands on an even word and its high half on the next odd word, in one
// carry-flag chain of multiply-adds; the last carry ripples into t[8], t[9].
__device__ __forceinline__ void mac_even(uint32_t t[10], uint32_t a0, uint32_t a2, uint32_t a4, uint32_t a6,
                                         uint32_t b) {
  asm("mad.lo.cc.u32 %0, %10, %14, %0;\n\t"
      "madc.hi.cc.u32 %1, %10, %14, %1;\n\t"
      "madc.lo.cc.u32 %2, %11, %14, %2;\n\t"
      "madc.hi.cc.u32 %3, %11, %14, %3;\n\t"
      "madc.lo.cc.u32 %4, %12, %14, %4;\n\t"
      "madc.hi.cc.u32 %5, %12, %14, %5;\n\t"
      "madc.lo.cc.u32 %6, %13, %14, %6;\n\t"
      "madc.hi.cc.u32 %7, %13, %14, %7;\n\t"
      "addc.cc.u32 %8, %8, 0;\n\t"
      "addc.u32 %9, %9, 0;"
      : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]),
        "+r"(t[8]), "+r"(t[9])
      : "r"(a0), "r"(a2), "r"(a4), "r"(a6), "r"(b));
}

// t[1..9] += (a1, a3, a5, a7) b at words 1, 3, 5, 7, the same way.
__device__ __forceinline__ void mac_odd(uint32_t t[10], uint32_t a1, uint32_t a3, uint32_t a5, uint32_t a7,
                                        uint32_t b) {
  asm("mad.lo.cc.u32 %0, %9, %13, %0;\n\t"
      "madc.hi.cc.u32 %1, %9, %13, %1;\n\t"
      "madc.lo.cc.u32 %2, %10, %13, %2;\n\t"
      "madc.hi.cc.u32 %3, %10, %13, %3;\n\t"
      "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"
      "madc.hi.cc.u32 %5, %11, %13, %5;\n\t"
      "madc.lo.cc.u32 %6, %12, %13, %6;\n\t"
      "madc.hi.cc.u32 %7, %12, %13, %7;\n\t"
      "addc.u32 %8, %8, 0;"
      : "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8]),
        "+r"(t[9])
      : "r"(a1), "r"(a3), "r"(a5), "r"(a7), "r"(b));
}

// CIOS (coarsely integrated operand scanning): for each word b_i, t += a b_i,
// then t = (t + m p) / 2^32 with m = t_0 (-p^-1) mod 2^32.
//
// Each t += a b_i (and t += m p) is two carry-flag chains of multiply-adds,
// one over the even words of a and one over the odd words (mac_even /
// mac_odd): within a chain no two products overlap, so every multiply-add
// takes its carry straight from the previous one. Ten words hold the sum
// (below 2^289 before the shift). Against the rows of wide multiply-adds that
// fe_mul2 and the squaring use (eight independent 32 x 32 -> 64-bit products
// joined by one add chain): bit-identical, 2.7 % more products per second in
// a loop of nothing but products, and 10 % faster NTTs (2^24: 4.95 to
// 4.47 ms, coset 5.44 to 4.91 ms, same box); the MSM's out-of-line product
// measured the same either way.
template <class F>
__device__ __forceinline__ void fe_mul_open(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                            const F& f) {
  uint32_t x[8], y[8], t[10];
  fe_copy(x, a);
  fe_copy(y, b);
#pragma unroll
  for (int j = 0; j < 10; ++j) t[j] = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    mac_even(t, x[0], x[2], x[4], x[6], y[i]);
    mac_odd(t, x[1], x[3], x[5], x[7], y[i]);
    const uint32_t m = t[0] * f.ninv();
    mac_even(t, f.p(0), f.p(2), f.p(4), f.p(6), m);
    mac_odd(t, f.p(1), f.p(3), f.p(5), f.p(7), m);
    // t[0] is zero by the choice of m: shift down one word
#pragma unroll
    for (int j = 0; j < 9; ++j) t[j] = t[j + 1];
    t[9] = 0;
  }
  fe_copy(r, t);
}

// fe_mul_open leaves out the last conditional subtraction: its result is
// (a b + M p) / 2^256 < (a b) / 2^256 + p, below 2p for a b < 2^256 p (for
// instance a < 4p and b < p when p < 2^254).
template <class F>
__device__ __forceinline__ void fe_mul(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                       const F& f) {
  uint32_t t[8];
  fe_mul_open(t, a, b, f);
  fe_reduce_once(t, f);
  fe_copy(r, t);
}

// r = (a b + c d) * 2^-256 mod p, canonical, for a, b, c, d <= p. r may alias
// any input.
//
// fe_mul's CIOS with two product rows per word i (t += a b_i, t += c d_i)
// before the Montgomery row: one reduction for the sum of two products, so
// 24 wide multiply-adds a word against 32 for two fe_mul calls and one
// conditional subtraction instead of two. Bounds: with T < 2^256 before word
// i, T + a b_i + c d_i + m p < 2^256 + 3 p 2^32 < 2^288 (word 8 never carries
// out) and the shifted sum stays below T / 2^32 + a + c + p < 2^224 + 3p < 2^256
// (p < 2^254); the final T = (ab + cd + M p) / 2^256 < 2p^2 / 2^256 + p < 2p.
// The curve formulas take Y3 = R (Q - X3) - Y1 PPP as R (Q - X3) + (p - Y1) PPP
// through it, the one place where two products are only summed.
template <class F>
__device__ __forceinline__ void fe_mul2(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                        const uint32_t c[8], const uint32_t d[8], const F& f) {
  uint32_t x[8], y[8], u[8], v[8], t[9];
  fe_copy(x, a);
  fe_copy(y, b);
  fe_copy(u, c);
  fe_copy(v, d);
#pragma unroll
  for (int j = 0; j < 9; ++j) t[j] = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    uint32_t lo[8], hi[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) split64((uint64_t)x[j] * y[i] + t[j], lo[j], hi[j]);
    ZKB_ROW_CHAIN(t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8], t[8], lo, hi);
    t[0] = lo[0];
#pragma unroll
    for (int j = 0; j < 8; ++j) split64((uint64_t)u[j] * v[i] + t[j], lo[j], hi[j]);
    ZKB_ROW_CHAIN(t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8], t[8], lo, hi);
    t[0] = lo[0];
    const uint32_t m = t[0] * f.ninv();
#pragma unroll
    for (int j = 0; j < 8; ++j) split64((uint64_t)m * f.p(j) + t[j], lo[j], hi[j]);
    ZKB_ROW_CHAIN(t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8], lo, hi);
    t[8] = 0;
  }
  fe_reduce_once(t, f);
  fe_copy(r, t);
}

// r = p - a for a <= p: the negation as an operand of fe_mul2, in [0, p]
// (a = 0 gives p, which fe_mul2 accepts). One borrow chain, no selection.
template <class F>
__device__ __forceinline__ void fe_p_minus(uint32_t r[8], const uint32_t a[8], const F& f) {
  asm("sub.cc.u32 %0, %8, %16;\n\t"
      "subc.cc.u32 %1, %9, %17;\n\t"
      "subc.cc.u32 %2, %10, %18;\n\t"
      "subc.cc.u32 %3, %11, %19;\n\t"
      "subc.cc.u32 %4, %12, %20;\n\t"
      "subc.cc.u32 %5, %13, %21;\n\t"
      "subc.cc.u32 %6, %14, %22;\n\t"
      "subc.u32 %7, %15, %23;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(f.p(0)), "r"(f.p(1)), "r"(f.p(2)), "r"(f.p(3)), "r"(f.p(4)), "r"(f.p(5)), "r"(f.p(6)),
        "r"(f.p(7)), "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]),
        "r"(a[7]));
}

// r = a^2 * 2^-256 mod p, canonical; r may alias a.
//
// SOS (separated operand scanning): the 512-bit square first, each
// off-diagonal product a_i a_j (i < j) computed once and the sum doubled,
// then the diagonal a_i^2: 36 word products instead of 64. Then eight
// Montgomery rows t = t + m p 2^(32 i), m = t_i (-p^-1) mod 2^32, as in fe_mul
// (64 products). With a < p < 2^255 every partial sum stays below 2^512, so
// 16 words hold it, and the result (t / 2^256 < 2p) needs one conditional
// subtraction. A Montgomery row is fe_mul's form (eight wide multiply-adds,
// one carry chain) at word offset i; its carry out of word i + 8 is kept in
// hc[i] and all eight are added to words 9..15 at the end (the multipliers m
// read only words 0..7, so the late carries change none of them). Measured on
// B200: 6.4 % more squarings per second than rows that pass the carry on to
// the next row, bit-identical results.
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
  uint32_t hc[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const uint32_t m = t[i] * f.ninv();
    uint32_t lo[8], hi[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) split64((uint64_t)m * f.p(j) + t[i + j], lo[j], hi[j]);
    // words i+1..i+7 take lo[j] + hi[j-1]; word i+8 takes t[i+8] + hi[7], carry to hc[i]
    asm("add.cc.u32 %0, %9, %17;\n\t"
        "addc.cc.u32 %1, %10, %18;\n\t"
        "addc.cc.u32 %2, %11, %19;\n\t"
        "addc.cc.u32 %3, %12, %20;\n\t"
        "addc.cc.u32 %4, %13, %21;\n\t"
        "addc.cc.u32 %5, %14, %22;\n\t"
        "addc.cc.u32 %6, %15, %23;\n\t"
        "addc.cc.u32 %7, %16, %24;\n\t"
        "addc.u32 %8, 0, 0;"
        : "=r"(t[i + 1]), "=r"(t[i + 2]), "=r"(t[i + 3]), "=r"(t[i + 4]), "=r"(t[i + 5]),
          "=r"(t[i + 6]), "=r"(t[i + 7]), "=r"(t[i + 8]), "=r"(hc[i])
        : "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]), "r"(lo[7]),
          "r"(t[i + 8]), "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]), "r"(hi[4]), "r"(hi[5]),
          "r"(hi[6]), "r"(hi[7]));
  }
  // hc[i] belongs at word i + 9: words 9..15 take hc[0..6]. hc[7] and the
  // carry out of word 15 are zero, since the total over 2^256 is below 2p.
  uint32_t out[8];
  asm("add.cc.u32 %0, %8, 0;\n\t"
      "addc.cc.u32 %1, %9, %16;\n\t"
      "addc.cc.u32 %2, %10, %17;\n\t"
      "addc.cc.u32 %3, %11, %18;\n\t"
      "addc.cc.u32 %4, %12, %19;\n\t"
      "addc.cc.u32 %5, %13, %20;\n\t"
      "addc.cc.u32 %6, %14, %21;\n\t"
      "addc.u32 %7, %15, %22;"
      : "=r"(out[0]), "=r"(out[1]), "=r"(out[2]), "=r"(out[3]), "=r"(out[4]), "=r"(out[5]),
        "=r"(out[6]), "=r"(out[7])
      : "r"(t[8]), "r"(t[9]), "r"(t[10]), "r"(t[11]), "r"(t[12]), "r"(t[13]), "r"(t[14]),
        "r"(t[15]), "r"(hc[0]), "r"(hc[1]), "r"(hc[2]), "r"(hc[3]), "r"(hc[4]), "r"(hc[5]),
        "r"(hc[6]));
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

template <class F>
static __device__ __noinline__ Fe8 fe_mul2_outlined(const Fe8 a, const Fe8 b, const Fe8 c, const Fe8 d) {
  Fe8 r;
  fe_mul2(r.w, a.w, b.w, c.w, d.w, F{});
  return r;
}

// the sum of two products' shared copy, as fe_mul_shared
template <class F>
__device__ __forceinline__ void fe_mul2_shared(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                               const uint32_t c[8], const uint32_t d[8], const F&) {
  Fe8 x, y, u, v;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    x.w[j] = a[j];
    y.w[j] = b[j];
    u.w[j] = c[j];
    v.w[j] = d[j];
  }
  const Fe8 z = fe_mul2_outlined<F>(x, y, u, v);
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = z.w[j];
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
