// field64.cu — prime-field arithmetic on 64-bit words (moduli below 2^63)
// and an NTT over them, with their C ABI: the reference's int64 path
// (zkgpu/field_gpu.py: gpu_batch_mul / gpu_batch_add / gpu_batch_pow;
// zkgpu/ntt_gpu.py: ntt_gpu), for fields whose elements fit one word.
//
// Inputs are any int64 values and are reduced into [0, m) first (floor
// semantics, so negative values land in the field, zkgpu/field_gpu.py:46-56).
// Products: for an odd modulus, Montgomery multiplication with R = 2^64 (four
// 64-bit multiply halves and one conditional subtraction: a, b < m < 2^63
// keep every intermediate below 2^64); for an even modulus, the exact 128-bit
// product and its remainder.
#include <cstring>

#include "common.cuh"
#include "profile.h"

namespace zkb {

struct Mod64 {
  uint64_t m;
  uint64_t ninv;  // -m^-1 mod 2^64 (odd m)
  uint64_t r2;    // 2^128 mod m (odd m)
  int odd;
};

static Mod64 make_mod64(uint64_t m) {
  Mod64 M;
  M.m = m;
  M.odd = (int)(m & 1);
  M.ninv = 0;
  M.r2 = 0;
  if (M.odd) {
    uint64_t x = m;  // Newton: correct to 3 bits for odd m, doubling each step
    for (int i = 0; i < 6; ++i) x *= 2 - m * x;
    M.ninv = (uint64_t)0 - x;
    const unsigned __int128 r = ((unsigned __int128)1 << 64) % m;  // R mod m
    M.r2 = (uint64_t)((r * r) % m);
  }
  return M;
}

// a b R^-1 mod m for a, b < m < 2^63, m odd
__device__ __forceinline__ uint64_t mont64(uint64_t a, uint64_t b, const Mod64& M) {
  const uint64_t lo = a * b, hi = __umul64hi(a, b);
  const uint64_t u = lo * M.ninv;
  const uint64_t uhi = __umul64hi(u, M.m);
  const uint64_t r = hi + uhi + (lo != 0);  // lo + u m is 0 or 2^64 in the low word
  const uint64_t d = r - M.m;  // r < 2m < 2^64: d is negative as int64 exactly when r < m
  return (int64_t)d < 0 ? r : d;
}

// x mod m in [0, m) for any int64 x (floor semantics). The 64-bit remainder
// measured faster here than two Montgomery reductions (0.79 against 0.89 ms
// for a 2^26-word product of full-range inputs).
__device__ __forceinline__ uint64_t reduce64(int64_t x, const Mod64& M) {
  if (x >= 0 && (uint64_t)x < M.m) return (uint64_t)x;
  const int64_t r = x % (int64_t)M.m;
  return (uint64_t)(r < 0 ? r + (int64_t)M.m : r);
}

// a b mod m for a, b < m
__device__ __forceinline__ uint64_t mulmod64(uint64_t a, uint64_t b, const Mod64& M) {
  if (M.odd) return mont64(mont64(a, b, M), M.r2, M);
  return (uint64_t)(((unsigned __int128)a * b) % M.m);
}

__device__ __forceinline__ uint64_t addmod64(uint64_t a, uint64_t b, uint64_t m) {
  const int64_t d = (int64_t)a - (int64_t)(m - b);  // in (-m, m): no overflow near 2^63
  return (uint64_t)(d < 0 ? d + (int64_t)m : d);
}

__device__ __forceinline__ uint64_t submod64(uint64_t a, uint64_t b, uint64_t m) {
  const int64_t d = (int64_t)(a - b);  // a, b < m < 2^63: the difference fits int64
  return (uint64_t)(d < 0 ? d + (int64_t)m : d);
}

template <int OP>  // 0 = mul, 1 = add
__global__ void __launch_bounds__(256) k_u64_binary(const int64_t* a, const int64_t* b, int64_t* out,
                                                    int64_t n, Mod64 M) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t x = reduce64(a[i], M), y = reduce64(b[i], M);
    out[i] = (int64_t)(OP == 0 ? mulmod64(x, y, M) : addmod64(x, y, M.m));
  }
}

// bases^e mod m, e given as little-endian 64-bit words (right-to-left
// square-and-multiply; in Montgomery form for an odd modulus, one product a step)
__global__ void __launch_bounds__(256) k_u64_pow(const int64_t* bases, int64_t* out, int64_t n,
                                                 const uint64_t* exp, int words, Mod64 M) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint64_t b = reduce64(bases[i], M), r = 1 % M.m;
    if (M.odd) {
      b = mont64(b, M.r2, M);
      r = mont64(r, M.r2, M);
    }
    for (int w = 0; w < words; ++w) {
      uint64_t e = exp[w];
      for (int bit = 0; bit < 64; ++bit) {
        if (w == words - 1 && e == 0) break;
        if (e & 1) r = M.odd ? mont64(r, b, M) : mulmod64(r, b, M);
        e >>= 1;
        b = M.odd ? mont64(b, b, M) : mulmod64(b, b, M);
      }
    }
    out[i] = (int64_t)(M.odd ? mont64(r, 1, M) : r);
  }
}

// ---- NTT over a prime m < 2^63 ---------------------------------------------
//
// Radix-2 DIT on bit-reversed input (the order of zkgpu/ntt.py:149-203), in
// one to four passes over HBM instead of one per stage; 32-bit butterflies for
// moduli below 2^31. The data stays in
// plain form and every twiddle w carries its Shoup quotient w' = floor(w 2^64 / m),
// so b w mod m = b w - umulhi(b, w') m (mod 2^64), less m at most once: about
// two thirds of a Montgomery product. w' comes without a division: from
// w 2^64 = w' m + (w R mod m), w' = (w R mod m) (-m^-1) mod 2^64.
//
// A pass loads a tile of (1 << K) rows x C = (1 << c) columns into shared
// memory, runs K stages on it and writes it back:
//  - the first pass (stages 0 .. K-1) covers bit-reversed positions
//    r = row + (tile << K) + (col << (log_n - c)); it gathers in[brev(r)],
//    whose C columns are C neighbouring input words, and reduces them into [0, m);
//  - a later pass (stages S .. S+K-1) covers r = colpart + (row << S) + (hi << (S+K))
//    with colpart = C neighbouring positions, so every row is one C-word segment;
//    the twiddle of stage S+t is w_{2^(S+t+1)}^colpart (per column, made once
//    per tile) times w_{2^(t+1)}^rlo from the stage table;
//  - the last pass multiplies by n^-1 (inverse transform) on the way out.

// Tile shapes (knobs ntt64.*, by size when unset): a tile holds at most 2^13 words
// (64 KiB) besides its twiddle rows. The passes are bound by integer issue (about 50
// instructions a butterfly in the first pass, 75 in later ones), not by HBM.
static constexpr int kNtt64MaxTileLog = 13;  // words per tile (log2)
static constexpr int kNtt64MaxK = 10;        // stages per pass (the knobs' upper bounds)
static constexpr int kNtt64Threads = 256;

struct Ntt64Roots {
  uint64_t p[32];  // p[k] = omega^(2^k) R mod m, k < log_n
};

struct Tw64 {
  uint64_t w, q;  // plain twiddle and its Shoup quotient
};

// b w mod m for any b < 2^64 and w < m
__device__ __forceinline__ uint64_t shoup64(uint64_t b, Tw64 t, uint64_t m) {
  const uint64_t q = __umul64hi(b, t.q);
  const uint64_t r = b * t.w - q * m;  // in [0, 2m)
  const uint64_t d = r - m;
  return (int64_t)d < 0 ? r : d;
}

// the twiddle pair of w R mod m (Montgomery form)
__device__ __forceinline__ Tw64 tw64_from_mont(uint64_t wm, const Mod64& M) {
  return Tw64{mont64(wm, 1, M), wm * M.ninv};
}

// Moduli below 2^31 (most NTT-friendly primes: 998244353, 7340033, 12289) take
// the same butterflies in 32-bit words (k32): Shoup's product with the quotient
// floor(w 2^32 / m), which is the stored floor(w 2^64 / m) shifted down by 32.
// b w mod m for b < 2^32 and w < m < 2^31.
__device__ __forceinline__ uint32_t shoup32(uint32_t b, uint32_t w, uint32_t q, uint32_t m) {
  const uint32_t r = b * w - __umulhi(b, q) * m;  // in [0, 2m)
  return r >= m ? r - m : r;
}

template <bool k32>
__device__ __forceinline__ uint64_t mulw64(uint64_t b, Tw64 t, uint64_t m) {
  if (k32) return shoup32((uint32_t)b, (uint32_t)t.w, (uint32_t)(t.q >> 32), (uint32_t)m);
  return shoup64(b, t, m);
}

// (a, b) <- (a + b w, a - b w)
template <bool k32>
__device__ __forceinline__ void bfly64(uint64_t& a, uint64_t& b, Tw64 w, uint64_t m) {
  const uint64_t v = mulw64<k32>(b, w, m), u = a;
  if (k32) {
    const uint32_t x = (uint32_t)u, y = (uint32_t)v, mm = (uint32_t)m, sum = x + y;  // < 2^32
    a = sum >= mm ? sum - mm : sum;
    b = x >= y ? x - y : x + (mm - y);
    return;
  }
  a = addmod64(u, v, m);
  b = submod64(u, v, m);
}

// the same with the twiddle given as two factors: (a, b) <- (a + b w1 w2, a - b w1 w2)
template <bool k32>
__device__ __forceinline__ void bfly64(uint64_t& a, uint64_t& b, Tw64 w1, Tw64 w2, uint64_t m) {
  uint64_t t = mulw64<k32>(b, w1, m);
  bfly64<k32>(a, t, w2, m);
  b = t;
}

// omega^e R from the powers omega^(2^k) R (one product per set bit of e)
__device__ __forceinline__ uint64_t ntt64_root_pow(const Ntt64Roots& P, uint64_t e, uint64_t one,
                                                   const Mod64& M) {
  uint64_t r = one;
  for (int k = 0; e; ++k, e >>= 1) {
    if (e & 1) r = mont64(r, P.p[k], M);
  }
  return r;
}

// stage table: entry 2^t + j = w_{2^(t+1)}^j = omega^(j << (log_n - 1 - t)), 1 <= 2^t + j < count
__global__ void __launch_bounds__(256) k_ntt64_stage_table(Tw64* tst, int count, int log_n, Ntt64Roots P,
                                                           uint64_t one, Mod64 M) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
    uint64_t wm = one;
    if (idx > 0) {
      const int t = 31 - __clz(idx);
      wm = ntt64_root_pow(P, (uint64_t)(idx - (1 << t)) << (log_n - 1 - t), one, M);
    }
    tst[idx] = tw64_from_mont(wm, M);
  }
}

template <bool kFirst, bool k32>
__global__ void __launch_bounds__(kNtt64Threads) k_ntt64_pass(const int64_t* in, int64_t* out, int log_n, int S,
                                                              int K, int c, const Tw64* tst, Ntt64Roots P,
                                                              uint64_t one, Tw64 scale, int scaled, Mod64 M) {
  // dynamic shared memory: the tile, (1 << K) rows x (1 << c) columns, column
  // fastest; the stage table's first 2^K entries; per stage and column the factor
  // w_{2^(S+t+1)}^colpart as a twiddle pair and in Montgomery form (later passes)
  extern __shared__ uint64_t s[];
  const uint64_t m = M.m;
  const int C = 1 << c, E = C << K;
  Tw64* tw = reinterpret_cast<Tw64*>(s + E);
  Tw64* base = tw + (1 << K);                                      // [t * C + col]
  uint64_t* base_m = reinterpret_cast<uint64_t*>(base + (kFirst ? 0 : K * C));
  const int64_t tile = blockIdx.x;
  // tile -> the bits of r outside the tile's rows and columns
  int64_t fixed;
  int64_t colbase = 0;
  if (kFirst) {
    fixed = tile << K;
  } else {
    const int64_t lo_tiles = (int64_t)1 << (S - c);
    colbase = (tile & (lo_tiles - 1)) << c;
    fixed = colbase + ((tile >> (S - c)) << (S + K));
  }
  for (int i = threadIdx.x; i < (1 << K); i += blockDim.x) tw[i] = tst[i];
  if (!kFirst && threadIdx.x < C) {
    // w_{2^(S+K)}^colpart, then squares down to stage S
    uint64_t b = ntt64_root_pow(P, (uint64_t)(colbase + threadIdx.x) << (log_n - S - K), one, M);
    for (int t = K - 1; t >= 0; --t) {
      base[t * C + threadIdx.x] = tw64_from_mont(b, M);
      base_m[t * C + threadIdx.x] = b;
      b = mont64(b, b, M);
    }
  }
  // Tile load by cp.async: every word of the thread in flight at once, no registers
  // held (a plain load loop kept about one load per thread in flight).
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    const int64_t col = e & (C - 1), row = e >> c;
    const int64_t* src;
    if (kFirst) {
      const int64_t r = fixed + row + (col << (log_n - c));
      src = in + (log_n ? (int64_t)(__brevll((unsigned long long)r) >> (64 - log_n)) : 0);
    } else {
      src = out + fixed + col + (row << S);
    }
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(s + e)),
                 "l"(src));
  }
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
  if (kFirst) {  // the same words this thread copied: reduce into [0, m)
    for (int e = threadIdx.x; e < E; e += blockDim.x) s[e] = reduce64((int64_t)s[e], M);
  }
  __syncthreads();
  // The twiddle of stage S+t at row offset x < 2^t is w_{2^(t+1)}^x, times
  // w_{2^(S+t+1)}^colpart in a later pass. A thread whose row offset is the same in
  // every group it takes (blockDim a multiple of C << t) makes the product pair once;
  // otherwise each butterfly applies the two factors in turn.
  auto composed = [&](int t, int x, int col) {
    if (kFirst) return tw[(1 << t) + x];
    const uint64_t wm = mont64(base_m[t * C + col], mont64(tw[(1 << t) + x].w, M.r2, M), M);
    return tw64_from_mont(wm, M);
  };
  // Radix-4 steps: stages t and t+1 on four rows r0 + {0, h, 2h, 3h} (h = 2^t) held in
  // registers, one barrier per two stages; a radix-2 stage closes an odd K.
  int t = 0;
  for (; t + 1 < K; t += 2) {
    const int h = 1 << t, d = h << c;
    const bool invariant = kFirst || ((blockDim.x >> c) & (h - 1)) == 0;
    Tw64 f0{0, 0}, f1{0, 0}, f2{0, 0};
    if (invariant) {
      const int col = threadIdx.x & (C - 1), rlo = (threadIdx.x >> c) & (h - 1);
      if (!kFirst) {
        f0 = composed(t, rlo, col);
        f1 = composed(t + 1, rlo, col);
        f2 = composed(t + 1, rlo + h, col);
      }
    }
    for (int g = threadIdx.x; g < E / 4; g += blockDim.x) {
      const int col = g & (C - 1), q = g >> c;
      const int rlo = q & (h - 1);
      const int i0 = ((((q >> t) << (t + 2)) | rlo) << c) | col;
      uint64_t x0 = s[i0], x1 = s[i0 + d], x2 = s[i0 + 2 * d], x3 = s[i0 + 3 * d];
      if (kFirst) {
        const Tw64 w0 = tw[h + rlo], w1 = tw[2 * h + rlo], w2 = tw[3 * h + rlo];
        bfly64<k32>(x0, x1, w0, m);
        bfly64<k32>(x2, x3, w0, m);
        bfly64<k32>(x0, x2, w1, m);
        bfly64<k32>(x1, x3, w2, m);
      } else if (invariant) {
        bfly64<k32>(x0, x1, f0, m);
        bfly64<k32>(x2, x3, f0, m);
        bfly64<k32>(x0, x2, f1, m);
        bfly64<k32>(x1, x3, f2, m);
      } else {
        const Tw64 w0 = tw[h + rlo], w1 = tw[2 * h + rlo], w2 = tw[3 * h + rlo];
        const Tw64 b0 = base[t * C + col], b1 = base[(t + 1) * C + col];
        bfly64<k32>(x0, x1, w0, b0, m);
        bfly64<k32>(x2, x3, w0, b0, m);
        bfly64<k32>(x0, x2, w1, b1, m);
        bfly64<k32>(x1, x3, w2, b1, m);
      }
      s[i0] = x0;
      s[i0 + d] = x1;
      s[i0 + 2 * d] = x2;
      s[i0 + 3 * d] = x3;
    }
    __syncthreads();
  }
  if (t < K) {
    const int h = 1 << t, d = h << c;
    for (int b = threadIdx.x; b < E / 2; b += blockDim.x) {
      const int col = b & (C - 1), q = b >> c;
      const int rlo = q & (h - 1);
      const int i0 = ((((q >> t) << (t + 1)) | rlo) << c) | col;
      uint64_t x0 = s[i0], x1 = s[i0 + d];
      if (kFirst) {
        bfly64<k32>(x0, x1, tw[h + rlo], m);
      } else {
        bfly64<k32>(x0, x1, tw[h + rlo], base[t * C + col], m);
      }
      s[i0] = x0;
      s[i0 + d] = x1;
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    const int64_t col = e & (C - 1), row = e >> c;
    const int64_t r = kFirst ? fixed + row + (col << (log_n - c)) : fixed + col + (row << S);
    out[r] = (int64_t)(scaled ? mulw64<k32>(s[e], scale, m) : s[e]);
  }
}

struct Ntt64Pass {
  int S, K, c;
};

// first pass: stages 0 .. K1-1 on tiles of 2^c1 columns (none below 2^(2 c1)); the
// rest split evenly into passes of at most kL stages on 2^c-column tiles. Shapes by
// size, measured on B200 (ms for the forward transform by (c1, K1, c, kL), over a
// 63-bit modulus / over 998244353, whose butterflies are 32-bit; every shape of
// {5 8, 4 9, 3 10} x {5 8, 4 9, 3 10} timed, the best and the runner-up given):
// 2^16: (3, 10, 3, 10) 0.036 / 0.030, (5, 8, 5, 8) 0.051 / 0.039;
// 2^20: (3, 10, 3, 10) 0.056 / 0.040, (5, 8, 5, 8) 0.069 / 0.052;
// 2^22: (5, 8, 5, 8) 0.183 / 0.124, (4, 9, 5, 8) 0.188 / 0.128;
// 2^23: (5, 8, 5, 8) 0.337 / 0.215, (3, 9, 4, 8) 0.378 / 0.264;
// 2^24: (4, 9, 5, 8) 0.655, (3, 9, 4, 8) 0.688;
// 2^25: (3, 9, 4, 8) 1.26, (3, 10, 5, 8) 1.29, (5, 8, 5, 8) 2.27.
static int plan_ntt64(int log_n, Ntt64Pass* passes) {
  int dcf = 3, dkf = 9, dcl = 4, dkl = 8;  // from 2^25
  if (log_n <= 20) {
    dcf = 3, dkf = 10, dcl = 3, dkl = 10;
  } else if (log_n <= 23) {
    dcf = 5, dkf = 8, dcl = 5, dkl = 8;
  } else if (log_n == 24) {
    dcf = 4, dkf = 9, dcl = 5, dkl = 8;
  }
  int cf = (int)tune_get("ntt64.first_col_log"), kf = (int)tune_get("ntt64.first_max_k");
  int cl = (int)tune_get("ntt64.col_log"), kL = (int)tune_get("ntt64.max_k");
  if (cf < 0) cf = dcf;
  if (kf < 4) kf = dkf;
  if (cl < 1) cl = dcl;
  if (kL < 2) kL = dkl;
  const int c1 = log_n >= 2 * cf ? cf : 0;
  int K1 = log_n - c1 < kf ? log_n - c1 : kf;
  if (K1 + c1 > kNtt64MaxTileLog) K1 = kNtt64MaxTileLog - c1;
  int count = 0;
  passes[count++] = {0, K1, c1};
  const int rest = log_n - K1;
  if (rest > 0) {
    const int c = K1 < cl ? K1 : cl;  // columns within the low S bits
    if (kL + c > kNtt64MaxTileLog) kL = kNtt64MaxTileLog - c;
    const int P = (rest + kL - 1) / kL;
    int S = K1;
    for (int p = 0; p < P; ++p) {
      const int K = rest / P + (p < rest % P ? 1 : 0);
      passes[count++] = {S, K, c};
      S += K;
    }
  }
  return count;
}

static int check_mod64(int64_t mod) {
  if (mod < 2) return fail(ZKB_EINVAL, "mod must satisfy 2 <= mod < 2^63 to fit in int64, got %lld",
                           (long long)mod);
  return ZKB_OK;
}

}  // namespace zkb

using namespace zkb;

extern "C" {

int zkb_u64_mul(const int64_t* a, const int64_t* b, int64_t* out, int64_t n, int64_t mod, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_mod64(mod));
  if (n < 0) return fail(ZKB_EINVAL, "negative length");
  if (n == 0) return ZKB_OK;
  if (!a || !b || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(a, 8, "a"));
  ZKB_TRY(check_align(b, 8, "b"));
  ZKB_TRY(check_align(out, 8, "out"));
  cudaStream_t s = as_stream(stream);
  k_u64_binary<0><<<grid_for(n, 256), 256, 0, s>>>(a, b, out, n, make_mod64((uint64_t)mod));
  return check_launch("int64 field mul");
}

int zkb_u64_add(const int64_t* a, const int64_t* b, int64_t* out, int64_t n, int64_t mod, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_mod64(mod));
  if (n < 0) return fail(ZKB_EINVAL, "negative length");
  if (n == 0) return ZKB_OK;
  if (!a || !b || !out) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(a, 8, "a"));
  ZKB_TRY(check_align(b, 8, "b"));
  ZKB_TRY(check_align(out, 8, "out"));
  cudaStream_t s = as_stream(stream);
  k_u64_binary<1><<<grid_for(n, 256), 256, 0, s>>>(a, b, out, n, make_mod64((uint64_t)mod));
  return check_launch("int64 field add");
}

int zkb_u64_pow(const int64_t* bases, int64_t* out, int64_t n, const uint64_t* exp_words, int words,
                int64_t mod, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_mod64(mod));
  if (n < 0 || words < 0) return fail(ZKB_EINVAL, "negative length");
  if (n == 0) return ZKB_OK;
  if (!bases || !out || (words && !exp_words)) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(bases, 8, "bases"));
  ZKB_TRY(check_align(out, 8, "out"));
  ZKB_TRY(check_align(exp_words, 8, "exponent"));
  cudaStream_t s = as_stream(stream);
  k_u64_pow<<<grid_for(n, 256), 256, 0, s>>>(bases, out, n, exp_words, words, make_mod64((uint64_t)mod));
  return check_launch("int64 field pow");
}

size_t zkb_ntt64_workspace_bytes(int64_t n) {
  if (n <= 0) return 0;
  return (size_t)(1 << kNtt64MaxK) * sizeof(Tw64) + 256;  // the stage table
}

int zkb_ntt64(const int64_t* in, int64_t* out, int64_t n, int64_t mod, int64_t omega, int invert,
              void* workspace, size_t workspace_bytes, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_mod64(mod));
  if ((mod & 1) == 0) return fail(ZKB_EINVAL, "the NTT needs an odd prime modulus, got %lld", (long long)mod);
  if (n < 0 || (n & (n - 1)) || n > (1ll << 30)) {
    return fail(ZKB_EINVAL, "NTT length must be a power of 2 up to 2^30, got %lld", (long long)n);
  }
  if (n == 0) return ZKB_OK;
  if (!in || !out) return fail(ZKB_EINVAL, "null buffer");
  const uintptr_t ia = reinterpret_cast<uintptr_t>(in), oa = reinterpret_cast<uintptr_t>(out);
  const uintptr_t bytes = (uintptr_t)n * 8;
  if (ia < oa + bytes && oa < ia + bytes) return fail(ZKB_EINVAL, "in and out must not overlap");
  if (omega <= 0 || omega >= mod) return fail(ZKB_EINVAL, "root of unity out of range");
  ZKB_TRY(check_align(in, 8, "in"));
  ZKB_TRY(check_align(out, 8, "out"));
  ZKB_TRY(check_align(workspace, 8, "workspace"));
  if (!workspace || workspace_bytes < zkb_ntt64_workspace_bytes(n)) {
    return fail(ZKB_EWORKSPACE, "NTT of %lld words needs %zu workspace bytes, got %zu", (long long)n,
                zkb_ntt64_workspace_bytes(n), workspace_bytes);
  }
  const Mod64 M = make_mod64((uint64_t)mod);
  int log_n = 0;
  while ((1ll << log_n) < n) ++log_n;
  // host-side constants: powers omega^(2^k) in Montgomery form (omega^-1 for an
  // inverse transform: x^-1 = x^(m-2), m prime) and the final factor n^-1
  const uint64_t m = (uint64_t)mod;
  auto mulm = [m](uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) % m); };
  auto powmod = [m, &mulm](uint64_t b, uint64_t e) {
    uint64_t r = 1 % m;
    for (b %= m; e; e >>= 1) {
      if (e & 1) r = mulm(r, b);
      b = mulm(b, b);
    }
    return r;
  };
  const uint64_t R = (uint64_t)(((unsigned __int128)1 << 64) % m);
  Ntt64Roots P;
  std::memset(&P, 0, sizeof(P));
  uint64_t w = invert ? powmod((uint64_t)omega, m - 2) : (uint64_t)omega;
  for (int k = 0; k < log_n; ++k, w = mulm(w, w)) P.p[k] = mulm(w, R);
  const uint64_t one = R;
  // n^-1 (inverse transform) as a twiddle pair: plain value and floor(v 2^64 / m)
  const uint64_t ninv_n = invert ? powmod((uint64_t)n, m - 2) : 1;
  const Tw64 scale{ninv_n, (uint64_t)(((unsigned __int128)ninv_n << 64) / m)};
  Tw64* tst = reinterpret_cast<Tw64*>(workspace);
  cudaStream_t s = as_stream(stream);
  Ntt64Pass passes[32];
  const int count = plan_ntt64(log_n, passes);
  int table = 1;
  for (int i = 0; i < count; ++i) table = (1 << passes[i].K) > table ? 1 << passes[i].K : table;
  k_ntt64_stage_table<<<(table + 255) / 256, 256, 0, s>>>(tst, table, log_n, P, one, M);
  ZKB_TRY(check_launch("int64 NTT stage table"));
  for (int i = 0; i < count; ++i) {
    const Ntt64Pass& p = passes[i];
    const unsigned tiles = (unsigned)(n >> (p.K + p.c));
    const size_t smem = ((size_t)8 << (p.K + p.c)) + ((size_t)sizeof(Tw64) << p.K) +
                        (i == 0 ? 0 : (size_t)(p.K << p.c) * (sizeof(Tw64) + 8));
    const int scaled = invert && i == count - 1;
    const bool k32 = m < (1ull << 31);
    auto kern = i == 0 ? (k32 ? k_ntt64_pass<true, true> : k_ntt64_pass<true, false>)
                       : (k32 ? k_ntt64_pass<false, true> : k_ntt64_pass<false, false>);
    ZKB_TRY(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                       "int64 NTT shared memory attribute"));
    ProfSpan span(i == 0 ? "ntt64_first_pass" : "ntt64_later_pass", s);
    kern<<<tiles, kNtt64Threads, smem, s>>>(in, out, log_n, p.S, p.K, p.c, tst, P, one, scale, scaled, M);
    ZKB_TRY(check_launch("int64 NTT pass"));
  }
  return ZKB_OK;
}

}  // extern "C"
