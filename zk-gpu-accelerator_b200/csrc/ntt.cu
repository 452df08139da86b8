// ntt.cu — natural-order radix-2 NTT over a 256-bit prime field, fused across
// stages, and its C ABI.
//
// Transform (zkgpu/ntt.py:149-203, zkgpu/field256_gpu.py:347-387):
//   forward  X[k] = sum_j x[j] w^(jk)            inverse  x[j] = n^-1 sum_k X[k] w^(-jk)
// with the coset forms of zkgpu/domain.py:122-135 (x[j] scaled by g^j before a
// forward transform, the result scaled by g^-j after an inverse one).
//
// Decomposition (four-step / Bailey): n = R_1 R_2 ... R_P with every R_q <= 4096.
// Pass q transforms digit q of the index (stride S_q = R_{q+1} ... R_P) for
// every fixed value of the other digits, then multiplies by the twiddle
// w_B^(j' k) of its sub-problem (B = R_q S_q, j' the lower digits, k the new
// frequency). The last pass writes X in natural order: position
// sum_q k_q S_q holds X[sum_q k_q R_1 ... R_{q-1}].
//
// Each CTA stages C columns of one pass (C * R <= 4096 elements = 128 KiB) in
// shared memory, bit-reverses them on the way in, runs all log2 R radix-2 DIT
// stages there (one Montgomery multiplication per butterfly), and applies the
// pass twiddle (and, for the first/last pass, the coset or n^-1 scaling) on
// the way out: one HBM read and one HBM write per element per pass.
#include <algorithm>
#include <cstring>
#include <list>
#include <mutex>
#include <vector>

#include "field_host.h"
#include "profile.h"
#include "tma.cuh"

namespace zkb {

static constexpr int kMaxLogR = 12;                 // largest sub-transform: 4096 points
static constexpr int kNttThreads = 512;
static constexpr int kMaxLogN = 28;

// w_{2^28} = 5^((r - 1) / 2^28) for BN254 Fr: the root every size derives from
// (zkgpu/ntt.py:74-124; snarkjs's w[28], tests/test_domain.py:15).
static const uint64_t kFrRoot28[4] = {0x9bd61b6e725b19f0ull, 0x402d111e41112ed4ull,
                                      0x00e0a7eb8ef62abcull, 0x2a3c09f0a58a7e85ull};

// ---------------------------------------------------------------------------
// Tables
// ---------------------------------------------------------------------------

// Root tables for w_N (N = 2^log_N): w_N^e = t_lo[e & (2^s - 1)] * t_hi[e >> s];
// stage tables w_fwd[j] = w_Rmax^j and w_inv[j] = w_Rmax^-j for j < Rmax / 2.
struct RootTables {
  uint64_t* t_lo = nullptr;
  uint64_t* t_hi = nullptr;
  uint64_t* w_fwd = nullptr;
  uint64_t* w_inv = nullptr;
  int log_N = 0, s = 0, log_rmax = 0;
};

// Per-transform scaling tables: forward coset: g^j = g_lo[j & m] g_hi[j >> gs];
// inverse: n^-1 g^-j (g = 1 without a coset, then only `scale` = n^-1 is used).
struct ScaleTables {
  uint64_t* g_lo = nullptr;
  uint64_t* g_hi = nullptr;
  uint64_t* scale = nullptr;  // one element: n^-1 (Montgomery)
  uint64_t* g_full = nullptr; // optional: the n products g_lo g_hi themselves (byte budget)
  size_t full_bytes = 0;
  int gs = 0;
};

template <class F>
__device__ __forceinline__ void fe_pow64(uint32_t r[8], const uint32_t base[8], uint64_t e,
                                         const F& f) {
  uint32_t acc[8], b[8];
  fe_one(acc, f);
  fe_copy(b, base);
  while (e) {
    if (e & 1) fe_mul(acc, acc, b, f);
    e >>= 1;
    if (e) fe_sqr(b, b, f);
  }
  fe_copy(r, acc);
}

// bases[0] = w (Montgomery), bases[1] = w^(2^s), bases[2] = w_Rmax = w^(N / Rmax),
// bases[3] = w_Rmax^-1 = w_Rmax^(Rmax - 1).
template <class F>
__global__ void k_root_bases(F f, const uint64_t* omega_plain, uint64_t* bases, int log_N, int s,
                             int log_rmax) {
  uint32_t w[8], t[8];
  fe_load(t, omega_plain);
  fe_to_mont(w, t, f);
  fe_store(bases, w);
  fe_pow64(t, w, 1ull << s, f);
  fe_store(bases + 4, t);
  uint32_t wr[8];
  fe_pow64(wr, w, 1ull << (log_N - log_rmax), f);
  fe_store(bases + 8, wr);
  fe_pow64(t, wr, (1ull << log_rmax) - 1, f);
  fe_store(bases + 12, t);
}

// out[i] = pre * base^i for i < count (pre = 1 when null).
template <class F>
__global__ void k_pow_table(F f, const uint64_t* base, const uint64_t* pre, uint64_t* out,
                            int64_t count) {
  uint32_t b[8], r[8];
  fe_load(b, base);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    fe_pow64(r, b, (uint64_t)i, f);
    if (pre) {
      uint32_t p[8];
      fe_load(p, pre);
      fe_mul(r, r, p, f);
    }
    fe_store(out + 4 * i, r);
  }
}

// out[i] = lo[(i << shift) & mask] * hi[(i << shift) >> s] for i < count: a two-level
// table expanded into one row per index (one product each).
template <class F>
__global__ void k_expand_table(F f, const uint64_t* lo, const uint64_t* hi, int s, int shift,
                               uint64_t* out, int64_t count) {
  const uint64_t mask = (1ull << s) - 1;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    const uint64_t e = (uint64_t)i << shift;
    uint32_t a[8], b[8];
    fe_load_nc(a, lo + 4 * (e & mask));
    fe_load_nc(b, hi + 4 * (e >> s));
    fe_mul(a, a, b, f);
    fe_store(out + 4 * i, a);
  }
}

// Scaling bases: g (Montgomery) or g^-1, g^(+-2^gs), and n^-1.
// out: [0] = step base for g_lo, [1] = step base for g_hi, [2] = n^-1, [3] = pre
// for g_hi (n^-1 for inverse transforms, 1 for forward ones).
template <class F>
__global__ void k_scale_bases(F f, const uint64_t* g_plain, int has_coset, int inverse,
                              int64_t n, int gs, uint64_t* out) {
  uint32_t g[8], t[8], ninv[8], one[8];
  fe_one(one, f);
  // n as a field element (n < 2^29 fits a limb; reduce for tiny moduli)
  uint32_t nv[8] = {(uint32_t)n, 0, 0, 0, 0, 0, 0, 0};
  fe_reduce_full(nv, f, 64);
  fe_to_mont(t, nv, f);
  fe_inv(ninv, t, f);
  fe_store(out + 8, ninv);
  if (has_coset) {
    fe_load(t, g_plain);
    fe_to_mont(g, t, f);
    if (inverse) fe_inv(g, g, f);
    fe_store(out, g);
    fe_pow64(t, g, 1ull << gs, f);
    fe_store(out + 4, t);
  } else {
    fe_store(out, one);
    fe_store(out + 4, one);
  }
  fe_store(out + 12, inverse ? ninv : one);
}

struct TableKey {
  uint64_t modulus[4];
  uint64_t omega[4];
  int log_N;
  int device;
  bool operator==(const TableKey& o) const {
    return std::memcmp(modulus, o.modulus, sizeof modulus) == 0 &&
           std::memcmp(omega, o.omega, sizeof omega) == 0 && log_N == o.log_N &&
           device == o.device;
  }
};

struct ScaleKey {
  TableKey root;
  uint64_t g[4];
  int has_coset, inverse;
  int64_t n;
  bool operator==(const ScaleKey& o) const {
    return root == o.root && std::memcmp(g, o.g, sizeof g) == 0 && has_coset == o.has_coset &&
           inverse == o.inverse && n == o.n;
  }
};

struct RootEntry {
  TableKey key;
  RootTables t;
  void* mem;
};
struct ScaleEntry {
  ScaleKey key;
  ScaleTables t;
  void* mem;
};

static std::mutex g_ntt_mutex;
static std::list<RootEntry> g_roots;    // most recently used first
static std::list<ScaleEntry> g_scales;  // most recently used first
static constexpr size_t kMaxRootEntries = 16;  // like the reference's lru_cache(16)
// At least the 64 transforms of one batch, whose tables must all stay alive
// until its launch (an entry used in the batch is never the least recent).
static constexpr size_t kMaxScaleEntries = 96;

// Expanded tables of single transforms (never of batches, whose tables must stay
// alive until their one launch): per (root, pass shape, direction) the boundary
// twiddles of a non-last pass laid out as its rows read them, and in a scale
// entry the n coset / inverse factors. Together they stay within the byte budget
// "ntt.full_table_mb"; a table that does not fit is not built and the pass falls
// back to the two-level tables (one more product per row).
struct FullEntry {
  TableKey key;
  int lr, ls, inverse;
  uint64_t* w;
  size_t bytes;
};
static std::list<FullEntry> g_fulls;  // most recently used first
static size_t g_full_bytes = 0;
static constexpr size_t kMaxFullEntries = 16;
static constexpr int kMinFullLog = 10;  // below, transforms are one pass with no boundary twiddle

template <class F>
static int build_roots(const F& f, const TableKey& key, RootTables& t, void** mem,
                       cudaStream_t s) {
  t.log_N = key.log_N;
  t.s = (key.log_N + 1) / 2;
  t.log_rmax = key.log_N < kMaxLogR ? key.log_N : kMaxLogR;
  const int64_t n_lo = 1ll << t.s, n_hi = 1ll << (key.log_N - t.s);
  const int64_t n_w = t.log_rmax > 0 ? (1ll << (t.log_rmax - 1)) : 1;
  const size_t elems = (size_t)(n_lo + n_hi + 2 * n_w + 4 + 1 /* omega */);
  uint64_t* base = nullptr;
  ZKB_TRY(check_cuda(cudaMalloc(&base, elems * 32), "NTT root table allocation"));
  *mem = base;
  t.t_lo = base;
  t.t_hi = t.t_lo + 4 * n_lo;
  t.w_fwd = t.t_hi + 4 * n_hi;
  t.w_inv = t.w_fwd + 4 * n_w;
  uint64_t* bases = t.w_inv + 4 * n_w;
  uint64_t* omega_dev = bases + 16;
  ZKB_TRY(check_cuda(cudaMemcpyAsync(omega_dev, key.omega, 32, cudaMemcpyHostToDevice, s),
                     "NTT root upload"));
  k_root_bases<<<1, 1, 0, s>>>(f, omega_dev, bases, key.log_N, t.s, t.log_rmax);
  ZKB_TRY(check_launch("NTT root bases"));
  k_pow_table<<<grid_for(n_lo, 128), 128, 0, s>>>(f, bases, nullptr, t.t_lo, n_lo);
  ZKB_TRY(check_launch("NTT root table (low powers)"));
  k_pow_table<<<grid_for(n_hi, 128), 128, 0, s>>>(f, bases + 4, nullptr, t.t_hi, n_hi);
  ZKB_TRY(check_launch("NTT root table (high powers)"));
  k_pow_table<<<grid_for(n_w, 128), 128, 0, s>>>(f, bases + 8, nullptr, t.w_fwd, n_w);
  ZKB_TRY(check_launch("NTT stage table"));
  k_pow_table<<<grid_for(n_w, 128), 128, 0, s>>>(f, bases + 12, nullptr, t.w_inv, n_w);
  ZKB_TRY(check_launch("NTT inverse stage table"));
  // Other streams may use the entry as soon as it is published.
  return check_cuda(cudaStreamSynchronize(s), "NTT root table build");
}

template <class F>
static int build_scale(const F& f, const ScaleKey& key, int log_n, ScaleTables& t, void** mem,
                       cudaStream_t s) {
  t.gs = (log_n + 1) / 2;
  const int64_t n_lo = 1ll << t.gs, n_hi = 1ll << (log_n - t.gs);
  const bool tables = key.has_coset != 0;
  const size_t elems = (size_t)((tables ? n_lo + n_hi : 0) + 4 + 1);
  uint64_t* base = nullptr;
  ZKB_TRY(check_cuda(cudaMalloc(&base, elems * 32), "NTT scale table allocation"));
  *mem = base;
  uint64_t* bases = base + (tables ? 4 * (n_lo + n_hi) : 0);
  uint64_t* g_dev = bases + 16;
  t.scale = bases + 8;
  ZKB_TRY(check_cuda(cudaMemcpyAsync(g_dev, key.g, 32, cudaMemcpyHostToDevice, s),
                     "NTT coset upload"));
  k_scale_bases<<<1, 1, 0, s>>>(f, g_dev, key.has_coset, key.inverse, key.n, t.gs, bases);
  ZKB_TRY(check_launch("NTT scale bases"));
  if (tables) {
    t.g_lo = base;
    t.g_hi = base + 4 * n_lo;
    k_pow_table<<<grid_for(n_lo, 128), 128, 0, s>>>(f, bases, nullptr, t.g_lo, n_lo);
    ZKB_TRY(check_launch("NTT coset table (low powers)"));
    k_pow_table<<<grid_for(n_hi, 128), 128, 0, s>>>(f, bases + 4, bases + 12, t.g_hi, n_hi);
    ZKB_TRY(check_launch("NTT coset table (high powers)"));
  }
  return check_cuda(cudaStreamSynchronize(s), "NTT scale table build");
}

// ---------------------------------------------------------------------------
// The pass kernel
// ---------------------------------------------------------------------------

struct NttPass {
  const uint64_t* in;
  uint64_t* out;
  int lr, ls, lc;       // log2 of: sub-transform size R, element stride S, columns per CTA C
  int last, first, inverse;
  int lR1, lR2;         // last pass: output index = (o >> lR2) + ((o & (R2-1)) << lR1) + k * (n / R)
  int log_n;
  // tables
  const uint64_t* t_lo;
  const uint64_t* t_hi;
  const uint64_t* w;    // stage table for this direction (w_Rmax^(+-j))
  int s, log_N, log_rmax;
  const uint64_t* g_lo; // coset tables (null without a coset)
  const uint64_t* g_hi;
  int gs;
  // optional expanded tables (null: use the two-level ones): t_full[(k << ls) + j] =
  // the boundary twiddle of row k, column j of a non-last pass; g_full[j] = the
  // coset / inverse scale of row j
  const uint64_t* t_full;
  const uint64_t* g_full;
  const uint64_t* scale;  // n^-1 for an inverse transform without coset tables
};

// Shared-memory address (in uint64 units) of element j of column c: columns
// are padded by 16 bytes so that consecutive columns start in different banks.
__device__ __forceinline__ int sm_index(int c, int j, int lr) {
  // XOR swizzle within each 128-byte row of four elements: the radix-4 rounds
  // with a small span (h = 1, 4, 16) touch rows 4h apart, which without it
  // would all fall into the same banks.
  return c * ((4 << lr) + 2) + 4 * (j ^ ((j >> 2) & 3));
}

// Products of the pass kernel: one shared out-of-line copy (kShared, the
// default: the expanded products of a radix-4 round and the store path
// overflow the instruction cache) or expanded in place.
template <bool kShared, class F>
__device__ __forceinline__ void ntt_mul(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                        const F& f) {
  if (kShared) {
    fe_mul_shared(r, a, b, f);
  } else {
    fe_mul(r, a, b, f);
  }
}

template <bool kShared, class F>
__device__ __forceinline__ void root_power(uint32_t r[8], const NttPass& a, uint64_t e, const F& f) {
  // w_N^e for 0 <= e < N
  const uint64_t mask = (1ull << a.s) - 1;
  uint32_t lo[8], hi[8];
  fe_load_nc(lo, a.t_lo + 4 * (e & mask));
  fe_load_nc(hi, a.t_hi + 4 * (e >> a.s));
  ntt_mul<kShared>(r, lo, hi, f);
}

// ---- lazy reduction inside a pass (moduli below 2^254) ----------------------
// Between the butterfly rounds of a pass, values may lie anywhere in [0, 2p)
// instead of [0, p): a difference becomes a - b + 2p, in (0, 4p), with no
// test, when a product by a canonical twiddle follows, and a product drops its
// last conditional subtraction. Both stay exact because 4p < 2^256: the sum of
// two values below 2p never carries out, and CIOS on a < 4p, b < p ends below
// (4p^2 + 2^256 p) / 2^256 < 2p. Values are canonical again before a pass stores
// them.

// 2p, word j (p < 2^254, so 2p fits eight words)
template <class F>
__device__ __forceinline__ uint32_t two_p(const F& f, int j) {
  return (f.p(j) << 1) | (j ? f.p(j - 1) >> 31 : 0u);
}

// r = a + b, then - 2p if that is at least 2p: [0, 2p) for a, b < 2p.
template <class F>
__device__ __forceinline__ void lz_add(uint32_t r[8], const uint32_t a[8], const uint32_t b[8], const F& f) {
  uint32_t s[8], d[8], bw;
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
  asm("sub.cc.u32 %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32 %8, 0, 0;"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(bw)
      : "r"(s[0]), "r"(s[1]), "r"(s[2]), "r"(s[3]), "r"(s[4]), "r"(s[5]), "r"(s[6]), "r"(s[7]),
        "r"(two_p(f, 0)), "r"(two_p(f, 1)), "r"(two_p(f, 2)), "r"(two_p(f, 3)), "r"(two_p(f, 4)),
        "r"(two_p(f, 5)), "r"(two_p(f, 6)), "r"(two_p(f, 7)));
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = bw ? s[j] : d[j];
}

// r = a - b + 2p in (0, 4p) for a, b < 2p: an operand of lz_mul only.
template <class F>
__device__ __forceinline__ void lz_sub_open(uint32_t r[8], const uint32_t a[8], const uint32_t b[8], const F& f) {
  uint32_t d[8];
  asm("sub.cc.u32 %0, %8, %16;\n\t"
      "subc.cc.u32 %1, %9, %17;\n\t"
      "subc.cc.u32 %2, %10, %18;\n\t"
      "subc.cc.u32 %3, %11, %19;\n\t"
      "subc.cc.u32 %4, %12, %20;\n\t"
      "subc.cc.u32 %5, %13, %21;\n\t"
      "subc.cc.u32 %6, %14, %22;\n\t"
      "subc.u32 %7, %15, %23;"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
        "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
  // modulo 2^256 the wrapped difference plus 2p is the exact a - b + 2p
  asm("add.cc.u32 %0, %0, %8;\n\t"
      "addc.cc.u32 %1, %1, %9;\n\t"
      "addc.cc.u32 %2, %2, %10;\n\t"
      "addc.cc.u32 %3, %3, %11;\n\t"
      "addc.cc.u32 %4, %4, %12;\n\t"
      "addc.cc.u32 %5, %5, %13;\n\t"
      "addc.cc.u32 %6, %6, %14;\n\t"
      "addc.u32 %7, %7, %15;"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]), "+r"(d[7])
      : "r"(two_p(f, 0)), "r"(two_p(f, 1)), "r"(two_p(f, 2)), "r"(two_p(f, 3)), "r"(two_p(f, 4)),
        "r"(two_p(f, 5)), "r"(two_p(f, 6)), "r"(two_p(f, 7)));
  fe_copy(r, d);
}

// r = a - b, + 2p on a borrow: [0, 2p) for a, b < 2p.
template <class F>
__device__ __forceinline__ void lz_sub(uint32_t r[8], const uint32_t a[8], const uint32_t b[8], const F& f) {
  uint32_t d[8], bw;
  asm("sub.cc.u32 %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32 %8, 0, 0;"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(bw)
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
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]), "+r"(d[7])
      : "r"(two_p(f, 0) & bw), "r"(two_p(f, 1) & bw), "r"(two_p(f, 2) & bw), "r"(two_p(f, 3) & bw),
        "r"(two_p(f, 4) & bw), "r"(two_p(f, 5) & bw), "r"(two_p(f, 6) & bw), "r"(two_p(f, 7) & bw));
  fe_copy(r, d);
}

// Fields whose modulus is known below 2^254 at compile time: BN254's Fr and Fq.
template <class F>
struct LazyOk {
  static constexpr bool value = false;
};
template <>
struct LazyOk<FrP> {
  static constexpr bool value = true;
};
template <>
struct LazyOk<FqP> {
  static constexpr bool value = true;
};

// One tile (CTA-sized piece) `bid` of pass a. kFresh: the pass reads rows
// that other CTAs wrote earlier in the same kernel (the batched form), so its
// row loads bypass L1.
template <class F, bool kFresh, bool kShared>
__device__ __forceinline__ void ntt_tile(const F& f, const NttPass& a, int64_t bid,
                                         uint64_t* sm) {
  const int lr = a.lr, lc = a.lc;
  const int R = 1 << lr, C = 1 << lc;
  const int total = C << lr;
  // lazy reduction between the rounds (inline products, BN254's fields): values in [0, 2p),
  // canonical again at the store
  constexpr bool kLz = !kShared && LazyOk<F>::value;
  auto mul_l = [&](uint32_t r[8], const uint32_t x[8], const uint32_t w[8]) {
    if (kLz) fe_mul_open(r, x, w, f); else ntt_mul<kShared>(r, x, w, f);
  };
  auto add_l = [&](uint32_t r[8], const uint32_t x[8], const uint32_t y[8]) {
    if (kLz) lz_add(r, x, y, f); else fe_add(r, x, y, f);
  };
  auto sub_l = [&](uint32_t r[8], const uint32_t x[8], const uint32_t y[8]) {
    if (kLz) lz_sub(r, x, y, f); else fe_sub(r, x, y, f);
  };
  // a difference that a product by a twiddle follows
  auto sub_mul_l = [&](uint32_t r[8], const uint32_t x[8], const uint32_t y[8]) {
    if (kLz) lz_sub_open(r, x, y, f); else fe_sub(r, x, y, f);
  };
  const int64_t S = 1ll << a.ls;
  const int64_t B = (int64_t)R << a.ls;

  // Column bases.
  //   non-last: o = bid / (S / C), first inner index j0 = (bid % (S / C)) * C,
  //             element (c, j) at position o B + j S + j0 + c.
  //   last:     k2 = bid % R2, k1_0 = (bid / R2) C; row o_c = (k1_0 + c) R2 + k2,
  //             element (c, j) at position o_c R + j.
  int64_t o = 0, j0 = 0, k2 = 0, k1_0 = 0;
  if (!a.last) {
    const int64_t groups = S >> lc;
    o = bid / groups;
    j0 = (bid % groups) << lc;
  } else {
    const int64_t R2 = 1ll << a.lR2;
    k2 = bid & (R2 - 1);
    k1_0 = (bid >> a.lR2) << lc;
  }

  // The stage table w_R^j (j < R/2) sits in shared memory after the columns.
  uint64_t* tw = sm + (size_t)C * ((4 << lr) + 2);
  for (int j = threadIdx.x; j < (R >> 1); j += blockDim.x) {
    uint32_t w[8];
    fe_load_nc(w, a.w + 4 * ((int64_t)j << (a.log_rmax - lr)));
    fe_store(tw + 4 * j, w);
  }

  // ---- load, with the coset pre-scale: shared position jr holds input row
  // brev(jr), so the bit reversal happens in the global gather and the
  // shared-memory stores stay consecutive (no bank conflicts) ----
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int c, jr;
    if (!a.last) {
      c = t & (C - 1);
      jr = t >> lc;
    } else {
      c = t >> lr;
      jr = t & (R - 1);
    }
    const int j = lr ? (int)(__brev((unsigned)jr) >> (32 - lr)) : 0;
    const int64_t pos = !a.last ? o * B + (int64_t)j * S + j0 + c
                                : (((k1_0 + c) << a.lR2) + k2) * R + j;
    uint32_t x[8];
    if (kFresh && !a.first) {
      fe_load_cg(x, a.in + 4 * pos);
    } else {
      fe_load_nc(x, a.in + 4 * pos);
    }
    if (a.first && a.g_lo && !a.inverse) {
      uint32_t lo[8];
      if (a.g_full) {
        fe_load_nc(lo, a.g_full + 4 * pos);
      } else {
        const uint64_t m = (1ull << a.gs) - 1;
        uint32_t hi[8];
        fe_load_nc(lo, a.g_lo + 4 * ((uint64_t)pos & m));
        fe_load_nc(hi, a.g_hi + 4 * ((uint64_t)pos >> a.gs));
        ntt_mul<kShared>(lo, lo, hi, f);
      }
      mul_l(x, x, lo);
    }
    fe_store(sm + sm_index(c, jr, lr), x);
  }
  __syncthreads();

  // ---- DIT stages in shared memory, two per round trip (radix 4) ----
  // A unit holds rows i0, i0 + h, i0 + 2h, i0 + 3h (h = 2^st, i0 = g 4h + jj):
  // stage st pairs (i0, i0 + h) and (i0 + 2h, i0 + 3h) with w_2h^jj; stage
  // st + 1 pairs (i0, i0 + 2h) with w_4h^jj and (i0 + h, i0 + 3h) with
  // w_4h^(jj + h). In the first round jj = 0, so only w_4 multiplies.
  int st = 0;
  for (; st + 1 < lr; st += 2) {
    const int h = 1 << st;
    const int units = total >> 2;
    for (int u = threadIdx.x; u < units; u += blockDim.x) {
      const int c = u >> (lr - 2);
      const int q = u & ((R >> 2) - 1);
      const int jj = q & (h - 1);
      const int i0 = ((q >> st) << (st + 2)) | jj;
      uint32_t x0[8], x1[8], x2[8], x3[8], w[8], t[8];
      fe_load(x0, sm + sm_index(c, i0, lr));
      fe_load(x1, sm + sm_index(c, i0 + h, lr));
      fe_load(x2, sm + sm_index(c, i0 + 2 * h, lr));
      fe_load(x3, sm + sm_index(c, i0 + 3 * h, lr));
      if (st > 0) {
        fe_load(w, tw + 4 * (jj << (lr - 1 - st)));  // w_2h^jj
        mul_l(x1, x1, w);
        mul_l(x3, x3, w);
      }
      add_l(t, x0, x1);
      sub_l(x1, x0, x1);
      fe_copy(x0, t);
      add_l(t, x2, x3);
      sub_mul_l(x3, x2, x3);  // multiplied below in every round
      fe_copy(x2, t);
      if (st > 0) {
        fe_load(w, tw + 4 * (jj << (lr - 2 - st)));  // w_4h^jj
        mul_l(x2, x2, w);
      }
      fe_load(w, tw + 4 * ((jj + h) << (lr - 2 - st)));  // w_4h^(jj + h)
      mul_l(x3, x3, w);
      add_l(t, x0, x2);
      sub_l(x2, x0, x2);
      fe_store(sm + sm_index(c, i0, lr), t);
      fe_store(sm + sm_index(c, i0 + 2 * h, lr), x2);
      add_l(t, x1, x3);
      sub_l(x3, x1, x3);
      fe_store(sm + sm_index(c, i0 + h, lr), t);
      fe_store(sm + sm_index(c, i0 + 3 * h, lr), x3);
    }
    __syncthreads();
  }
  if (st < lr) {  // an odd number of stages: one radix-2 stage left
    const int h = 1 << st;
    const int half_total = total >> 1;
    for (int b = threadIdx.x; b < half_total; b += blockDim.x) {
      const int c = b >> (lr - 1);
      const int k = b & ((R >> 1) - 1);
      const int jj = k & (h - 1);
      const int i0 = ((k >> st) << (st + 1)) | jj;
      uint32_t u[8], v[8], w[8], x[8];
      fe_load(u, sm + sm_index(c, i0, lr));
      fe_load(v, sm + sm_index(c, i0 + h, lr));
      if (st > 0) {
        fe_load(w, tw + 4 * (jj << (lr - 1 - st)));
        mul_l(v, v, w);
      }
      add_l(x, u, v);
      sub_l(v, u, v);
      fe_store(sm + sm_index(c, i0, lr), x);
      fe_store(sm + sm_index(c, i0 + h, lr), v);
    }
    __syncthreads();
  }

  // ---- store, with the pass twiddle or the final scaling ----
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int c = t & (C - 1);
    const int k = t >> lc;
    uint32_t x[8];
    fe_load(x, sm + sm_index(c, k, lr));
    if (!a.last) {
      // w_B^((j0 + c) k) = w_N^((j0 + c) k N / B); inverse uses w_N^-e = w_N^(N - e)
      const int64_t jp = j0 + c;
      uint64_t e = ((uint64_t)(jp * k)) << (a.log_N - (lr + a.ls));
      if (a.inverse && e) e = (1ull << a.log_N) - e;
      if (e) {
        uint32_t tw[8];
        if (a.t_full) {
          fe_load_nc(tw, a.t_full + 4 * (((int64_t)k << a.ls) + jp));
        } else {
          root_power<kShared>(tw, a, e, f);
        }
        ntt_mul<kShared>(x, x, tw, f);  // canonical for x < 2p as well
      } else if (kLz) {
        fe_reduce_once(x, f);
      }
      const int64_t pos = o * B + (int64_t)k * S + jp;
      fe_store(a.out + 4 * pos, x);
    } else {
      const int64_t oc = ((k1_0 + c) << a.lR2) + k2;
      const int64_t outidx = (oc >> a.lR2) + ((oc & ((1ll << a.lR2) - 1)) << a.lR1) +
                             ((int64_t)k << (a.log_n - lr));
      if (a.inverse) {
        uint32_t sc[8];
        if (a.g_full) {
          fe_load_nc(sc, a.g_full + 4 * outidx);
        } else if (a.g_lo) {
          const uint64_t m = (1ull << a.gs) - 1;
          uint32_t lo[8], hi[8];
          fe_load_nc(lo, a.g_lo + 4 * ((uint64_t)outidx & m));
          fe_load_nc(hi, a.g_hi + 4 * ((uint64_t)outidx >> a.gs));
          ntt_mul<kShared>(sc, lo, hi, f);
        } else {
          fe_load_nc(sc, a.scale);
        }
        ntt_mul<kShared>(x, x, sc, f);
      } else if (kLz) {
        fe_reduce_once(x, f);
      }
      fe_store(a.out + 4 * outidx, x);
    }
  }
}

template <class F, bool kShared>
__global__ void __launch_bounds__(kNttThreads, 1) k_ntt_pass(F f, NttPass a) {
  extern __shared__ uint4 smem_raw[];
  ntt_tile<F, false, kShared>(f, a, blockIdx.x, reinterpret_cast<uint64_t*>(smem_raw));
}

// ---------------------------------------------------------------------------
// The pass kernel fed by TMA (the default for transforms of two or more passes)
// ---------------------------------------------------------------------------
//
// Each CTA takes tiles blockIdx.x, blockIdx.x + gridDim.x, ...: by default one
// tile per CTA (a grid of all tiles), or one persistent wave ("ntt.tma_grid" =
// 0). One thread issues the tile's tensor loads (cp.async.bulk.tensor) into a
// shared-memory buffer and the copies complete on that buffer's mbarrier; in
// the persistent form two buffers let the loads of the CTA's next tile run
// while this tile computes.
// A tile is C columns of R rows in natural order, split into two planes of
// 16-byte half-elements (the low and the high 16 bytes of each 32-byte row),
// so that consecutive rows read by consecutive lanes fall into distinct banks.
// Two box loads per plane cover it (the low halves at word 0, the high halves
// at word 2 of each row: both innermost coordinates are multiples of 16 bytes).
//
// The butterflies run decimation in frequency (natural order in, bit-reversed
// order out): radix-4 rounds from the largest span down, after a radix-2 stage
// when log2 R is odd. The first round applies the coset pre-scale as it reads
// its rows. The store phase reads position p and writes it as frequency
// k = brev(p), with the pass twiddle or the final scaling, as ntt_tile does.
//
// Plane layouts, as the boxes land: a non-last pass holds element (c, j) at
// index j C + c (a box row is C neighbouring columns), the last pass at
// c R + j (a box row is R neighbouring rows of one column). Lanes walk the
// index that is contiguous, so each warp's accesses to a plane are
// consecutive 16-byte words wherever the butterfly span allows.

static constexpr uint32_t kTmaWaitLimit = 1u << 24;  // polls before a tile wait gives up
static constexpr int kTmaBoxRows = 256;              // a TMA box extent is at most 256

// Tiles whose TMA wait gave up (each such CTA stops early: its outputs are incomplete).
__device__ unsigned g_ntt_tma_timeouts = 0;

struct TmaPass {
  int64_t ntiles;
  int nbuf;       // 2: the next tile's loads overlap this tile's work; 1: one buffer
  int four_d;     // the tensor map has four dimensions (else three: a last pass of a two-pass plan)
};

template <class F>
__device__ __forceinline__ void plane_load(uint32_t x[8], const uint4* lo, const uint4* hi, int i) {
  const uint4 l = lo[i], h = hi[i];
  x[0] = l.x; x[1] = l.y; x[2] = l.z; x[3] = l.w;
  x[4] = h.x; x[5] = h.y; x[6] = h.z; x[7] = h.w;
}

__device__ __forceinline__ void plane_store(uint4* lo, uint4* hi, int i, const uint32_t x[8]) {
  lo[i] = make_uint4(x[0], x[1], x[2], x[3]);
  hi[i] = make_uint4(x[4], x[5], x[6], x[7]);
}

template <class F, int kThreads = kNttThreads, int kMinBlocks = 1, bool kLazy = false>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_ntt_pass_tma(F f, const NttPass a, const TmaPass tp,
                                                                      const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(1024) unsigned char smem_raw_tma[];
  // the buffers start on a 1 KiB boundary (the launch asks for 1 KiB more)
  unsigned char* smem_tma = smem_raw_tma + ((1024u - (smem_u32(smem_raw_tma) & 1023u)) & 1023u);
  const int lr = a.lr, lc = a.lc;
  const int R = 1 << lr, C = 1 << lc, T = C << lr;
  const int64_t S = 1ll << a.ls;
  const int64_t B = (int64_t)R << a.ls;
  const int nbuf = tp.nbuf;
  const size_t plane = (size_t)T * 16;
  unsigned char* bufs = smem_tma;
  uint64_t* tw = reinterpret_cast<uint64_t*>(smem_tma + (size_t)nbuf * 2 * plane);
  uint64_t* bars = tw + 4 * (R >> 1);
  const int tid = threadIdx.x;
  // butterfly arithmetic: canonical, or lazy (values in [0, 2p) between rounds)
  auto bf_add = [&](uint32_t r[8], const uint32_t x[8], const uint32_t y[8]) {
    if (kLazy) lz_add(r, x, y, f); else fe_add(r, x, y, f);
  };
  // a difference that a product by a twiddle follows (open: any value below 4p)
  auto bf_sub_mul = [&](uint32_t r[8], const uint32_t x[8], const uint32_t y[8]) {
    if (kLazy) lz_sub_open(r, x, y, f); else fe_sub(r, x, y, f);
  };
  auto bf_sub = [&](uint32_t r[8], const uint32_t x[8], const uint32_t y[8]) {
    if (kLazy) lz_sub(r, x, y, f); else fe_sub(r, x, y, f);
  };
  auto bf_mul = [&](uint32_t r[8], const uint32_t x[8], const uint32_t w[8]) {
    if (kLazy) fe_mul_open(r, x, w, f); else fe_mul(r, x, w, f);
  };

  for (int j = tid; j < (R >> 1); j += blockDim.x) {
    uint32_t w[8];
    fe_load_nc(w, a.w + 4 * ((int64_t)j << (a.log_rmax - lr)));
    fe_store(tw + 4 * j, w);
  }
  if (tid == 0) {
    for (int b = 0; b < nbuf; ++b) mbar_init(&bars[b], 1);
    fence_mbar_init();
  }
  __syncthreads();

  const int rows_box = R < kTmaBoxRows ? R : kTmaBoxRows;
  const int64_t groups = S >> lc;  // non-last pass: tiles per block of B rows
  // thread 0: announce the tile's bytes and issue its box loads into buffer b
  auto issue = [&](int64_t tile, int b) {
    unsigned char* lo = bufs + (size_t)b * 2 * plane;
    unsigned char* hi = lo + plane;
    mbar_arrive_expect_tx(&bars[b], (uint32_t)T * 32u);
    if (!a.last) {
      const int o = (int)(tile / groups);
      const int j0 = (int)((tile % groups) << lc);
      for (int r0 = 0; r0 < R; r0 += rows_box) {
        const size_t off = (size_t)r0 * C * 16;
        tma_load_4d(lo + off, &tmap, &bars[b], 0, j0, r0, o);
        tma_load_4d(hi + off, &tmap, &bars[b], 2, j0, r0, o);
      }
    } else {
      // a box holds all C columns when a column fits one box (R <= 256), else one
      // column's run of rows_box rows; either way column c lands at c R
      const int k2 = (int)(tile & ((1ll << a.lR2) - 1));
      const int k1_0 = (int)((tile >> a.lR2) << lc);
      const int box_cols = R <= kTmaBoxRows ? C : 1;
      for (int c0 = 0; c0 < C; c0 += box_cols) {
        for (int r0 = 0; r0 < R; r0 += rows_box) {
          const size_t off = ((size_t)c0 * R + r0) * 16;
          if (tp.four_d) {
            tma_load_4d(lo + off, &tmap, &bars[b], 0, r0, k2, k1_0 + c0);
            tma_load_4d(hi + off, &tmap, &bars[b], 2, r0, k2, k1_0 + c0);
          } else {
            tma_load_3d(lo + off, &tmap, &bars[b], 0, r0, k1_0 + c0);
            tma_load_3d(hi + off, &tmap, &bars[b], 2, r0, k1_0 + c0);
          }
        }
      }
    }
  };
  // plane index of element (c, j)
  auto pidx = [&](int c, int j) { return a.last ? (c << lr) + j : (j << lc) + c; };

  int64_t tile = blockIdx.x;
  if (tid == 0 && tile < tp.ntiles) issue(tile, 0);
  bool failed = false;
  int64_t i = 0;
  for (; tile < tp.ntiles; ++i, tile += gridDim.x) {
    const int b = nbuf == 2 ? (int)(i & 1) : 0;
    const uint32_t parity = nbuf == 2 ? (uint32_t)((i >> 1) & 1) : (uint32_t)(i & 1);
    if (nbuf == 2 && tid == 0 && tile + gridDim.x < tp.ntiles) issue(tile + gridDim.x, b ^ 1);
    const bool got = mbar_wait_bounded(&bars[b], parity, kTmaWaitLimit);
    if (__syncthreads_or(!got)) {
      failed = true;
      break;
    }
    uint4* lo = reinterpret_cast<uint4*>(bufs + (size_t)b * 2 * plane);
    uint4* hi = reinterpret_cast<uint4*>(bufs + (size_t)b * 2 * plane + plane);

    // tile origin in the pass's index space
    int64_t o = 0, j0 = 0, k2 = 0, k1_0 = 0;
    if (!a.last) {
      o = tile / groups;
      j0 = (tile % groups) << lc;
    } else {
      k2 = tile & ((1ll << a.lR2) - 1);
      k1_0 = (tile >> a.lR2) << lc;
    }
    const bool prescale = a.first && a.g_lo && !a.inverse;
    // the coset factor g^pos of element (c, j): only the first pass, which is never the last
    auto scale_in = [&](uint32_t x[8], int c, int j) {
      const int64_t pos = o * B + (int64_t)j * S + j0 + c;
      uint32_t g[8];
      if (a.g_full) {
        fe_load_nc(g, a.g_full + 4 * pos);
      } else {
        const uint64_t m = (1ull << a.gs) - 1;
        uint32_t hi2[8];
        fe_load_nc(g, a.g_lo + 4 * ((uint64_t)pos & m));
        fe_load_nc(hi2, a.g_hi + 4 * ((uint64_t)pos >> a.gs));
        fe_mul(g, g, hi2, f);
      }
      bf_mul(x, x, g);
    };

    // ---- decimation in frequency ----
    bool first_round = true;
    int st = lr - 1;
    if (lr & 1) {  // radix-2 stage of half-span R / 2
      const int h = 1 << st;
      for (int u = tid; u < (T >> 1); u += blockDim.x) {
        int c, q;
        if (!a.last) {
          c = u & (C - 1);
          q = u >> lc;
        } else {
          q = u & (h - 1);
          c = u >> (lr - 1);
        }
        uint32_t x0[8], x1[8], t[8];
        const int i0 = pidx(c, q), i1 = pidx(c, q + h);
        plane_load<F>(x0, lo, hi, i0);
        plane_load<F>(x1, lo, hi, i1);
        if (prescale) {
          scale_in(x0, c, q);
          scale_in(x1, c, q + h);
        }
        bf_add(t, x0, x1);
        if (st > 0) {
          uint32_t w[8];
          bf_sub_mul(x1, x0, x1);
          fe_load(w, tw + 4 * q);  // w_R^q
          bf_mul(x1, x1, w);
        } else {
          bf_sub(x1, x0, x1);
        }
        plane_store(lo, hi, i0, t);
        plane_store(lo, hi, i1, x1);
      }
      first_round = false;
      __syncthreads();
      st -= 1;
    }
    // radix-4 rounds: st is the lower stage of the pair (half-spans 2h and h)
    for (st -= 1; st >= 0; st -= 2) {
      const int h = 1 << st;
      const int R4 = R >> 2;
      for (int u = tid; u < (T >> 2); u += blockDim.x) {
        int c, q;
        if (!a.last) {
          c = u & (C - 1);
          q = u >> lc;
        } else {
          q = u & (R4 - 1);
          c = u >> (lr - 2);
        }
        const int jj = q & (h - 1);
        const int i0 = ((q >> st) << (st + 2)) | jj;
        uint32_t x0[8], x1[8], x2[8], x3[8], t[8], w[8];
        plane_load<F>(x0, lo, hi, pidx(c, i0));
        plane_load<F>(x1, lo, hi, pidx(c, i0 + h));
        plane_load<F>(x2, lo, hi, pidx(c, i0 + 2 * h));
        plane_load<F>(x3, lo, hi, pidx(c, i0 + 3 * h));
        if (prescale && first_round) {
          scale_in(x0, c, i0);
          scale_in(x1, c, i0 + h);
          scale_in(x2, c, i0 + 2 * h);
          scale_in(x3, c, i0 + 3 * h);
        }
        // half-span 2h: (x0, x2) with w_4h^jj, (x1, x3) with w_4h^(jj + h)
        bf_add(t, x0, x2);
        if (st > 0) bf_sub_mul(x2, x0, x2); else bf_sub(x2, x0, x2);
        fe_copy(x0, t);
        bf_add(t, x1, x3);
        bf_sub_mul(x3, x1, x3);
        fe_copy(x1, t);
        if (st > 0) {
          fe_load(w, tw + 4 * (jj << (lr - 2 - st)));
          bf_mul(x2, x2, w);
        }
        fe_load(w, tw + 4 * ((jj + h) << (lr - 2 - st)));
        bf_mul(x3, x3, w);
        // half-span h: (x0, x1) and (x2, x3) with w_2h^jj
        bf_add(t, x0, x1);
        if (st > 0) bf_sub_mul(x1, x0, x1); else bf_sub(x1, x0, x1);
        fe_copy(x0, t);
        bf_add(t, x2, x3);
        if (st > 0) bf_sub_mul(x3, x2, x3); else bf_sub(x3, x2, x3);
        fe_copy(x2, t);
        if (st > 0) {
          fe_load(w, tw + 4 * (jj << (lr - 1 - st)));
          bf_mul(x1, x1, w);
          bf_mul(x3, x3, w);
        }
        plane_store(lo, hi, pidx(c, i0), x0);
        plane_store(lo, hi, pidx(c, i0 + h), x1);
        plane_store(lo, hi, pidx(c, i0 + 2 * h), x2);
        plane_store(lo, hi, pidx(c, i0 + 3 * h), x3);
      }
      first_round = false;
      __syncthreads();
    }

    // ---- store: position p holds frequency k = brev(p) ----
    for (int t = tid; t < T; t += blockDim.x) {
      int c, p;
      if (!a.last) {
        c = t & (C - 1);
        p = t >> lc;
      } else {
        p = t & (R - 1);
        c = t >> lr;
      }
      const int k = lr ? (int)(__brev((unsigned)p) >> (32 - lr)) : 0;
      uint32_t x[8];
      plane_load<F>(x, lo, hi, pidx(c, p));
      if (!a.last) {
        const int64_t jp = j0 + c;
        uint64_t e = ((uint64_t)(jp * k)) << (a.log_N - (lr + a.ls));
        if (a.inverse && e) e = (1ull << a.log_N) - e;
        if (e) {
          uint32_t w[8];
          if (a.t_full) {
            fe_load_nc(w, a.t_full + 4 * (((int64_t)k << a.ls) + jp));
          } else {
            root_power<false>(w, a, e, f);
          }
          fe_mul(x, x, w, f);  // canonical for x < 2p as well
        } else if (kLazy) {
          fe_reduce_once(x, f);
        }
        fe_store(a.out + 4 * (o * B + (int64_t)k * S + jp), x);
      } else {
        const int64_t oc = ((k1_0 + c) << a.lR2) + k2;
        const int64_t outidx = (oc >> a.lR2) + ((oc & ((1ll << a.lR2) - 1)) << a.lR1) +
                               ((int64_t)k << (a.log_n - lr));
        if (a.inverse) {
          uint32_t sc[8];
          if (a.g_full) {
            fe_load_nc(sc, a.g_full + 4 * outidx);
          } else if (a.g_lo) {
            const uint64_t m = (1ull << a.gs) - 1;
            uint32_t l2[8], h2[8];
            fe_load_nc(l2, a.g_lo + 4 * ((uint64_t)outidx & m));
            fe_load_nc(h2, a.g_hi + 4 * ((uint64_t)outidx >> a.gs));
            fe_mul(sc, l2, h2, f);
          } else {
            fe_load_nc(sc, a.scale);
          }
          fe_mul(x, x, sc, f);
        } else if (kLazy) {
          fe_reduce_once(x, f);
        }
        fe_store(a.out + 4 * outidx, x);
      }
    }
    // every thread is done with this buffer (generic accesses) before the next
    // TMA write into it
    fence_proxy_async_smem();
    __syncthreads();
    if (nbuf == 1 && tid == 0 && tile + gridDim.x < tp.ntiles) issue(tile + gridDim.x, 0);
  }
  if (failed) {
    // a wait gave up: record it, and let the copies still in flight land (bounded)
    // before the CTA's shared memory goes away
    if (tid == 0) {
      atomicAdd(&g_ntt_tma_timeouts, 1u);
      const int b = nbuf == 2 ? (int)(i & 1) : 0;
      mbar_wait_bounded(&bars[b], nbuf == 2 ? (uint32_t)((i >> 1) & 1) : (uint32_t)(i & 1), kTmaWaitLimit);
      if (nbuf == 2 && tile + gridDim.x < tp.ntiles) {
        mbar_wait_bounded(&bars[b ^ 1], (uint32_t)(((i + 1) >> 1) & 1), kTmaWaitLimit);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Batched form: one persistent launch for many transforms
// ---------------------------------------------------------------------------
//
// Every pass of every transform in the batch is a list of tiles; the tiles
// are numbered pass by pass, all first passes before all second passes (and
// those before all third passes). CTAs take tile numbers from a device
// counter in that order. A tile of pass q > 0 may start only when every tile
// of pass q - 1 of its transform has finished: thread 0 waits on that pass's
// completion counter. The tiles it waits for carry smaller numbers, so they
// were taken earlier by CTAs that are already running and that wait, if at
// all, only on still smaller numbers: the waits always end. Each wait is
// still bounded (about a second); a CTA that gives up sets the status word
// to ZKB_ETIMEOUT and stops taking tiles.

static constexpr int kMaxBatchPasses = 192;  // 64 transforms x 3 passes
static constexpr int kBatchThreads = 256;
// Default bound of a dependency wait ("ntt.batch_spin_limit"): 2^22 polls,
// each after a >= 256 ns sleep, about a second.
static constexpr unsigned kBatchSpinLimit = 1u << 22;

struct NttBatchTable {
  int num_passes;
  int64_t tile_start[kMaxBatchPasses + 1];  // first tile number of each pass
  int dep[kMaxBatchPasses];                 // pass that must finish first, or -1
  NttPass pass[kMaxBatchPasses];
};

template <class F, bool kShared>
__global__ void __launch_bounds__(kBatchThreads) k_ntt_batch(F f, const __grid_constant__ NttBatchTable T,
                                                             unsigned long long* next_tile,
                                                             unsigned* done, int* status,
                                                             unsigned spin_limit) {
  extern __shared__ uint4 smem_raw[];
  uint64_t* sm = reinterpret_cast<uint64_t*>(smem_raw);
  __shared__ long long s_tile;
  __shared__ int s_pass, s_go;
  const long long total = T.tile_start[T.num_passes];
  for (;;) {
    if (threadIdx.x == 0) {
      const long long tile = (long long)atomicAdd(next_tile, 1ull);
      int p = 0, go = tile < total && *(volatile int*)status == 0;
      if (go) {
        int lo = 0, hi = T.num_passes - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (T.tile_start[mid] <= tile) lo = mid; else hi = mid - 1;
        }
        p = lo;
        const int d = T.dep[p];
        if (d >= 0) {
          const unsigned need = (unsigned)(T.tile_start[d + 1] - T.tile_start[d]);
          unsigned spins = 0;
          while (*(volatile unsigned*)(done + d) < need) {
            if (++spins > spin_limit) {
              atomicExch(status, ZKB_ETIMEOUT);
              go = 0;
              break;
            }
            __nanosleep(256);
          }
          __threadfence();
        }
      }
      s_tile = tile;
      s_pass = p;
      s_go = go;
    }
    __syncthreads();
    if (!s_go) break;
    const int p = s_pass;
    ntt_tile<F, true, kShared>(f, T.pass[p], s_tile - T.tile_start[p], sm);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(done + p, 1u);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

static int ilog2(int64_t n) {
  int l = 0;
  while ((1ll << l) < n) ++l;
  return l;
}

// Splits log_n into P parts of at most "ntt.max_log_radix" bits (at most 12,
// the shared-memory limit), the larger parts first. At most three passes:
// the last pass's output mapping covers P <= 3, which 12-bit passes reach up
// to 2^36. From 2^10 rows on, a transform that fits one pass is still split
// in two: one pass would be a single CTA on one SM, while two passes of
// 2^5..2^6-point sub-transforms spread it over 32-64 CTAs (2^12 rows: 0.048
// ms instead of 0.11 ms on a B200).
// A per-size table entry (an autotuner's) takes precedence over the knob.
// The radices (log2 sub-transform sizes) of the passes of a 2^log_n-row NTT.
// The largest sub-transform per pass comes from a per-size table entry, else the
// "ntt.max_log_radix" knob, else the size. A single transform takes three passes
// from 2^19 rows (256-row sub-transforms at 2^24), else up to 4096 rows a pass:
// measured on B200 with 512-row tiles of 128 threads, 2^24 rows 4.96 ms in three
// passes against 5.74 in two 4096-row passes, 2^23 2.41 against 2.94, 2^20 0.300
// against 0.306; two passes stay best to 2^18 (0.0929 against 0.0946). A batch
// (`batch`) keeps up to 4096 rows a pass: its persistent kernel starts a pass's
// tiles only after the transform's previous pass, and the served jobs' small
// batches measured far slower with the third pass.
static std::vector<int> plan_radices(int log_n, bool batch = false) {
  const int tuned = tune_get_sized("ntt.max_log_radix", log_n);
  int max_r = tuned > 0 ? tuned : tune_get("ntt.max_log_radix");
  if (max_r < 8) max_r = log_n >= 19 && !batch ? (log_n + 2) / 3 : kMaxLogR;
  int P = (log_n + max_r - 1) / max_r;
  if (P > 3) P = 3;
  if (P < (log_n + kMaxLogR - 1) / kMaxLogR) P = (log_n + kMaxLogR - 1) / kMaxLogR;
  if (P < 2 && log_n >= 10) P = 2;
  if (P < 1) P = 1;
  std::vector<int> r(P, log_n / P);
  for (int q = 0; q < log_n % P; ++q) r[q] += 1;
  return r;
}

size_t workspace_bytes(int64_t n) {
  int log_n = 0;
  while ((1ll << log_n) < n) ++log_n;
  if (n <= 1 || plan_radices(log_n).size() == 1) return 0;
  return (size_t)n * 32;
}

// Cached tables for a transform of n = 2^log_n rows: the root tables of `key`
// and, for an inverse or coset transform, its scaling tables.
template <class F>
static int lookup_tables(const F& f, const TableKey& key, int64_t n, int log_n, int invert,
                         const uint64_t* coset, RootTables& rt, ScaleTables& st, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_ntt_mutex);
  auto it = g_roots.begin();
  for (; it != g_roots.end(); ++it)
    if (it->key == key) break;
  if (it == g_roots.end()) {
    RootEntry e;
    e.key = key;
    e.mem = nullptr;
    int rc = build_roots(f, key, e.t, &e.mem, s);
    if (rc != ZKB_OK) {
      if (e.mem) cudaFree(e.mem);
      return rc;
    }
    g_roots.push_front(e);
    if (g_roots.size() > kMaxRootEntries) {
      // kernels queued on any stream may still read the evicted tables
      cudaDeviceSynchronize();
      cudaFree(g_roots.back().mem);
      g_roots.pop_back();
    }
  } else {
    g_roots.splice(g_roots.begin(), g_roots, it);
  }
  rt = g_roots.front().t;
  st = ScaleTables();
  if (!invert && !coset) return ZKB_OK;
  ScaleKey sk;
  sk.root = key;
  std::memset(sk.g, 0, sizeof sk.g);
  if (coset) std::memcpy(sk.g, coset, sizeof sk.g);
  sk.has_coset = coset != nullptr;
  sk.inverse = invert;
  sk.n = n;
  auto jt = g_scales.begin();
  for (; jt != g_scales.end(); ++jt)
    if (jt->key == sk) break;
  if (jt == g_scales.end()) {
    ScaleEntry e;
    e.key = sk;
    e.mem = nullptr;
    int rc = build_scale(f, sk, log_n, e.t, &e.mem, s);
    if (rc != ZKB_OK) {
      if (e.mem) cudaFree(e.mem);
      return rc;
    }
    g_scales.push_front(e);
    if (g_scales.size() > kMaxScaleEntries) {
      cudaDeviceSynchronize();
      cudaFree(g_scales.back().mem);
      if (g_scales.back().t.g_full) {
        cudaFree(g_scales.back().t.g_full);
        g_full_bytes -= g_scales.back().t.full_bytes;
      }
      g_scales.pop_back();
    }
  } else {
    g_scales.splice(g_scales.begin(), g_scales, jt);
  }
  st = g_scales.front().t;
  return ZKB_OK;
}

// The boundary twiddles of a non-last pass of 2^lr rows at stride 2^ls, as its
// store reads them: out[(k << ls) + j] = w_B^(j k) (w_B^-(j k) inverse) for
// k < 2^lr, j < 2^ls, B = 2^(lr + ls), from the two-level root tables, so that
// neighbouring columns of a row read neighbouring entries.
template <class F>
__global__ void k_expand_twiddles(F f, const uint64_t* lo, const uint64_t* hi, int s, int log_N, int lr,
                                  int ls, int inverse, uint64_t* out) {
  const uint64_t mask = (1ull << s) - 1;
  const int64_t count = 1ll << (lr + ls);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    const uint64_t k = (uint64_t)i >> ls, j = (uint64_t)i & ((1ull << ls) - 1);
    uint64_t e = (j * k) << (log_N - (lr + ls));
    if (inverse && e) e = (1ull << log_N) - e;
    uint32_t a[8], b[8];
    fe_load_nc(a, lo + 4 * (e & mask));
    fe_load_nc(b, hi + 4 * (e >> s));
    fe_mul(a, a, b, f);
    fe_store(out + 4 * i, a);
  }
}

// The expanded boundary twiddles of a non-last pass (null when they do not fit
// the byte budget, or the budget is 0).
template <class F>
static int lookup_twiddles(const F& f, const TableKey& key, const RootTables& rt, int lr, int ls, int inverse,
                           const uint64_t** t_full, cudaStream_t s) {
  *t_full = nullptr;
  const size_t budget = (size_t)tune_get("ntt.full_table_mb") << 20;
  if (lr + ls < kMinFullLog || budget == 0) return ZKB_OK;
  const size_t bytes = (size_t)32 << (lr + ls);
  std::lock_guard<std::mutex> lock(g_ntt_mutex);
  auto it = g_fulls.begin();
  for (; it != g_fulls.end(); ++it)
    if (it->key == key && it->lr == lr && it->ls == ls && it->inverse == inverse) break;
  if (it != g_fulls.end()) {
    g_fulls.splice(g_fulls.begin(), g_fulls, it);
    *t_full = g_fulls.front().w;
  } else {
    // room among the expanded root tables, least recently used first
    while (g_full_bytes + bytes > budget && !g_fulls.empty()) {
      cudaDeviceSynchronize();  // kernels queued on any stream may still read it
      cudaFree(g_fulls.back().w);
      g_full_bytes -= g_fulls.back().bytes;
      g_fulls.pop_back();
    }
    if (g_full_bytes + bytes <= budget) {
      FullEntry e{key, lr, ls, inverse, nullptr, bytes};
      ZKB_TRY(check_cuda(cudaMalloc(&e.w, bytes), "NTT expanded twiddle table allocation"));
      k_expand_twiddles<<<grid_for(1ll << (lr + ls), 128), 128, 0, s>>>(f, rt.t_lo, rt.t_hi, rt.s, rt.log_N,
                                                                        lr, ls, inverse, e.w);
      int rc = check_launch("NTT expanded twiddle table");
      if (rc == ZKB_OK) rc = check_cuda(cudaStreamSynchronize(s), "NTT expanded twiddle table build");
      if (rc != ZKB_OK) {
        cudaFree(e.w);
        return rc;
      }
      g_fulls.push_front(e);
      g_full_bytes += bytes;
      if (g_fulls.size() > kMaxFullEntries) {
        cudaDeviceSynchronize();
        cudaFree(g_fulls.back().w);
        g_full_bytes -= g_fulls.back().bytes;
        g_fulls.pop_back();
      }
      *t_full = e.w;
    }
  }
  return ZKB_OK;
}

// The coset / inverse scale factors of a transform of n = 2^log_n rows, expanded
// inside its scale entry (st->g_full; null when it does not fit the byte budget).
template <class F>
static int lookup_scale_full(const F& f, int64_t n, int log_n, ScaleTables* st, cudaStream_t s) {
  const size_t budget = (size_t)tune_get("ntt.full_table_mb") << 20;
  if (log_n < kMinFullLog || budget == 0) {
    st->g_full = nullptr;  // a budget of 0 means the two-level tables, cached expansions or not
    return ZKB_OK;
  }
  const size_t bytes = (size_t)n * 32;
  std::lock_guard<std::mutex> lock(g_ntt_mutex);
  if (st->g_lo && !st->g_full && g_full_bytes + bytes <= budget) {
    for (ScaleEntry& e : g_scales) {
      if (e.t.g_lo != st->g_lo) continue;
      if (!e.t.g_full) {
        uint64_t* g = nullptr;
        ZKB_TRY(check_cuda(cudaMalloc(&g, bytes), "NTT expanded scale table allocation"));
        k_expand_table<<<grid_for(n, 128), 128, 0, s>>>(f, e.t.g_lo, e.t.g_hi, e.t.gs, 0, g, n);
        int rc = check_launch("NTT expanded scale table");
        if (rc == ZKB_OK) rc = check_cuda(cudaStreamSynchronize(s), "NTT expanded scale table build");
        if (rc != ZKB_OK) {
          cudaFree(g);
          return rc;
        }
        e.t.g_full = g;
        e.t.full_bytes = bytes;
        g_full_bytes += bytes;
      }
      st->g_full = e.t.g_full;
      break;
    }
  }
  return ZKB_OK;
}

static TableKey table_key(const zkb_field* field, const uint64_t* omega, int log_n, int device) {
  TableKey key;
  std::memcpy(key.modulus, field->modulus, sizeof key.modulus);
  if (omega) {
    std::memcpy(key.omega, omega, sizeof key.omega);
    key.log_N = log_n;
  } else {
    std::memcpy(key.omega, kFrRoot28, sizeof key.omega);
    key.log_N = kMaxLogN;
  }
  key.device = device;
  return key;
}

// One launch of the pass kernel: its parameters and shape.
struct PassLaunch {
  NttPass a;
  int64_t ctas;
  int threads;
  size_t smem;
};

// The passes of one transform. cta_log / threads: the tile and block size,
// or 0 for the size-based choice (and the "ntt.cta_log_elems" / "ntt.threads"
// knobs, which override it). batch: the transform is part of a batch launch
// (the pass split of plan_radices for batches).
static void plan_passes(int64_t n, int log_n, int invert, const RootTables& rt,
                        const ScaleTables& st, const uint64_t* in, uint64_t* out, uint64_t* tmp,
                        int cta_log, int threads, bool batch, std::vector<PassLaunch>& passes) {
  const std::vector<int> radices = plan_radices(log_n, batch);
  const int P = (int)radices.size();
  // columns per CTA: the tile C R is at most 2^cta_log elements, and at least
  // one sub-transform. Auto: 512-row tiles (one column once a pass's
  // sub-transform has 512 rows), with 128 threads up to 512-row tiles, 256 up
  // to 2048 and 512 for 4096. Small tiles put several CTAs on each SM, so one
  // CTA's loads and barriers overlap another's products; measured on B200
  // against 1024-row tiles of 256 threads (and 4096-row tiles of 512 threads
  // from 2^24): 18-27 % faster from 2^11 to 2^16 rows, within 2 % at 2^17-2^18.
  // A per-size table entry takes precedence over the knob, which takes
  // precedence over the rule.
  if (cta_log == 0) {
    cta_log = tune_get_sized("ntt.cta_log_elems", log_n);
    if (cta_log < 9) cta_log = tune_get("ntt.cta_log_elems");
    if (cta_log < 9) cta_log = 9;
  }
  if (threads == 0) {
    threads = tune_get_sized("ntt.threads", log_n);
    if (threads < 64) threads = tune_get("ntt.threads");
    if (threads < 64) threads = 0;  // by each pass's tile, below
  }
  passes.clear();
  int ls = log_n;  // stride exponent of the current pass: S_q = 2^(log_n - sum of radices so far)
  for (int q = 0; q < P; ++q) {
    NttPass a;
    std::memset(&a, 0, sizeof a);
    a.lr = radices[q];
    ls -= a.lr;
    a.ls = ls;
    a.last = q == P - 1;
    a.first = q == 0;
    a.inverse = invert;
    a.log_n = log_n;
    a.in = q == 0 ? in : tmp;
    a.out = a.last ? out : tmp;
    a.t_lo = rt.t_lo;
    a.t_hi = rt.t_hi;
    a.w = invert ? rt.w_inv : rt.w_fwd;
    a.s = rt.s;
    a.log_N = rt.log_N;
    a.log_rmax = rt.log_rmax;
    a.g_lo = st.g_lo;
    a.g_hi = st.g_hi;
    a.gs = st.gs;
    a.scale = st.scale;
    a.g_full = st.g_full;
    int lc = cta_log > a.lr ? cta_log - a.lr : 0;
    if (!a.last) {
      if (lc > a.ls) lc = a.ls;
    } else {
      // R1 = first radix, R2 = the middle radix (P <= 3)
      a.lR1 = P >= 2 ? radices[0] : 0;
      a.lR2 = P >= 3 ? radices[1] : 0;
      if (lc > a.lR1) lc = a.lR1;
    }
    a.lc = lc;
    PassLaunch L;
    L.a = a;
    L.ctas = n >> (a.lr + lc);
    // padded columns, then the stage table (R / 2 rows)
    L.smem = (size_t)(1 << lc) * ((32u << a.lr) + 16) + ((size_t)16 << a.lr);
    const int half_total = (1 << (a.lr + lc)) >> 1;
    const int tile_log = a.lr + lc;
    L.threads = threads ? threads : tile_log >= kMaxLogR ? 512 : tile_log >= 10 ? 256 : 128;
    if (half_total < L.threads) L.threads = half_total < 32 ? 32 : half_total;
    passes.push_back(L);
  }
}

static int sm_count(int device, int* sms) {
  return check_cuda(cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, device),
                    "SM count");
}

// One pass through k_ntt_pass_tma: its tensor map over the pass's input, the
// shared-memory plan (two tile buffers when four planes fit in about 110 KiB,
// else one) and a one-wave persistent grid.
template <class F>
static int launch_pass_tma(const F& f, const PassLaunch& L, int64_t n, int P, int sms, cudaStream_t s, int q) {
  const NttPass& a = L.a;
  const int R = 1 << a.lr, C = 1 << a.lc;
  const int64_t T = (int64_t)C << a.lr;
  const uint32_t rows_box = (uint32_t)std::min(R, kTmaBoxRows);
  CUtensorMap map;
  TmaPass tp;
  tp.ntiles = n / T;
  if (!a.last) {
    const uint64_t S = 1ull << a.ls, B = (uint64_t)R << a.ls;
    const uint64_t dims[4] = {4, S, (uint64_t)R, (uint64_t)n / B};
    const uint64_t strides[3] = {32, S * 32, B * 32};
    const uint32_t box[4] = {2, (uint32_t)C, rows_box, 1};
    ZKB_TRY(encode_tensor_map_u64(&map, a.in, 4, dims, strides, box));
    tp.four_d = 1;
  } else if (a.lR2 > 0) {
    const uint64_t R1 = 1ull << a.lR1, R2 = 1ull << a.lR2;
    const uint32_t box_cols = R <= kTmaBoxRows ? (uint32_t)C : 1u;  // as the kernel's issue loop
    const uint64_t dims[4] = {4, (uint64_t)R, R2, R1};
    const uint64_t strides[3] = {32, (uint64_t)R * 32, R2 * R * 32};
    const uint32_t box[4] = {2, rows_box, 1, box_cols};
    ZKB_TRY(encode_tensor_map_u64(&map, a.in, 4, dims, strides, box));
    tp.four_d = 1;
  } else {
    const uint64_t R1 = 1ull << a.lR1;
    const uint32_t box_cols = R <= kTmaBoxRows ? (uint32_t)C : 1u;
    const uint64_t dims[3] = {4, (uint64_t)R, R1};
    const uint64_t strides[2] = {32, (uint64_t)R * 32};
    const uint32_t box[3] = {2, rows_box, box_cols};
    ZKB_TRY(encode_tensor_map_u64(&map, a.in, 3, dims, strides, box));
    tp.four_d = 0;
  }
  // One tile per block ("ntt.tma_grid" = 1, the default) lets the block scheduler
  // refill each SM as its blocks finish; measured on B200 against one persistent
  // wave of double-buffered blocks: 2^24 rows 4.97 against 5.29 ms (and against
  // 5.27 ms for the per-thread gather form), 2^22 1.19 against 1.25 ms.
  const bool per_tile = tune_get("ntt.tma_grid") != 0;
  const size_t plane = (size_t)T * 16;
  const size_t rest = ((size_t)R >> 1) * 32 + 2 * 8 + 1024;  // stage table, barriers, alignment slack
  tp.nbuf = !per_tile && 4 * plane + rest <= (110u << 10) ? 2 : 1;
  const size_t smem = (size_t)tp.nbuf * 2 * plane + rest;
  // 128-thread blocks may take a register cap for 5 or 6 blocks per SM ("ntt.tma_blocks_per_sm")
  const int cap = L.threads == 128 ? tune_get("ntt.tma_blocks_per_sm") : 0;
  // lazy reduction between the rounds ("ntt.lazy") needs p < 2^254 (true of BN254's fields)
  const bool lazy = tune_get("ntt.lazy") != 0 && (f.p(7) >> 30) == 0;
  auto kern = cap == 6  ? k_ntt_pass_tma<F, 128, 6>
              : cap == 5 ? k_ntt_pass_tma<F, 128, 5>
              : lazy     ? k_ntt_pass_tma<F, kNttThreads, 1, true>
                         : k_ntt_pass_tma<F>;
  ZKB_TRY(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                     "NTT pass shared memory attribute"));
  int per_sm = 0;
  ZKB_TRY(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, L.threads, smem),
                     "NTT pass occupancy"));
  if (per_sm < 1) return fail(ZKB_ECUDA, "NTT pass of %d threads and %zu bytes does not fit an SM", L.threads, smem);
  const int64_t grid = per_tile ? tp.ntiles : std::min<int64_t>(tp.ntiles, (int64_t)sms * per_sm);
  ProfSpan span(a.last ? "ntt_last_pass" : "ntt_column_pass", s);
  (void)q;
  kern<<<(unsigned)grid, L.threads, smem, s>>>(f, a, tp, map);
  return check_launch("NTT pass launch (TMA)");
}

template <class F>
static int run_ntt(const F& f, const zkb_field* field, const uint64_t* in, uint64_t* out,
                   int64_t n, int invert, const uint64_t* omega, const uint64_t* coset,
                   void* workspace, size_t ws_bytes, cudaStream_t s) {
  const int log_n = ilog2(n);
  int device = 0;
  ZKB_TRY(check_cuda(cudaGetDevice(&device), "cudaGetDevice"));
  const TableKey key = table_key(field, omega, log_n, device);
  RootTables rt;
  ScaleTables st;
  ZKB_TRY(lookup_tables(f, key, n, log_n, invert, coset, rt, st, s));
  ZKB_TRY(lookup_scale_full(f, n, log_n, &st, s));

  const size_t need = workspace_bytes(n);
  if (need && (!workspace || ws_bytes < need)) {
    return fail(ZKB_EWORKSPACE, "NTT of %lld rows needs %zu workspace bytes, got %zu",
                (long long)n, need, ws_bytes);
  }
  std::vector<PassLaunch> passes;
  plan_passes(n, log_n, invert, rt, st, in, out, reinterpret_cast<uint64_t*>(workspace), 0, 0,
              false, passes);
  const int P = (int)passes.size();
  const bool tma = P >= 2 && tune_get("ntt.tma") != 0;
  int sms = 0;
  if (tma) ZKB_TRY(sm_count(device, &sms));
  for (int q = 0; q < P; ++q) {
    if (!passes[q].a.last) {
      ZKB_TRY(lookup_twiddles(f, key, rt, passes[q].a.lr, passes[q].a.ls, invert, &passes[q].a.t_full, s));
    }
    const PassLaunch& L = passes[q];
    if (tma) {
      ZKB_TRY(launch_pass_tma(f, L, n, P, sms, s, q));
      continue;
    }
    auto kern = tune_get("ntt.call_products") ? k_ntt_pass<F, true> : k_ntt_pass<F, false>;
    ZKB_TRY(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)L.smem),
                       "NTT shared memory attribute"));
    ProfSpan span(L.a.last ? (q == 0 ? "ntt_single_pass" : "ntt_last_pass") : "ntt_column_pass", s);
    kern<<<(unsigned)L.ctas, L.threads, L.smem, s>>>(f, L.a);
    ZKB_TRY(check_launch("NTT pass launch"));
  }
  return ZKB_OK;
}

// ---- batches ----------------------------------------------------------------

static constexpr int kMaxBatchJobs = 64;

// Workspace of a batch: the tile counter and status word, one completion
// counter per pass, then each multi-pass transform's intermediate rows.
struct BatchLayout {
  size_t off_counters = 0;  // next tile (u64), status (i32)
  size_t off_done = 0;      // u32 per pass
  std::vector<size_t> off_tmp;
  size_t total = 0;
};

static int batch_layout(const zkb_ntt_job* jobs, int count, BatchLayout& L) {
  if (count < 0 || count > kMaxBatchJobs) {
    return fail(ZKB_EINVAL, "an NTT batch holds 0..%d transforms, got %d", kMaxBatchJobs, count);
  }
  if (count > 0 && !jobs) return fail(ZKB_EINVAL, "null job array");
  L.off_tmp.assign(count, 0);
  size_t off = 0;
  L.off_counters = off;
  off += 256;
  L.off_done = off;
  off += (size_t)kMaxBatchPasses * 4;
  off = (off + 255) & ~(size_t)255;
  for (int j = 0; j < count; ++j) {
    const int64_t n = jobs[j].n;
    if (n < 0 || (n & (n - 1)) || n > (1ll << kMaxLogN)) {
      return fail(ZKB_EINVAL, "job %d: NTT length must be a power of 2 up to 2^28, got %lld", j,
                  (long long)n);
    }
    const size_t need = workspace_bytes(n);
    L.off_tmp[j] = off;
    off += (need + 255) & ~(size_t)255;
  }
  L.total = off;
  return ZKB_OK;
}

template <class F>
static int run_ntt_batch(const F& f, const zkb_field* field, const zkb_ntt_job* jobs, int count,
                         char* ws, const BatchLayout& L, int32_t* status_out, cudaStream_t s) {
  int device = 0;
  ZKB_TRY(check_cuda(cudaGetDevice(&device), "cudaGetDevice"));
  int sms = 0;
  ZKB_TRY(sm_count(device, &sms));
  // largest transforms first, so that their long passes start early
  std::vector<int> order;
  for (int j = 0; j < count; ++j)
    if (jobs[j].n > 1) order.push_back(j);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return jobs[a].n > jobs[b].n; });

  static NttBatchTable T;  // 26 KB: built under the table mutex below, copied into the launch
  static std::mutex table_mutex;
  std::lock_guard<std::mutex> tlock(table_mutex);
  std::memset(&T, 0, sizeof T);
  // tables (built on first use; at most 64 scaling tables, which the cache holds)
  std::vector<RootTables> rts(order.size());
  std::vector<ScaleTables> sts(order.size());
  int max_lr = 0;
  for (size_t k = 0; k < order.size(); ++k) {
    const zkb_ntt_job& J = jobs[order[k]];
    const int log_n = ilog2(J.n);
    ZKB_TRY(lookup_tables(f, table_key(field, nullptr, log_n, device), J.n, log_n, J.invert,
                          J.has_coset ? J.coset : nullptr, rts[k], sts[k], s));
    for (int r : plan_radices(log_n, true)) max_lr = std::max(max_lr, r);
  }
  // one tile shape for every pass: 2^max(10, largest radix) rows, 256 threads
  const int cta_log = std::max(10, max_lr);
  std::vector<std::vector<PassLaunch>> plans(order.size());
  for (size_t k = 0; k < order.size(); ++k) {
    const zkb_ntt_job& J = jobs[order[k]];
    plan_passes(J.n, ilog2(J.n), J.invert, rts[k], sts[k], J.in, J.out,
                reinterpret_cast<uint64_t*>(ws + L.off_tmp[order[k]]), cta_log, kBatchThreads,
                true, plans[k]);
  }
  // tile numbering: pass q of every transform before pass q + 1 of any
  size_t smem = 0;
  int np = 0;
  int64_t tiles = 0;
  std::vector<int> pass_index(order.size() * 3, -1);
  for (int q = 0; q < 3; ++q) {
    for (size_t k = 0; k < order.size(); ++k) {
      if (q >= (int)plans[k].size()) continue;
      if (np >= kMaxBatchPasses) return fail(ZKB_EINVAL, "NTT batch has too many passes");
      const PassLaunch& P = plans[k][q];
      T.pass[np] = P.a;
      T.dep[np] = q > 0 ? pass_index[k * 3 + q - 1] : -1;
      T.tile_start[np] = tiles;
      pass_index[k * 3 + q] = np;
      tiles += P.ctas;
      smem = std::max(smem, P.smem);
      ++np;
    }
  }
  T.num_passes = np;
  T.tile_start[np] = tiles;

  // n = 1 transforms are copies
  for (int j = 0; j < count; ++j) {
    if (jobs[j].n == 1) {
      ZKB_TRY(check_cuda(cudaMemcpyAsync(jobs[j].out, jobs[j].in, 32, cudaMemcpyDeviceToDevice, s),
                         "NTT copy"));
    }
  }
  unsigned long long* next_tile = reinterpret_cast<unsigned long long*>(ws + L.off_counters);
  int* status = reinterpret_cast<int*>(ws + L.off_counters + 8);
  unsigned* done = reinterpret_cast<unsigned*>(ws + L.off_done);
  ZKB_TRY(check_cuda(cudaMemsetAsync(ws, 0, L.off_done + (size_t)kMaxBatchPasses * 4, s),
                     "NTT batch counters"));
  if (np > 0) {
    auto kern = tune_get("ntt.call_products") ? k_ntt_batch<F, true> : k_ntt_batch<F, false>;
    ZKB_TRY(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem),
                       "NTT batch shared memory attribute"));
    int per_sm = 0;
    ZKB_TRY(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchThreads,
                                                                     smem),
                       "NTT batch occupancy"));
    if (per_sm < 1) per_sm = 1;
    const int64_t grid = std::min<int64_t>(tiles, (int64_t)sms * per_sm);
    ProfSpan span("ntt_batch", s);
    const int spin_knob = tune_get("ntt.batch_spin_limit");
    const unsigned spin_limit = spin_knob > 0 ? (unsigned)spin_knob : kBatchSpinLimit;
    kern<<<(unsigned)grid, kBatchThreads, smem, s>>>(f, T, next_tile, done, status, spin_limit);
    ZKB_TRY(check_launch("NTT batch launch"));
  }
  if (status_out) {
    ZKB_TRY(check_cuda(cudaMemcpyAsync(status_out, status, 4, cudaMemcpyDeviceToDevice, s),
                       "NTT batch status"));
  }
  return ZKB_OK;
}

// ---------------------------------------------------------------------------
// The cross-part step of an NTT split over G parts (one per GPU)
// ---------------------------------------------------------------------------
//
// n = G m, and part r holds the rows x[r m .. r m + m) (block layout). With
// j = j1 m + j2 (j1 < G, j2 < m) and k = k1 + k2 G:
//   y[k1 + k2 G] = sum_j2 w_m^(j2 k2) [ w_n^(j2 k1) sum_j1 x[j1 m + j2] w_G^(j1 k1) ].
// After a first exchange part s holds, for its columns j2 = s c + i (c = m / G),
// the G rows x[j1 m + j2] of every j1 (input block j1 came from part j1). This
// step computes, per column, the G-point transform over j1 in registers, the
// twiddle w_n^(j2 k1) and an optional per-block factor post[k1], and writes
// output block k1 (bound for part k1). After a second exchange part t holds
// the bracket for k1 = t and every j2, and an ordinary m-point NTT of it gives
// y[t + k2 G]: the output is in cyclic layout. An inverse uses w^-1 and
// post[k1] = G^-1 (times g^-k1 for a coset); a forward coset transform scales
// x[j] by g^j on the way in.

template <class F, int LG>
__global__ void __launch_bounds__(128) k_ntt_cross(F f, const uint64_t* in, uint64_t* out,
                                                    int64_t c, int64_t m, int part, int log_n,
                                                    int inverse, RootTables rt, ScaleTables st,
                                                    const uint64_t* post) {
  constexpr int G = 1 << LG;
  const uint64_t N = 1ull << rt.log_N;
  const int shift = rt.log_N - log_n;  // w_n^e = w_N^(e 2^shift)
  const uint64_t mask = (1ull << rt.s) - 1;
  auto root = [&](uint32_t r[8], uint64_t e_n) {  // w_n^(+-e_n), e_n < n
    uint64_t e = e_n << shift;
    if (inverse && e) e = N - e;
    uint32_t lo[8], hi[8];
    fe_load_nc(lo, rt.t_lo + 4 * (e & mask));
    fe_load_nc(hi, rt.t_hi + 4 * (e >> rt.s));
    fe_mul(r, lo, hi, f);
  };
  // w_G^t for t < G / 2
  uint32_t wg[G / 2 > 0 ? G / 2 : 1][8];
#pragma unroll
  for (int t = 0; t < G / 2; ++t) root(wg[t], (uint64_t)t * (uint64_t)m);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c; i += stride) {
    const int64_t j2 = (int64_t)part * c + i;
    uint32_t a[G][8];
#pragma unroll
    for (int j1 = 0; j1 < G; ++j1) {
      // bit-reversed order for the in-place decimation-in-time transform below
      const int src = (int)(__brev((unsigned)j1) >> (32 - (LG > 0 ? LG : 1))) & (G - 1);
      fe_load_nc(a[j1], in + 4 * ((int64_t)src * c + i));
      if (st.g_lo && !inverse) {
        const uint64_t j = (uint64_t)src * (uint64_t)m + (uint64_t)j2;
        const uint64_t gm = (1ull << st.gs) - 1;
        uint32_t lo[8], hi[8];
        fe_load_nc(lo, st.g_lo + 4 * (j & gm));
        fe_load_nc(hi, st.g_hi + 4 * (j >> st.gs));
        fe_mul(lo, lo, hi, f);
        fe_mul(a[j1], a[j1], lo, f);
      }
    }
#pragma unroll
    for (int h = 1; h < G; h <<= 1) {
#pragma unroll
      for (int b = 0; b < G; b += 2 * h) {
#pragma unroll
        for (int jj = 0; jj < h; ++jj) {
          uint32_t v[8], u[8];
          fe_copy(u, a[b + jj]);
          if (jj) {
            fe_mul(v, a[b + jj + h], wg[jj * (G / (2 * h))], f);
          } else {
            fe_copy(v, a[b + jj + h]);
          }
          fe_add(a[b + jj], u, v, f);
          fe_sub(a[b + jj + h], u, v, f);
        }
      }
    }
    // twiddle w_n^(j2 k1) by successive powers of w_n^j2, then the block factor
    uint32_t base[8], tw[8];
    root(base, (uint64_t)j2);
    fe_copy(tw, base);
#pragma unroll
    for (int k1 = 0; k1 < G; ++k1) {
      uint32_t x[8];
      fe_copy(x, a[k1]);
      if (k1 > 0) {
        fe_mul(x, x, tw, f);
        if (k1 + 1 < G) fe_mul(tw, tw, base, f);
      }
      if (post) {  // Montgomery row post[k1]
        uint32_t pf[8];
        fe_load_nc(pf, post + 4 * k1);
        fe_mul(x, x, pf, f);
      }
      fe_store(out + 4 * ((int64_t)k1 * c + i), x);
    }
  }
}

template <class F>
static int run_cross(const F& f, const zkb_field* field, const uint64_t* in, uint64_t* out,
                     int64_t n, int parts, int part, int invert, const uint64_t* coset,
                     const uint64_t* post, cudaStream_t s) {
  const int log_n = ilog2(n);
  int lg = 0;
  while ((1 << lg) < parts) ++lg;
  int device = 0;
  ZKB_TRY(check_cuda(cudaGetDevice(&device), "cudaGetDevice"));
  RootTables rt;
  ScaleTables st;
  // forward coset: the scaling tables g^j of size n (inverse transforms take post[])
  ZKB_TRY(lookup_tables(f, table_key(field, nullptr, log_n, device), n, log_n, 0,
                        invert ? nullptr : coset, rt, st, s));
  const int64_t m = n >> lg, c = m >> lg;
  const unsigned grid = grid_for(c, 128);
  switch (lg) {
    case 1: k_ntt_cross<F, 1><<<grid, 128, 0, s>>>(f, in, out, c, m, part, log_n, invert, rt, st, post); break;
    case 2: k_ntt_cross<F, 2><<<grid, 128, 0, s>>>(f, in, out, c, m, part, log_n, invert, rt, st, post); break;
    case 3: k_ntt_cross<F, 3><<<grid, 128, 0, s>>>(f, in, out, c, m, part, log_n, invert, rt, st, post); break;
    default: k_ntt_cross<F, 4><<<grid, 128, 0, s>>>(f, in, out, c, m, part, log_n, invert, rt, st, post); break;
  }
  return check_launch("NTT cross-part step");
}

}  // namespace zkb

using namespace zkb;

extern "C" {

size_t zkb_ntt_workspace_bytes(int64_t n) { return zkb::workspace_bytes(n); }

uint64_t zkb_ntt_wait_timeouts(void) {
  unsigned v = 0;
  if (cudaMemcpyFromSymbol(&v, zkb::g_ntt_tma_timeouts, sizeof v) != cudaSuccess) return ~0ull;
  return v;
}

int zkb_ntt(const zkb_field* f, const uint64_t* in, uint64_t* out, int64_t n, int invert,
            const uint64_t* omega, const uint64_t* coset, void* workspace,
            size_t workspace_bytes, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_field(f));
  if (n < 0 || (n & (n - 1)) || n > (1ll << kMaxLogN)) {
    return fail(ZKB_EINVAL, "NTT length must be a power of 2 up to 2^28, got %lld", (long long)n);
  }
  if (n == 0) return ZKB_OK;
  if (!in || !out) return fail(ZKB_EINVAL, "null buffer");
  if (in == out) return fail(ZKB_EINVAL, "NTT output must not alias its input");
  ZKB_TRY(check_align(in, 16, "in"));
  ZKB_TRY(check_align(out, 16, "out"));
  ZKB_TRY(check_align(workspace, 16, "workspace"));
  if (!omega && f->kind != ZKB_FIELD_BN254_FR) {
    return fail(ZKB_EINVAL, "a root of unity is required for fields other than BN254 Fr");
  }
  cudaStream_t s = as_stream(stream);
  if (n == 1) {
    // a single value transforms to itself; n^-1 = 1 and g^0 = 1
    return check_cuda(cudaMemcpyAsync(out, in, 32, cudaMemcpyDeviceToDevice, s), "NTT copy");
  }
  return with_field(f, [&](auto fp) {
    return run_ntt(fp, f, in, out, n, invert, omega, coset, workspace, workspace_bytes, s);
  });
}

int zkb_ntt_cross_step(const zkb_field* f, const uint64_t* in, uint64_t* out, int64_t n, int parts,
                       int part, int invert, const uint64_t* coset, const uint64_t* post,
                       void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_field(f));
  if (f->kind != ZKB_FIELD_BN254_FR) {
    return fail(ZKB_EINVAL, "split NTTs use BN254 Fr's built-in roots of unity");
  }
  if (parts < 2 || parts > 16 || (parts & (parts - 1))) {
    return fail(ZKB_EINVAL, "parts must be a power of 2 in 2..16, got %d", parts);
  }
  if (part < 0 || part >= parts) return fail(ZKB_EINVAL, "part %d out of 0..%d", part, parts - 1);
  if (n < (int64_t)parts * parts || (n & (n - 1)) || n > (1ll << kMaxLogN)) {
    return fail(ZKB_EINVAL, "NTT length must be a power of 2 in parts^2..2^28, got %lld",
                (long long)n);
  }
  if (!in || !out) return fail(ZKB_EINVAL, "null buffer");
  if (in == out) return fail(ZKB_EINVAL, "output must not alias the input");
  ZKB_TRY(check_align(in, 16, "in"));
  ZKB_TRY(check_align(out, 16, "out"));
  ZKB_TRY(check_align(post, 16, "post"));
  cudaStream_t s = as_stream(stream);
  return run_cross(FrP{}, f, in, out, n, parts, part, invert, coset, post, s);
}

size_t zkb_ntt_batch_workspace_bytes(const zkb_ntt_job* jobs, int count) {
  set_error("%s", "");
  BatchLayout L;
  if (batch_layout(jobs, count, L) != ZKB_OK) return 0;
  return L.total;
}

int zkb_ntt_batch(const zkb_field* f, const zkb_ntt_job* jobs, int count, void* workspace,
                  size_t workspace_bytes, int32_t* status, void* stream) {
  set_error("%s", "");
  ZKB_TRY(check_field(f));
  if (f->kind != ZKB_FIELD_BN254_FR) {
    return fail(ZKB_EINVAL, "batched NTTs use BN254 Fr's built-in roots of unity");
  }
  BatchLayout L;
  ZKB_TRY(batch_layout(jobs, count, L));
  if (!workspace || workspace_bytes < L.total) {
    return fail(ZKB_EWORKSPACE, "NTT batch of %d transforms needs %zu workspace bytes, got %zu",
                count, L.total, workspace_bytes);
  }
  ZKB_TRY(check_align(workspace, 256, "workspace"));
  if (status) ZKB_TRY(check_align(status, 4, "status"));
  for (int j = 0; j < count; ++j) {
    const zkb_ntt_job& J = jobs[j];
    if (J.n == 0) continue;
    if (!J.in || !J.out) return fail(ZKB_EINVAL, "job %d: null buffer", j);
    if (J.in == J.out) return fail(ZKB_EINVAL, "job %d: NTT output must not alias its input", j);
    ZKB_TRY(check_align(J.in, 16, "in"));
    ZKB_TRY(check_align(J.out, 16, "out"));
  }
  cudaStream_t s = as_stream(stream);
  return run_ntt_batch(FrP{}, f, jobs, count, reinterpret_cast<char*>(workspace), L, status, s);
}

}  // extern "C"
