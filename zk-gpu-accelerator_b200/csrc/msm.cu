// msm.cu — Pippenger multi-scalar multiplication over BN254 G1, entirely on
// the device, and its C ABI.
//
// Pipeline for sum_i s_i P_i (zkgpu/msm_gpu.py:1-35 describes the reference's
// version; here every step, including the final combination, is on the GPU):
//   1. digits    one thread per scalar: reduce mod r, recode into W signed
//                w-bit digits d (|d| <= 2^(w-1)), and emit one (bucket, point)
//                pair per nonzero digit: key = window * 2^(w-1) + |d| - 1,
//                value = point index | sign << 31.
//   2. sort      group the pairs by key, so every bucket's points are
//                contiguous: either a counting sort ("msm.sort" = 1): the
//                digits pass counts each key (warp-aggregated atomics, zero
//                digits skipped), a scan turns counts into bucket offsets, and
//                a second digits pass scatters each pair into its bucket's
//                range; or a radix sort of all 2 W n pairs by key (CUB
//                onesweep, "msm.sort" = 0), zero digits carrying the largest
//                key and sorting to the end.
//   3. buckets   level 1: each thread adds a fixed run of K1 sorted pairs into
//                XYZZ accumulators with mixed additions, so every thread does
//                the same work however skewed the buckets are. A bucket wholly
//                inside one thread's run is written out directly; a bucket
//                that crosses a run boundary leaves partial sums in per-thread
//                slots, which later levels merge the same way (full XYZZ
//                additions) until every bucket is complete. No host sync.
//   4. reduction sum_b (b + 1) B_b per window by running sums over segments of
//                L buckets, recursively over the segment sums (below).
//   5. finalize  Horner over the window sums (w doublings per window) and one
//                inversion to affine (zkgpu/msm.py:156-169, curve.py:221-233).
//
// Window-sum recursion: for a segment t of L consecutive entries X_{tL+i},
// running sums from the top give S_t = sum_i X_{tL+i} and
// U_t = sum_i (i + delta) X_{tL+i}; then
//   sum_b (b + delta) X_b = sum_t U_t + L * sum_t t S_t,
// and the last term is the same problem on the L S_t with delta = 0.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "curve.cuh"
#include "fanout.h"
#include "field_host.h"
#include "profile.h"

namespace zkb {

static constexpr int kMsmMaxWindow = 20;
static constexpr int kHalfBits = 128;       // GLV halves: |k1|, |k2| < 2^127

// Windows per GLV half: signed digits need W w >= 128 so that the top window
// (at most 127 - (W - 1) w value bits, plus a borrow) never exceeds 2^(w-1).
static int num_windows(int w) { return (kHalfBits + w - 1) / w; }

// ---------------------------------------------------------------------------
// GLV: BN254 G1 has the endomorphism phi(x, y) = (beta x, y) = lambda (x, y)
// for cube roots of unity beta in Fq and lambda in Fr. Each scalar splits as
// k = k1 + k2 lambda (mod r) with |k1|, |k2| < 2^127, so sum k_i P_i =
// sum k1_i P_i + k2_i phi(P_i): twice the points at half the bits. The
// accumulation work is unchanged, but the windows (and so the bucket
// reduction) halve, and the final doubling chain is 112 doublings instead of
// 240. Only the affine sum is compared with the reference, which is the same
// for every decomposition.
//
// Decomposition (Babai rounding against the reduced lattice basis
// v1 = (a1, b1), v2 = (a2, b2) of {(x, y): x + y lambda = 0 mod r}, computed
// offline from lambda by the extended Euclidean algorithm):
//   c1 = floor(k g1 / 2^256), g1 = round(b2 2^256 / r)
//   c2 = floor(k g2 / 2^256), g2 = round(-b1 2^256 / r)
//   k1 = k - c1 a1 - c2 a2,   k2 = -c1 b1 - c2 b2
// The exact products cancel (a1 b2 - a2 b1 = r), leaving
// |k1| <= |a1| + |a2| < 2^127 and |k2| <= |b1| + |b2| < 2^127.
// ---------------------------------------------------------------------------

// beta (Montgomery form over Fq), the cube root of unity with phi = lambda.
// beta = 0x59e26bcea0d48bacd4f263f1acdb5c4f5763473177fffffe.
__device__ __forceinline__ void glv_beta_mont(uint32_t r[8]) {
  const uint32_t beta[8] = {0x77fffffeu, 0x57634731u, 0xacdb5c4fu, 0xd4f263f1u,
                            0xa0d48bacu, 0x59e26bceu, 0u, 0u};
  fe_to_mont(r, beta, FqP{});
}

// Basis and rounding constants, little-endian 32-bit limbs:
//   a1 = b2 = 9931322734385697763 (64 bits)
//   b1 = -147946756881789319000765030803803410728 (|b1| has 127 bits)
//   a2 = 147946756881789319010696353538189108491 (127 bits)
//   g1 = round(b2 2^256 / r) (66 bits), g2 = round(-b1 2^256 / r) (130 bits)
__device__ __forceinline__ uint32_t glv_a1(int i) {
  constexpr uint32_t v[2] = {0x94d213e3u, 0x89d32568u};
  return v[i];
}
__device__ __forceinline__ uint32_t glv_b1_abs(int i) {
  constexpr uint32_t v[4] = {0x7d4f1128u, 0x8211bbebu, 0xeeb859fcu, 0x6f4d8248u};
  return v[i];
}
__device__ __forceinline__ uint32_t glv_a2(int i) {
  constexpr uint32_t v[4] = {0x1221250bu, 0x0be4e154u, 0xeeb859fdu, 0x6f4d8248u};
  return v[i];
}
__device__ __forceinline__ uint32_t glv_g1(int i) {
  constexpr uint32_t v[3] = {0xc7e0b3d7u, 0xd91d232eu, 0x00000002u};
  return v[i];
}
__device__ __forceinline__ uint32_t glv_g2(int i) {
  constexpr uint32_t v[5] = {0x391eb18eu, 0x7a7bd9d4u, 0xa773d2cfu, 0x4ccef014u, 0x00000002u};
  return v[i];
}

// k1, k2 (as 128-bit magnitudes with signs) for a scalar k < r (8 limbs).
__device__ __forceinline__ void glv_split(const uint32_t k[8], uint32_t k1[4], uint32_t& neg1,
                                          uint32_t k2[4], uint32_t& neg2) {
  // c1 = floor(k g1 / 2^256): limbs 8..9 of the 8 x 3 product
  uint32_t p1[11];
#pragma unroll
  for (int i = 0; i < 11; ++i) p1[i] = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    uint64_t c = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint64_t t = (uint64_t)k[i] * glv_g1(j) + p1[i + j] + c;
      p1[i + j] = (uint32_t)t;
      c = t >> 32;
    }
    p1[8 + j] = (uint32_t)c;
  }
  const uint32_t c1[2] = {p1[8], p1[9]};
  // c2 = floor(k g2 / 2^256): limbs 8..11 of the 8 x 5 product
  uint32_t p2[13];
#pragma unroll
  for (int i = 0; i < 13; ++i) p2[i] = 0;
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    uint64_t c = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint64_t t = (uint64_t)k[i] * glv_g2(j) + p2[i + j] + c;
      p2[i + j] = (uint32_t)t;
      c = t >> 32;
    }
    p2[8 + j] = (uint32_t)c;
  }
  const uint32_t c2[4] = {p2[8], p2[9], p2[10], p2[11]};
  // low 128 bits of c1 a1, c2 a2, c1 |b1|, c2 b2
  uint32_t t1[4] = {0, 0, 0, 0}, t2[4] = {0, 0, 0, 0}, t3[4] = {0, 0, 0, 0}, t4[4] = {0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    uint64_t ca = 0, cb = 0;
#pragma unroll
    for (int j = 0; i + j < 4; ++j) {
      const uint64_t x = (uint64_t)c1[i] * (j < 2 ? glv_a1(j) : 0u) + t1[i + j] + ca;
      t1[i + j] = (uint32_t)x;
      ca = x >> 32;
      const uint64_t y = (uint64_t)c1[i] * glv_b1_abs(j) + t3[i + j] + cb;
      t3[i + j] = (uint32_t)y;
      cb = y >> 32;
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    uint64_t ca = 0, cb = 0;
#pragma unroll
    for (int j = 0; i + j < 4; ++j) {
      const uint64_t x = (uint64_t)c2[i] * glv_a2(j) + t2[i + j] + ca;
      t2[i + j] = (uint32_t)x;
      ca = x >> 32;
      const uint64_t y = (uint64_t)c2[i] * (j < 2 ? glv_a1(j) : 0u) + t4[i + j] + cb;  // b2 = a1
      t4[i + j] = (uint32_t)y;
      cb = y >> 32;
    }
  }
  // k1 = k - t1 - t2 and k2 = t3 - t4, both mod 2^128 (the true values lie in
  // (-2^127, 2^127)); the carry is signed: floor(d / 2^32) by arithmetic shift
  int64_t carry = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t d = (int64_t)k[i] - (int64_t)t1[i] - (int64_t)t2[i] + carry;
    k1[i] = (uint32_t)d;
    carry = d >> 32;
  }
  carry = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t d = (int64_t)t3[i] - (int64_t)t4[i] + carry;
    k2[i] = (uint32_t)d;
    carry = d >> 32;
  }
  // magnitudes and signs
  neg1 = k1[3] >> 31;
  neg2 = k2[3] >> 31;
  uint64_t c = 1;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint64_t v = (uint64_t)(neg1 ? ~k1[i] : k1[i]) + (neg1 ? c : 0);
    k1[i] = (uint32_t)v;
    c = v >> 32;
  }
  c = 1;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint64_t v = (uint64_t)(neg2 ? ~k2[i] : k2[i]) + (neg2 ? c : 0);
    k2[i] = (uint32_t)v;
    c = v >> 32;
  }
}

// ---------------------------------------------------------------------------
// Batches: several independent MSMs with one window size run through one
// pipeline. Job j's buckets take keys [j K, (j + 1) K) with K = W 2^(w-1), so
// "window" j W + win of the batch is window win of job j: the sort, the
// bucket levels and the reduction see one MSM with count * W windows, and
// only the digits, the point lookups and the finalize know about jobs. The
// table travels as a kernel parameter (2.6 KB), so a batch needs no host to
// device copy and can be captured in a CUDA graph.
// ---------------------------------------------------------------------------

static constexpr int kMsmMaxBatch = 64;

struct MsmJobs {
  int count;
  uint32_t keys_per_job;              // W 2^(w-1)
  int64_t first[kMsmMaxBatch + 1];    // prefix sums of the jobs' point counts
  const uint64_t* points[kMsmMaxBatch];
  const uint64_t* scalars[kMsmMaxBatch];
  uint64_t* phi[kMsmMaxBatch];        // phi images, in the workspace
  uint64_t* result[kMsmMaxBatch];
  int64_t pts_n[kMsmMaxBatch];        // rows of points[j]: n_j, or n_j 2 W for a fixed-base table
};

// The job holding batch-wide point index i (first[j] <= i < first[j + 1]).
__device__ __forceinline__ int job_of_point(const MsmJobs& J, int64_t i) {
  int lo = 0, hi = J.count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (J.first[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// 1. digits
// ---------------------------------------------------------------------------

// Bits [lo, lo + w) of a 128-bit little-endian magnitude (w <= 20, so at most
// two limbs; bits at and above 128 are zero).
__device__ __forceinline__ uint32_t half_bits(const uint32_t s[4], int lo, int w) {
  if (lo >= 128) return 0;
  const int limb = lo >> 5, off = lo & 31;
  uint64_t v = s[limb];
  if (limb + 1 < 4) v |= (uint64_t)s[limb + 1] << 32;
  return (uint32_t)(v >> off) & ((1u << w) - 1u);
}

// Signed w-bit digits of one GLV half |k| (sign neg) of point `point`: the pair
// (key, value) for window win goes to entry first_entry + win * n, its key is
// key_base + win 2^(w-1) + |d| - 1.
__device__ __forceinline__ void emit_digits(const uint32_t k[4], uint32_t neg, uint32_t point,
                                            int64_t first_entry, int64_t n, int w, int W,
                                            uint32_t key_base, uint32_t none, uint32_t* keys,
                                            uint32_t* vals) {
  const uint32_t half = 1u << (w - 1);
  uint32_t carry = 0;
  for (int win = 0; win < W; ++win) {
    const uint32_t raw = half_bits(k, win * w, w) + carry;
    uint32_t mag, dneg = 0;
    if (win + 1 < W && raw > half) {
      // raw - 2^w in [-(2^(w-1) - 1), 0], borrowing 1 from the next window
      mag = (1u << w) - raw;
      dneg = 1;
      carry = 1;
    } else {
      mag = raw;
      carry = 0;
    }
    const int64_t e = first_entry + (int64_t)win * n;
    if (mag == 0) {
      keys[e] = none;
      vals[e] = 0;
    } else {
      keys[e] = key_base + (((uint32_t)win << (w - 1)) | (mag - 1));
      vals[e] = point | ((neg ^ dneg) << 31);
    }
  }
}

// One thread per scalar of the batch: reduce mod r, split k = k1 + k2 lambda,
// and emit the digits of k1 (the job's points 0..n-1) and of k2 (its points
// n..2n-1, the phi images). Job j's 2 W n_j entries start at 2 W first[j].
__global__ void __launch_bounds__(256) k_msm_digits(const MsmJobs J, int w, int W, uint32_t none,
                                                    uint32_t* keys, uint32_t* vals) {
  FrP fr;
  const int64_t N = J.first[J.count];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += stride) {
    const int j = job_of_point(J, g);
    const int64_t n = J.first[j + 1] - J.first[j], i = g - J.first[j];
    const int64_t base = 2 * (int64_t)W * J.first[j];
    const uint32_t key_base = (uint32_t)j * J.keys_per_job;
    uint32_t s[8];
    fe_load_nc(s, J.scalars[j] + 4 * i);
    fe_reduce_full(s, fr, 5);  // any 256-bit value -> [0, r)
    uint32_t k1[4], k2[4], neg1, neg2;
    glv_split(s, k1, neg1, k2, neg2);
    emit_digits(k1, neg1, (uint32_t)i, base + i, n, w, W, key_base, none, keys, vals);
    emit_digits(k2, neg2, (uint32_t)(n + i), base + (int64_t)W * n + i, n, w, W, key_base, none,
                keys, vals);
  }
}

// Counting sort of the pairs (no entry for a zero digit). One thread per scalar,
// a warp at a time: lanes whose digits fall in the same bucket take one atomic
// together (__match_any_sync), so a bucket that most scalars share (skewed
// scalars: digit 1 of window 0) costs one atomic per warp, not per lane.
// kScatter = false: count[key] += pairs. kScatter = true: each pair takes the
// next slot of its bucket, cursor[key]++ (the cursors start at the bucket
// offsets), and is written there as one 8-byte (key, value) word. Within a bucket the order of the pairs
// varies from run to run; the bucket sum, and so the result, does not.
// With a fixed-base table (table = 1) every window shares the job's one set of
// 2^(w-1) buckets: key = |d| - 1, and the value names the table row of
// 2^(w win) P (or of its phi image), (point 2 + half) W + win.
template <bool kScatter>
__global__ void __launch_bounds__(256) k_msm_bucket_digits(const MsmJobs J, int w, int W, uint32_t none,
                                                           int table, uint32_t* ctr, uint2* pairs) {
  FrP fr;
  const int64_t N = J.first[J.count];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;  // a multiple of 32
  const int lane = threadIdx.x & 31;
  const uint32_t half = 1u << (w - 1);
  for (int64_t g0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); g0 < N; g0 += stride) {
    const int64_t g = g0 + lane;  // the whole warp runs every iteration; lanes past N have no digits
    uint32_t k[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}}, neg[2] = {0, 0};
    int64_t n = 0, i = 0;
    uint32_t key_base = 0;
    if (g < N) {
      const int j = job_of_point(J, g);
      n = J.first[j + 1] - J.first[j];
      i = g - J.first[j];
      key_base = (uint32_t)j * J.keys_per_job;
      uint32_t sc[8];
      fe_load_nc(sc, J.scalars[j] + 4 * i);
      fe_reduce_full(sc, fr, 5);
      glv_split(sc, k[0], neg[0], k[1], neg[1]);
    }
    for (int h = 0; h < 2; ++h) {
      const uint32_t point = (uint32_t)(h ? n + i : i);
      uint32_t carry = 0;
      for (int win = 0; win < W; ++win) {
        const uint32_t raw = half_bits(k[h], win * w, w) + carry;
        uint32_t mag, dneg = 0;
        if (win + 1 < W && raw > half) {
          mag = (1u << w) - raw;
          dneg = 1;
          carry = 1;
        } else {
          mag = raw;
          carry = 0;
        }
        const uint32_t key =
            mag ? key_base + (table ? mag - 1 : (((uint32_t)win << (w - 1)) | (mag - 1))) : none;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(peers) - 1;
        if (!kScatter) {
          if (lane == leader && key != none) atomicAdd(ctr + key, (uint32_t)__popc(peers));
        } else {
          uint32_t base = 0;
          if (lane == leader && key != none) base = atomicAdd(ctr + key, (uint32_t)__popc(peers));
          base = __shfl_sync(0xffffffffu, base, leader);
          if (key != none) {
            const uint32_t pos = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
            const uint32_t row = table ? (uint32_t)((2 * i + h) * W + win) : point;
            pairs[pos] = make_uint2(key, row | ((neg[h] ^ dneg) << 31));
          }
        }
      }
    }
  }
}

// phi(P_i) = (beta x_i, y_i), the points that the k2 halves multiply.
__global__ void __launch_bounds__(256) k_msm_phi(const MsmJobs J) {
  FqP f;
  uint32_t beta[8];
  glv_beta_mont(beta);
  const int64_t N = J.first[J.count];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += stride) {
    const int j = job_of_point(J, g);
    const int64_t i = g - J.first[j];
    uint32_t x[8], y[8];
    fe_load_nc(x, J.points[j] + 8 * i);
    fe_load_nc(y, J.points[j] + 8 * i + 4);
    fe_mul(x, x, beta, f);
    fe_store(J.phi[j] + 8 * i, x);
    fe_store(J.phi[j] + 8 * i + 4, y);
  }
}

// ---------------------------------------------------------------------------
// Fixed-base tables (no counterpart in the reference, which takes its points
// with every call). For a base set that stays resident across many MSMs, the
// table holds per point P_i its 2 W rows 2^(w win) P_i and phi(2^(w win) P_i),
// win < W, affine Montgomery, at rows (2 i + half) W + win. An MSM over the
// table adds every window's digits into one set of 2^(w-1) buckets, so a job
// reduces one window and its final combination needs no doublings; the
// smaller bucket work allows larger windows, i.e. fewer mixed additions.
// ---------------------------------------------------------------------------

static constexpr int kTableMinWindow = 8, kTableMaxWindow = 24;
static constexpr int kTableMaxWindows = 16;  // ceil(128 / 8)

// One thread per base point: the W multiples by w doublings each (XYZZ), one
// inversion for all of them (prefix products of ZZ ZZZ), then x = X / ZZ,
// y = Y / ZZZ and the phi images (beta x, y).
__global__ void __launch_bounds__(128) k_msm_table_build(const uint64_t* points, int64_t n, int w, int W,
                                                         uint64_t* table) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  G1F f;
  uint32_t beta[8];
  glv_beta_mont(beta);
  Aff p;
  aff_load_nc(p, points + 8 * i);
  Xyzz m[kTableMaxWindows];
  xyzz_from_affine(m[0], p);
  for (int k = 1; k < W; ++k) {
    m[k] = m[k - 1];
    for (int d = 0; d < w; ++d) xyzz_dbl<CallMul>(m[k], m[k]);
  }
  uint32_t pre[kTableMaxWindows][8];  // pre[k] = prod_{t <= k} ZZ_t ZZZ_t
  fe_mul(pre[0], m[0].zz, m[0].zzz, f);
  for (int k = 1; k < W; ++k) {
    uint32_t t[8];
    fe_mul(t, m[k].zz, m[k].zzz, f);
    fe_mul(pre[k], pre[k - 1], t, f);
  }
  uint32_t inv[8];  // 1 / pre[k], walking down
  fe_inv(inv, pre[W - 1], f);
  for (int k = W - 1; k >= 0; --k) {
    uint32_t ik[8], t[8], x[8], y[8];
    if (k > 0) {
      fe_mul(ik, inv, pre[k - 1], f);  // 1 / (ZZ_k ZZZ_k)
      fe_mul(t, m[k].zz, m[k].zzz, f);
      fe_mul(inv, inv, t, f);          // 1 / pre[k - 1]
    } else {
      fe_copy(ik, inv);
    }
    fe_mul(t, ik, m[k].zzz, f);  // 1 / ZZ
    fe_mul(x, m[k].x, t, f);
    fe_mul(t, ik, m[k].zz, f);   // 1 / ZZZ
    fe_mul(y, m[k].y, t, f);
    uint64_t* row = table + 8 * ((2 * i) * W + k);
    fe_store(row, x);
    fe_store(row + 4, y);
    fe_mul(x, x, beta, f);
    row = table + 8 * ((2 * i + 1) * W + k);
    fe_store(row, x);
    fe_store(row + 4, y);
  }
}

// ---------------------------------------------------------------------------
// 3. bucket accumulation
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_xyzz_fill_identity(uint64_t* pts, int64_t count) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    // ZZ = ZZZ = 0 marks the identity; X and Y are ignored then
    const uint4 z = make_uint4(0, 0, 0, 0);
    uint4* p = reinterpret_cast<uint4*>(pts + 16 * i);
#pragma unroll
    for (int k = 0; k < 8; ++k) p[k] = z;
  }
}

// Writes a finished run: straight to its bucket when the run lies wholly in
// this thread's range, else into this thread's head slot (first run) or tail
// slot (last run). A single run that is shared fills the head slot and puts an
// identity with the same key in the tail slot, so the slots of one bucket stay
// contiguous for the next level.
struct RunSink {
  uint64_t* buckets;
  uint32_t* slot_keys;
  uint64_t* slot_pts;
  int64_t t;
  uint32_t prev_key, next_key, none;

  __device__ __forceinline__ void flush(uint32_t key, const Xyzz& acc, bool is_first,
                                        bool is_last) const {
    if (key == none) return;
    const bool shared = (is_first && prev_key == key) || (is_last && next_key == key);
    if (!shared) {
      xyzz_store(buckets + 16 * (int64_t)key, acc);
      return;
    }
    if (is_first) {
      slot_keys[2 * t] = key;
      xyzz_store(slot_pts + 16 * (2 * t), acc);
      if (is_last) {
        Xyzz id;
        xyzz_set_identity(id);
        slot_keys[2 * t + 1] = key;
        xyzz_store(slot_pts + 16 * (2 * t + 1), id);
      }
    } else {
      slot_keys[2 * t + 1] = key;
      xyzz_store(slot_pts + 16 * (2 * t + 1), acc);
    }
  }
};

// The points of the job that owns bucket key `key`.
struct JobPoints {
  const uint64_t* points;
  const uint64_t* phi;
  int64_t n;
};

__device__ __forceinline__ JobPoints job_points(const MsmJobs& J, uint32_t key) {
  const int j = (int)(key / J.keys_per_job);
  return JobPoints{J.points[j], J.phi[j], J.pts_n[j]};
}

// Level 1: K1 sorted (key, value) pairs per thread, mixed additions of affine
// input points. kBatch = false is the one-job form: the job lookup at each
// new run costs 40+ registers, so a single MSM keeps its point arrays fixed.
// E_dev (null for the radix sort): the number of pairs the counting sort wrote,
// at most E; the threads past it only clear their slots. Pair e is
// (keys[e st], vals[e st]): st = 1 for the radix sort's two arrays, 2 for the
// counting sort's interleaved (key, value) words.
template <bool kBatch, class M>
__device__ __forceinline__ void acc_points(const MsmJobs& J, const uint32_t* keys,
                                           const uint32_t* vals, int st, int64_t E, const uint32_t* E_dev,
                                           int K, uint32_t none, uint64_t* buckets, uint32_t* slot_keys,
                                           uint64_t* slot_pts) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t T = (E + K - 1) / K;
  if (t >= T) return;
  slot_keys[2 * t] = none;
  slot_keys[2 * t + 1] = none;
  if (E_dev) E = *E_dev;
  const int64_t start = t * K;
  if (start >= E) return;
  const int64_t end = start + K < E ? start + K : E;
  RunSink sink{buckets, slot_keys, slot_pts, t, start > 0 ? keys[(start - 1) * st] : none,
               end < E ? keys[end * st] : none, none};
  uint32_t cur = keys[start * st];
  bool first = true;
  Xyzz acc;
  xyzz_set_identity(acc);
  JobPoints jp = job_points(J, (!kBatch || cur == none) ? 0 : cur);
  for (int64_t e = start; e < end; ++e) {
    const uint32_t k = keys[e * st];
    if (k != cur) {
      sink.flush(cur, acc, first, false);
      first = false;
      xyzz_set_identity(acc);
      cur = k;
      if (kBatch && k != none) jp = job_points(J, k);
    }
    if (k == none) break;  // zero digits sort last: nothing after them
    const uint32_t v = vals[e * st];
    const int64_t idx = (int64_t)(v & 0x7fffffffu);
    Aff q;
    aff_load_nc(q, idx < jp.n ? jp.points + 8 * idx : jp.phi + 8 * (idx - jp.n));
    if (aff_is_inf(q)) continue;  // a bucket entry that summed to infinity in an affine round
    if (v >> 31) aff_neg(q);
    xyzz_add_affine<M>(acc, q);
  }
  if (cur != none) sink.flush(cur, acc, first, true);
}

// One MSM: capped at 128 registers, four CTAs per SM.
template <class M>
__global__ void __launch_bounds__(128, 4) k_msm_acc_points(const MsmJobs J, const uint32_t* keys,
                                                        const uint32_t* vals, int st, int64_t E,
                                                        const uint32_t* E_dev, int K, uint32_t none,
                                                        uint64_t* buckets, uint32_t* slot_keys,
                                                        uint64_t* slot_pts) {
  acc_points<false, M>(J, keys, vals, st, E, E_dev, K, none, buckets, slot_keys, slot_pts);
}

// A batch: capped at 128 registers (a few bytes of spill on the job-change
// path) to keep four CTAs per SM.
template <class M>
__global__ void __launch_bounds__(128, 4) k_msm_acc_points_batch(const MsmJobs J,
                                                                 const uint32_t* keys,
                                                                 const uint32_t* vals, int st, int64_t E,
                                                                 const uint32_t* E_dev, int K,
                                                                 uint32_t none, uint64_t* buckets,
                                                                 uint32_t* slot_keys,
                                                                 uint64_t* slot_pts) {
  acc_points<true, M>(J, keys, vals, st, E, E_dev, K, none, buckets, slot_keys, slot_pts);
}

// ---------------------------------------------------------------------------
// 3a. affine rounds before the XYZZ levels (large MSMs)
// ---------------------------------------------------------------------------
//
// Each round halves every bucket's list: entry m of a bucket's output is the
// sum of its input entries 2m and 2m + 1 (or a copy of entry 2m when it is the
// last), added in affine coordinates. An affine addition needs the inverse of
// x2 - x1; with the inverses shared (Montgomery's simultaneous inversion) it
// costs 5 products and 1 squaring, against 8 and 2 for the XYZZ mixed
// addition the run kernels use. Round 0 reads the sorted pairs and gathers the
// points (signs applied); later rounds read the previous round's points. The
// bucket layout of a round is its list of bucket ends (an inclusive scan of
// the halved counts). After the last round, the short lists go through the
// XYZZ run and merge levels as (bucket, entry) pairs.
//
// The sharing is per block and pipelined. Warps 0..6 are workers: in a batch
// each worker thread chains the denominators of its k output entries into one
// running product, and the workers' products are combined by prefix and
// suffix products across lanes (shuffles) and across warps. Warp 7 inverts the
// batch's product (one exponentiation, a few hundred dependent products) while
// the workers walk the previous batch's chains back with the inverse it
// produced one iteration earlier; so the exponentiation's latency overlaps the
// additions instead of stalling them. Blocks are persistent: block b takes
// batches b, b + gridDim.x, ... of 224 k output entries.
//
// Special cases, decided when the denominator is formed (the case travels to
// the backward walk in `meta`): equal x and equal y is a doubling (the
// denominator is 2y); equal x otherwise (P + (-P)) gives the point at infinity;
// an operand at infinity (bit 255 of x set) makes the result the other
// operand. Those cases put 1 into the chain, so no zero reaches an inversion.

static constexpr int kAffThreads = 256;
static constexpr int kAffWorkerWarps = 7;
static constexpr int kAffWorkers = kAffWorkerWarps * 32;
static constexpr uint32_t kAffAdd = 0, kAffDbl = 1, kAffInf = 2, kAffCopy1 = 3, kAffCopy2 = 4;

__device__ __forceinline__ void aff_store_inf(uint64_t* dst) {
  uint32_t z[8];
  fe_zero(z);
  fe_store(dst + 4, z);
  z[7] = 0x80000000u;
  fe_store(dst, z);
}

// half[b] = ceil(n_b / 2), n_b = ends[b] - ends[b - 1] (ends[-1] = 0).
__global__ void __launch_bounds__(256) k_msm_half_counts(const uint32_t* ends, int keys, uint32_t* half) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < keys; b += stride) {
    const uint32_t n = ends[b] - (b ? ends[b - 1] : 0u);
    half[b] = (n + 1u) >> 1;
  }
}

// The bucket holding output entry e: the first b with ends[b] > e.
__device__ __forceinline__ int bucket_of_entry(const uint32_t* ends, int keys, uint32_t e) {
  int lo = 0, hi = keys - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ends[mid] > e) hi = mid; else lo = mid + 1;
  }
  return lo;
}

__device__ __forceinline__ void shfl_up8(uint32_t r[8], const uint32_t a[8], int o) {
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = __shfl_up_sync(0xffffffffu, a[j], o);
}
__device__ __forceinline__ void shfl_down8(uint32_t r[8], const uint32_t a[8], int o) {
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = __shfl_down_sync(0xffffffffu, a[j], o);
}

// Exclusive prefix and suffix products of v across the warp's lanes (1 at the ends).
template <class M>
__device__ __forceinline__ void warp_exclusive_products(uint32_t xp[8], uint32_t xs[8], const uint32_t v[8],
                                                        int lane) {
  G1F f;
  uint32_t pre[8], suf[8], t[8];
  fe_copy(pre, v);
  fe_copy(suf, v);
#pragma unroll 1
  for (int o = 1; o < 32; o <<= 1) {
    shfl_up8(t, pre, o);
    if (lane >= o) M::mul(pre, pre, t);
    shfl_down8(t, suf, o);
    if (lane + o < 32) M::mul(suf, suf, t);
  }
  shfl_up8(xp, pre, 1);
  shfl_down8(xs, suf, 1);
  if (lane == 0) fe_one(xp, f);
  if (lane == 31) fe_one(xs, f);
}

// An entry's two source rows, as the forward walk resolves them and the
// backward walk reads them back from `meta`: the row addresses with the sign
// of the y coordinate in bit 0 (rows are 64-byte aligned) and the entry's case
// in bits 1..3 of the first.
struct AffMeta {
  uint64_t a, b;
};

__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ const uint64_t* meta_row(uint64_t v) {
  return reinterpret_cast<const uint64_t*>(v & ~(uint64_t)15);
}

__device__ __forceinline__ void load_row(Aff& p, uint64_t v) {
  aff_load(p, meta_row(v));
  if (v & 1) aff_neg(p);
}

template <bool kFirst, class M>
__global__ void __launch_bounds__(kAffThreads, 2) k_msm_affine_round(
    const MsmJobs J, const uint2* pairs, const uint64_t* in_pts, const uint32_t* in_ends,
    const uint32_t* out_ends, int keys, int k, uint64_t* out_pts, uint64_t* scratch, AffMeta* meta,
    uint2* out_pairs) {
  G1F f;
  __shared__ uint32_t s_wtot[3][kAffWorkerWarps][8];
  __shared__ uint32_t s_wpre[3][kAffWorkerWarps][8], s_wsuf[3][kAffWorkerWarps][8];
  __shared__ uint32_t s_inv[3][8];
  __shared__ uint32_t s_others[3][kAffWorkers][8];  // per worker: the product of its warp's other chains
  const uint32_t total = out_ends[keys - 1];
  const int64_t per_batch = (int64_t)kAffWorkers * k;
  // batches of this block: b, b + G, ... while their first entry is below total (uniform in the block)
  int64_t nb = 0;
  if ((int64_t)blockIdx.x * per_batch < (int64_t)total) {
    nb = ((int64_t)total - (int64_t)blockIdx.x * per_batch + (int64_t)gridDim.x * per_batch - 1) /
         ((int64_t)gridDim.x * per_batch);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool worker = w < kAffWorkerWarps;
  const int wi = worker ? (int)threadIdx.x : 0;
  const int64_t nw_grid = (int64_t)gridDim.x * kAffWorkers;
  const int64_t gw = (int64_t)blockIdx.x * kAffWorkers + wi;
  auto first_entry = [&](int64_t batch) { return (batch * gridDim.x + blockIdx.x) * per_batch + (int64_t)wi * k; };
  auto count_of = [&](int64_t e0) {
    return e0 < (int64_t)total ? (int)min((int64_t)k, (int64_t)total - e0) : 0;
  };
  // the source rows of output entry e (bucket walk from *b)
  auto resolve = [&](uint32_t e, int* b, AffMeta* m, bool* pair) {
    while (out_ends[*b] <= e) ++*b;
    const uint32_t ostart = *b ? out_ends[*b - 1] : 0u;
    const uint32_t istart = *b ? in_ends[*b - 1] : 0u;
    const uint32_t in = istart + 2u * (e - ostart);
    *pair = in + 1u < in_ends[*b];
    if (kFirst) {
      const uint2 kv1 = pairs[in];
      const JobPoints jp = job_points(J, kv1.x);
      const int64_t i1 = (int64_t)(kv1.y & 0x7fffffffu);
      m->a = reinterpret_cast<uint64_t>(i1 < jp.n ? jp.points + 8 * i1 : jp.phi + 8 * (i1 - jp.n)) | (kv1.y >> 31);
      m->b = 0;
      if (*pair) {
        const uint2 kv2 = pairs[in + 1u];
        const int64_t i2 = (int64_t)(kv2.y & 0x7fffffffu);
        m->b = reinterpret_cast<uint64_t>(i2 < jp.n ? jp.points + 8 * i2 : jp.phi + 8 * (i2 - jp.n)) | (kv2.y >> 31);
      }
    } else {
      m->a = reinterpret_cast<uint64_t>(in_pts + 8 * (int64_t)in);
      m->b = *pair ? m->a + 64 : 0;
    }
  };

  int64_t e0_1 = 0, e0_2 = 0;  // first entries of batches t - 1 and t - 2
  int cnt_1 = 0, cnt_2 = 0;
  uint32_t acc[8];

  for (int64_t t = 0; t <= nb + 1; ++t) {
    const int qf = (int)(t % 3), qb = (int)((t + 1) % 3), qi = (int)((t + 2) % 3);  // batches t, t - 2, t - 1
    if (worker) {
      const bool fwd = t < nb, bwd = t >= 2 && cnt_2 > 0;
      const int64_t e0 = fwd ? first_entry(t) : 0;
      const int n_f = fwd ? count_of(e0) : 0;
      const int n_b = bwd ? cnt_2 : 0;
      uint64_t* fscr = scratch + 4 * (int64_t)qf * k * nw_grid;
      AffMeta* fmet = meta + (int64_t)qf * k * nw_grid;
      const uint64_t* bscr = scratch + 4 * (int64_t)qb * k * nw_grid;
      const AffMeta* bmet = meta + (int64_t)qb * k * nw_grid;
      fe_one(acc, f);
      uint32_t inv[8];
      if (n_b > 0) {
        M::mul(inv, s_inv[qb], s_wpre[qb][w]);
        M::mul(inv, inv, s_wsuf[qb][w]);
        M::mul(inv, inv, s_others[qb][wi]);  // = 1 / (this thread's chain of batch t - 2)
      }
      // forward look-ahead: entry 0 resolved and its rows on their way to L2
      int fb = n_f > 0 ? bucket_of_entry(out_ends, keys, (uint32_t)e0) : 0;
      AffMeta fm{0, 0};
      bool fpair = false;
      if (n_f > 0) {
        resolve((uint32_t)e0, &fb, &fm, &fpair);
        prefetch_l2(meta_row(fm.a));
        if (fpair) prefetch_l2(meta_row(fm.b));
      }
      AffMeta bm{0, 0};
      if (n_b > 0) {
        bm = bmet[(int64_t)(n_b - 1) * nw_grid + gw];
        prefetch_l2(meta_row(bm.a));
        if (bm.b) prefetch_l2(meta_row(bm.b));
      }
      const int steps = n_f > n_b ? n_f : n_b;
      for (int i = 0; i < steps; ++i) {
        // ---- forward entry i: its x coordinates start loading now ----
        uint32_t x1[8], x2[8];
        const AffMeta cur = fm;
        const bool cur_pair = fpair;
        const int cur_b = fb;  // entry i's bucket (fb moves on to entry i + 1's below)
        if (i < n_f) {
          fe_load(x1, meta_row(cur.a));
          if (cur_pair) fe_load(x2, meta_row(cur.b));
          if (i + 1 < n_f) {  // resolve entry i + 1 and prefetch its rows
            resolve((uint32_t)(e0 + i + 1), &fb, &fm, &fpair);
            prefetch_l2(meta_row(fm.a));
            if (fpair) prefetch_l2(meta_row(fm.b));
          }
        }
        // ---- backward entry n_b - 1 - i of batch t - 2 ----
        if (i < n_b) {
          const int bi = n_b - 1 - i;
          const AffMeta m = bm;
          if (bi > 0) {
            bm = bmet[(int64_t)(bi - 1) * nw_grid + gw];
            prefetch_l2(meta_row(bm.a));
            if (bm.b) prefetch_l2(meta_row(bm.b));
          }
          const uint32_t cs = (uint32_t)(m.a >> 1) & 7u;
          uint64_t* dst = out_pts + 8 * (e0_2 + bi);
          if (cs == kAffInf) {
            aff_store_inf(dst);
          } else if (cs == kAffCopy1 || cs == kAffCopy2) {
            Aff p;
            load_row(p, cs == kAffCopy1 ? m.a : m.b);
            fe_store(dst, p.x);
            fe_store(dst + 4, p.y);
          } else {
            uint32_t inv_i[8];
            if (bi > 0) {
              uint32_t prev[8];
              fe_load(prev, bscr + 4 * ((int64_t)(bi - 1) * nw_grid + gw));
              M::mul(inv_i, inv, prev);
            } else {
              fe_copy(inv_i, inv);
            }
            Aff p1, p2;
            load_row(p1, m.a);
            uint32_t d[8], lam[8], x3[8], y3[8];
            if (cs == kAffAdd) {
              load_row(p2, m.b);
              fe_sub(d, p2.x, p1.x, f);
              fe_sub(lam, p2.y, p1.y, f);
            } else {
              fe_dbl(d, p1.y, f);
              M::sqr(lam, p1.x);
              uint32_t t2[8];
              fe_dbl(t2, lam, f);
              fe_add(lam, lam, t2, f);  // 3 x1^2
              fe_copy(p2.x, p1.x);
            }
            if (bi > 0) M::mul(inv, inv, d);  // now 1 / (the chain before entry bi)
            M::mul(lam, lam, inv_i);
            M::sqr(x3, lam);
            fe_sub(x3, x3, p1.x, f);
            fe_sub(x3, x3, p2.x, f);
            fe_sub(y3, p1.x, x3, f);
            M::mul(y3, lam, y3);
            fe_sub(y3, y3, p1.y, f);
            fe_store(dst, x3);
            fe_store(dst + 4, y3);
          }
        }
        // ---- forward entry i: its denominator joins the chain ----
        if (i < n_f) {
          uint32_t d[8], cs;
          if (!cur_pair) {
            fe_one(d, f);
            cs = kAffCopy1;
          } else {
            const bool i1 = (x1[7] >> 31) != 0, i2 = (x2[7] >> 31) != 0;
            if (i1 || i2) {
              fe_one(d, f);
              cs = i1 && i2 ? kAffInf : (i1 ? kAffCopy2 : kAffCopy1);
            } else {
              fe_sub(d, x2, x1, f);
              cs = kAffAdd;
              if (fe_is_zero(d)) {
                Aff q1, q2;
                load_row(q1, cur.a);
                load_row(q2, cur.b);
                if (fe_eq(q1.y, q2.y) && !fe_is_zero(q1.y)) {
                  fe_dbl(d, q1.y, f);
                  cs = kAffDbl;
                } else {
                  fe_one(d, f);
                  cs = kAffInf;
                }
              }
            }
          }
          if (i == 0) {
            fe_copy(acc, d);
          } else {
            M::mul(acc, acc, d);
          }
          fe_store(fscr + 4 * ((int64_t)i * nw_grid + gw), acc);
          fmet[(int64_t)i * nw_grid + gw] = AffMeta{cur.a | ((uint64_t)cs << 1), cur.b};
          if (out_pairs) out_pairs[e0 + i] = make_uint2((uint32_t)cur_b, (uint32_t)(e0 + i));
        }
      }
      // the forward chain's place among the block's chains (every worker lane joins)
      if (fwd) {
        uint32_t xp[8], xs[8], o[8];
        warp_exclusive_products<M>(xp, xs, acc, lane);
        M::mul(o, xp, xs);
        fe_copy(s_others[qf][wi], o);
        if (lane == 31) {
          uint32_t tot[8];
          M::mul(tot, xp, acc);
          fe_copy(s_wtot[qf][w], tot);
        }
      }
      e0_2 = e0_1;
      cnt_2 = cnt_1;
      e0_1 = e0;
      cnt_1 = n_f;
    } else if (t >= 1 && t <= nb) {
      // ---- warp 7: combine the worker warps of batch t - 1 and invert it ----
      uint32_t v[8], xp[8], xs[8];
      if (lane < kAffWorkerWarps) {
        fe_copy(v, s_wtot[qi][lane]);
      } else {
        fe_one(v, f);
      }
      warp_exclusive_products<M>(xp, xs, v, lane);
      if (lane < kAffWorkerWarps) {
        fe_copy(s_wpre[qi][lane], xp);
        fe_copy(s_wsuf[qi][lane], xs);
      }
      uint32_t tot[8], inv[8];
      M::mul(tot, xp, v);  // lane 6: the product of all seven warps
#pragma unroll
      for (int c = 0; c < 8; ++c) tot[c] = __shfl_sync(0xffffffffu, tot[c], kAffWorkerWarps - 1);
      fe_inv(inv, tot, f);  // never zero: every factor is nonzero
      if (lane == 0) fe_copy(s_inv[qi], inv);
    }
    __syncthreads();
  }
}

// Levels 2+: K2 slots per thread, full XYZZ additions; slots without a key
// (none) may sit anywhere between runs and are skipped.
template <class Mul>
__global__ void __launch_bounds__(128) k_msm_acc_slots(const uint32_t* in_keys,
                                                       const uint64_t* in_pts, int64_t M, int K,
                                                       uint32_t none, uint64_t* buckets,
                                                       uint32_t* slot_keys, uint64_t* slot_pts) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t T = (M + K - 1) / K;
  if (t >= T) return;
  const int64_t start = t * K;
  const int64_t end = start + K < M ? start + K : M;
  RunSink sink{buckets, slot_keys, slot_pts, t, start > 0 ? in_keys[start - 1] : none,
               end < M ? in_keys[end] : none, none};
  slot_keys[2 * t] = none;
  slot_keys[2 * t + 1] = none;
  uint32_t cur = in_keys[start];
  bool first = true;
  Xyzz acc;
  xyzz_set_identity(acc);
  for (int64_t e = start; e < end; ++e) {
    const uint32_t k = in_keys[e];
    if (k != cur) {
      sink.flush(cur, acc, first, false);
      first = false;
      xyzz_set_identity(acc);
      cur = k;
    }
    if (k == none) continue;
    Xyzz q;
    xyzz_load(q, in_pts + 16 * e);
    xyzz_add<Mul>(acc, acc, q);
  }
  sink.flush(cur, acc, first, true);
}

// ---------------------------------------------------------------------------
// 4. window reduction
// ---------------------------------------------------------------------------

// sum_b (b + 1) B_b per window, in levels. A level's items are pairs
// (A_i, T_i): T_i is the sum of the buckets item i covers, scaled by D (the
// buckets an item covers), and A_i their sum weighted 1, 2, ... from the
// item's first bucket. Level 1's items are the buckets themselves (A = T = B,
// D = 1). One warp takes a chunk of 32 L consecutive items of one window, L
// per lane:
//   lane t, items j = 0..L-1:  R_t = sum_j T_j,  V_t = sum_j A_j + sum_j j T_j
//       (running sums from the top: two additions an item, three above level 1)
//   chunk:  A = sum_t V_t + L sum_t t R_t,  T = 32 L sum_t R_t
// and sum_t t R_t = sum_(t >= 1) SR_t with SR_t = sum_(u >= t) R_u, a suffix
// scan across the lanes (five shuffled additions), then a tree sum of
// Y_t = V_t + L SR_t (five more). The chunk's pair is the next level's item;
// a level with one chunk per window writes the window sums. Per bucket that is
// 2 + (11 + log2 L) / L XYZZ operations at level 1, and two or three levels
// in all.
__device__ __forceinline__ void shfl_down_xyzz(Xyzz& r, const Xyzz& a, int o) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    r.x[j] = __shfl_down_sync(0xffffffffu, a.x[j], o);
    r.y[j] = __shfl_down_sync(0xffffffffu, a.y[j], o);
    r.zz[j] = __shfl_down_sync(0xffffffffu, a.zz[j], o);
    r.zzz[j] = __shfl_down_sync(0xffffffffu, a.zzz[j], o);
  }
}

// A_in / T_in are [W][G_in] (T_in null at level 1: the buckets are both); a
// warp per (window, chunk), chunks_per_window chunks of 32 << lL items. Out:
// [W][chunks_per_window] pairs, or (T_out null) the window sums.
template <class Mul>
__global__ void __launch_bounds__(128) k_msm_reduce(const uint64_t* A_in, const uint64_t* T_in,
                                                    int64_t G_in, int lL, int64_t chunks_per_window,
                                                    int64_t total_chunks, uint64_t* A_out,
                                                    uint64_t* T_out) {
  const int64_t chunk = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (chunk >= total_chunks) return;  // whole warps: the shuffles below see all 32 lanes
  const int64_t win = chunk / chunks_per_window;
  const int64_t c = chunk - win * chunks_per_window;
  const int L = 1 << lL;
  const int64_t first = (c * 32 + lane) * (int64_t)L;
  const uint64_t* A = A_in + 16 * win * G_in;
  const uint64_t* T = T_in ? T_in + 16 * win * G_in : nullptr;
  Xyzz run, tot, x;
  xyzz_set_identity(run);
  xyzz_set_identity(tot);
  for (int k = L - 1; k >= 0; --k) {
    const int64_t i = first + k;
    if (i < G_in) {
      xyzz_load(x, (T ? T : A) + 16 * i);
      xyzz_add<Mul>(run, run, x);
      if (T) {
        xyzz_load(x, A + 16 * i);
        xyzz_add<Mul>(tot, tot, x);
      }
    }
    if (k > 0 || !T) xyzz_add<Mul>(tot, tot, run);  // level 1: weights 1..L, else 0..L-1 on T
  }
  // run = R_t, tot = V_t. Suffix scan: run becomes SR_t.
#pragma unroll 1
  for (int o = 1; o < 32; o <<= 1) {
    shfl_down_xyzz(x, run, o);
    if (lane + o < 32) xyzz_add<Mul>(run, run, x);
  }
  if (lane > 0) {  // Y_t = V_t + L SR_t (lane 0 keeps SR_0, the chunk's total)
    Xyzz sr = run;
    for (int k = 0; k < lL; ++k) xyzz_dbl<Mul>(sr, sr);
    xyzz_add<Mul>(tot, tot, sr);
  }
#pragma unroll 1
  for (int o = 16; o > 0; o >>= 1) {
    shfl_down_xyzz(x, tot, o);
    if (lane < o) xyzz_add<Mul>(tot, tot, x);
  }
  if (lane == 0) {
    xyzz_store(A_out + 16 * chunk, tot);
    if (T_out) {
      for (int k = 0; k < 5 + lL; ++k) xyzz_dbl<Mul>(run, run);
      xyzz_store(T_out + 16 * chunk, run);
    }
  }
}

// ---------------------------------------------------------------------------
// 5. finalize
// ---------------------------------------------------------------------------

// One thread per job. Horner from the top window: acc = 2^w acc + S_win, the w
// doublings in Jacobian coordinates (7 products each against 9 in XYZZ; the
// conversions cost 6 a window), the additions in XYZZ; then affine
// x = X / ZZ, y = Y / ZZZ with one inversion of ZZ ZZZ, as plain canonical
// values.
template <class Mul>
__global__ void k_msm_finalize(const MsmJobs J, const uint64_t* all_window_sums, int W, int w) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= J.count) return;
  const uint64_t* window_sums = all_window_sums + 16 * (int64_t)j * W;
  uint64_t* result = J.result[j];
  G1F f;
  Xyzz acc, s;
  xyzz_load(acc, window_sums + 16 * (W - 1));
  for (int win = W - 2; win >= 0; --win) {
    Jac j;
    xyzz_to_jac<Mul>(j, acc);
    for (int k = 0; k < w; ++k) jac_dbl_m<Mul>(j, j);
    jac_to_xyzz<Mul>(acc, j);
    xyzz_load(s, window_sums + 16 * win);
    xyzz_add<Mul>(acc, acc, s);
  }
  uint32_t x[8], y[8];
  uint64_t flag = 0;
  if (xyzz_is_identity(acc)) {
    fe_zero(x);
    fe_zero(y);
    flag = 1;
  } else {
    uint32_t prod[8], inv[8], t[8];
    fe_mul(prod, acc.zz, acc.zzz, f);
    fe_inv(inv, prod, f);
    fe_mul(t, inv, acc.zzz, f);  // 1 / ZZ
    fe_mul(x, acc.x, t, f);
    fe_mul(t, inv, acc.zz, f);   // 1 / ZZZ
    fe_mul(y, acc.y, t, f);
    fe_from_mont(x, x, f);
    fe_from_mont(y, y, f);
  }
  // 8-byte stores: the result buffer only has to be 8-byte aligned
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    result[j] = (uint64_t)x[2 * j] | ((uint64_t)x[2 * j + 1] << 32);
    result[4 + j] = (uint64_t)y[2 * j] | ((uint64_t)y[2 * j + 1] << 32);
  }
  result[8] = flag;
}

__global__ void k_msm_identity_result(uint64_t* result) {
  for (int k = 0; k < 8; ++k) result[k] = 0;
  result[8] = 1;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

int default_window(int64_t n) {
  // argmin over w of windows * (cost of the 2n GLV-half mixed additions +
  // 2^(w-1) buckets' share of the reduction), in units of field
  // multiplications: 10 per mixed addition, about 42 per bucket in the
  // running sums.
  if (n <= 1) return 1;
  int log_n = 0;
  while ((1ll << log_n) < n) ++log_n;
  const int tuned = tune_get_sized("msm.window", log_n);  // a measured table's entry
  if (tuned > 0) return tuned;
  int best_w = 1;
  double best = 1e300;
  for (int w = 1; w <= 16; ++w) {
    const double cost =
        (double)num_windows(w) * (20.0 * (double)n + 42.0 * (double)(1ll << (w - 1)));
    if (cost < best) {
      best = cost;
      best_w = w;
    }
  }
  return best_w;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct MsmPlan {
  int count = 1;                // jobs in the batch (all at window w)
  std::vector<int64_t> first;   // prefix sums of the jobs' point counts
  int64_t n = 0;                // points of all jobs
  int w = 0, W = 0, key_bits = 0;
  uint32_t none = 0;
  int64_t nb = 0;  // buckets per window
  int k1 = 64;     // sorted pairs per bucket thread ("msm.pairs_per_thread", else by size)
  int k2 = 8;      // slots per merge thread ("msm.slots_per_thread")
  int log_l = 4;   // log2 of the buckets a lane sums in reduction level 1 ("msm.reduce_log_segment")
  int call_products = 1;  // bucket kernels call one shared product ("msm.call_products")
  int counting_sort = 1;  // counting sort (1) or radix sort (0) of the pairs ("msm.sort")
  int table = 0;          // points are fixed-base tables: one bucket set per job
  int64_t windows = 0;    // bucket sets of the batch: count W, or count with tables
  int64_t keys_used = 0;  // bucket keys of the batch (count * W * 2^(w-1))
  int64_t E = 0;   // sorted pairs
  int aff_rounds = 0;               // affine rounds before the XYZZ levels ("msm.affine_rounds")
  int aff_k = 64;                   // output entries per thread of an affine round ("msm.affine_batch")
  std::vector<int64_t> aff_bound;   // bound on each round's list: aff_bound[0] = E, then per round
  int64_t E_list = 0;               // entries the XYZZ levels start from (E, or the last round's bound)
  int64_t T1 = 0;  // level-1 threads
  std::vector<int64_t> slot_levels;  // thread count of each merge level
  size_t cub_bytes = 0;
  // workspace offsets
  size_t off_keys0, off_keys1, off_vals0, off_vals1, off_cub, off_phi, off_buckets,
      off_slot_keys_a, off_slot_pts_a, off_slot_keys_b, off_slot_pts_b, off_red_s0, off_red_u0,
      off_red_s1, off_red_u1, off_wsum, off_counts, off_offsets, off_aff_ends0, off_aff_ends1,
      off_aff_half, off_aff_pts0, off_aff_pts1, off_aff_scratch, off_aff_meta, total;
};

// Blocks of an affine round over a list of `entries`: persistent, at most two per
// SM (their register budget), and no more than the batches of 224 k entries.
static int64_t aff_blocks(int64_t entries, int k) {
  const int64_t per = (int64_t)kAffWorkers * k;
  return std::max<int64_t>(1, std::min<int64_t>((entries + per - 1) / per, 2 * 148));
}

// The longest automatic run of sorted pairs a bucket thread takes in a one-MSM
// call ("msm.call_pairs_cap", default 16; batches go up to 64). A bucket block
// then lasts about 0.5 ms instead of 2 ms at 2^22 points, so kernels the caller
// runs beside the MSM on other streams (a transform of higher priority) wait at
// most that long for an SM at each of their launches. Measured on B200, the
// bench's end-to-end step (two one-call MSMs beside two transforms and their
// copies): 47.3 to 44.3 ms; the one-call MSM 2^22 alone 18.06 to 18.29 ms.
static int single_call_pairs_cap() { return tune_get("msm.call_pairs_cap"); }

// Plan for a batch of jobs with point counts sizes[0..count) at window w.
static int make_plan(const int64_t* sizes, int count, int w, MsmPlan& p, int table = 0, int k1 = 0,
                     int log_l = 0, int k1_cap = 64) {
  p.count = count;
  p.first.assign(count + 1, 0);
  for (int j = 0; j < count; ++j) p.first[j + 1] = p.first[j] + sizes[j];
  const int64_t n = p.first[count];
  p.n = n;
  p.w = w;
  p.W = num_windows(w);
  p.nb = 1ll << (w - 1);
  p.table = table;
  p.windows = table ? count : (int64_t)count * p.W;
  const int64_t keys_used = p.windows * p.nb;
  int bits = 1;
  while ((1ll << bits) <= keys_used) ++bits;  // keys_used itself must fit below none
  p.key_bits = bits;
  p.none = (uint32_t)((1ull << bits) - 1);
  p.keys_used = keys_used;
  p.counting_sort = table ? 1 : tune_get("msm.sort");
  p.E = 2 * (int64_t)p.W * n;  // both GLV halves
  // Affine rounds (counting sort only: they start from its bucket ends). By
  // default a round runs while its list still fills every SM with two blocks of
  // full batches; "msm.affine_rounds" > 0 forces that many at any size, 0 turns
  // them off. A round's list has at most sum ceil(n_b / 2) <= B / 2 + keys / 2
  // entries.
  p.aff_k = tune_get("msm.affine_batch");
  const int forced = tune_get("msm.affine_rounds");
  p.aff_bound.assign(1, p.E);
  if (p.counting_sort && forced != 0) {
    const int64_t min_out = (int64_t)2 * 148 * kAffWorkers * p.aff_k;
    for (int r = 0; r < 8; ++r) {
      const int64_t b = p.aff_bound.back();
      const int64_t nb = std::min(b, (b + 1) / 2 + (keys_used + 1) / 2);
      if (forced > 0 ? r >= forced : nb < min_out) break;
      p.aff_bound.push_back(nb);
    }
  }
  p.aff_rounds = (int)p.aff_bound.size() - 1;
  p.E_list = p.aff_bound.back();
  // pairs per level-1 thread: the knob, else by size. A thread adds its pairs one
  // after another, so small MSMs want short chains and many threads; each thread
  // may leave two partial sums for the merge levels, so large ones want long
  // chains. E / 2^19 rounded down to a power of two, within 8..64: measured on
  // B200 (uniform scalars, default windows), 8 pairs against 64 take 2^10 points
  // from 1.89 to 1.56 ms, 2^14 from 2.07 to 1.79, 2^16 from 2.36 to 2.14; from
  // 2^19 points 16-32 pairs match 64 (skewed scalars gain 5-12 %), and 2^21 up
  // keeps 64.
  p.k1 = k1 > 0 ? k1 : tune_get("msm.pairs_per_thread");
  if (p.k1 < 8) {
    p.k1 = 8;
    while (p.k1 < k1_cap && ((int64_t)p.k1 << 20) <= p.E_list) p.k1 <<= 1;
  }
  p.k2 = tune_get("msm.slots_per_thread");
  p.log_l = log_l > 0 ? log_l : tune_get("msm.reduce_log_segment");
  p.call_products = tune_get("msm.call_products");
  p.T1 = (p.E_list + p.k1 - 1) / p.k1;
  p.slot_levels.clear();
  int64_t M = 2 * p.T1;
  int64_t T = p.T1;
  while (T > 1) {
    T = (M + p.k2 - 1) / p.k2;
    p.slot_levels.push_back(T);
    M = 2 * T;
  }
  // CUB's temporary storage for sorting E pairs (a size query; launches nothing)
  cub::DoubleBuffer<uint32_t> kb(nullptr, nullptr), vb(nullptr, nullptr);
  size_t cub_bytes = 0;
  cudaError_t err = cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, kb, vb, (int)p.E, 0,
                                                    p.key_bits, (cudaStream_t)0);
  if (err != cudaSuccess) return check_cuda(err, "CUB sort size query");
  size_t scan_bytes = 0;
  err = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                      (int)(keys_used + 1), (cudaStream_t)0);
  if (err != cudaSuccess) return check_cuda(err, "CUB scan size query");
  p.cub_bytes = cub_bytes > scan_bytes ? cub_bytes : scan_bytes;
  if (p.aff_rounds > 0) {
    size_t incl_bytes = 0;
    err = cub::DeviceScan::InclusiveSum(nullptr, incl_bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                        (int)keys_used, (cudaStream_t)0);
    if (err != cudaSuccess) return check_cuda(err, "CUB scan size query");
    p.cub_bytes = std::max(p.cub_bytes, incl_bytes);
  }

  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t at = off;
    off += align256(bytes);
    return at;
  };
  p.off_keys0 = take((size_t)p.E * 4);
  p.off_keys1 = take((size_t)p.E * 4);
  p.off_vals0 = take((size_t)p.E * 4);
  p.off_vals1 = take((size_t)p.E * 4);
  p.off_cub = take(p.cub_bytes);
  p.off_phi = take(table ? 0 : (size_t)n * 64);
  const int64_t windows = p.windows;
  p.off_buckets = take((size_t)windows * p.nb * 128);
  p.off_slot_keys_a = take((size_t)2 * p.T1 * 4);
  p.off_slot_pts_a = take((size_t)2 * p.T1 * 128);
  const int64_t second = p.slot_levels.empty() ? 1 : p.slot_levels[0];
  p.off_slot_keys_b = take((size_t)2 * second * 4);
  p.off_slot_pts_b = take((size_t)2 * second * 128);
  const int64_t red = windows * (p.nb >> p.log_l > 0 ? p.nb >> p.log_l : 1);
  p.off_red_s0 = take((size_t)red * 128);
  p.off_red_u0 = take((size_t)red * 128);
  p.off_red_s1 = take((size_t)red * 128);
  p.off_red_u1 = take((size_t)red * 128);
  p.off_wsum = take((size_t)windows * 128);
  // counting sort: per-key counts, then offsets / cursors (one more entry: the total)
  p.off_counts = take((size_t)(keys_used + 1) * 4);
  p.off_offsets = take((size_t)(keys_used + 1) * 4);
  // affine rounds: two bucket-end arrays and the halved counts, two point lists
  // (rounds alternate), and the per-entry chain prefixes and cases of the
  // largest round (round 0)
  const bool aff = p.aff_rounds > 0;
  p.off_aff_ends0 = take(aff ? (size_t)keys_used * 4 : 0);
  p.off_aff_ends1 = take(aff ? (size_t)keys_used * 4 : 0);
  p.off_aff_half = take(aff ? (size_t)keys_used * 4 : 0);
  p.off_aff_pts0 = take(aff ? (size_t)p.aff_bound[1] * 64 : 0);
  p.off_aff_pts1 = take(p.aff_rounds >= 2 ? (size_t)p.aff_bound[2] * 64 : 0);
  // three batches in flight per worker thread (one being chained, one being
  // inverted, one being walked back): 3 k chain prefixes and source records each
  const int64_t aff_entries = aff ? 3 * aff_blocks(p.aff_bound[1], p.aff_k) * kAffWorkers * p.aff_k : 0;
  p.off_aff_scratch = take((size_t)aff_entries * 32);
  p.off_aff_meta = take((size_t)aff_entries * 16);
  p.total = off;
  return ZKB_OK;
}

// The kernel-parameter job table of a planned batch.
static MsmJobs job_table(const MsmPlan& p, const uint64_t* const* points,
                         const uint64_t* const* scalars, uint64_t* const* results, char* ws) {
  MsmJobs J;
  std::memset(&J, 0, sizeof J);
  J.count = p.count;
  J.keys_per_job = (uint32_t)(p.windows / p.count * p.nb);
  uint64_t* phi = reinterpret_cast<uint64_t*>(ws + p.off_phi);
  for (int j = 0; j <= p.count; ++j) J.first[j] = p.first[j];
  for (int j = 0; j < p.count; ++j) {
    J.points[j] = points[j];
    J.scalars[j] = scalars[j];
    J.result[j] = results[j];
    J.phi[j] = p.table ? nullptr : phi + 8 * p.first[j];
    J.pts_n[j] = (p.first[j + 1] - p.first[j]) * (p.table ? 2 * p.W : 1);
  }
  return J;
}

static int run_msm(const MsmJobs& J, const MsmPlan& p, char* ws, cudaStream_t s) {
  uint32_t* keys0 = reinterpret_cast<uint32_t*>(ws + p.off_keys0);
  uint32_t* keys1 = reinterpret_cast<uint32_t*>(ws + p.off_keys1);
  uint32_t* vals0 = reinterpret_cast<uint32_t*>(ws + p.off_vals0);
  uint32_t* vals1 = reinterpret_cast<uint32_t*>(ws + p.off_vals1);
  uint64_t* buckets = reinterpret_cast<uint64_t*>(ws + p.off_buckets);
  const int64_t windows = p.windows;

  // 1-2. digits (GLV halves), grouped by bucket; the phi images of the points
  const uint32_t* skeys = keys1;
  const uint32_t* svals = vals1;
  int st = 1;
  const uint32_t* e_dev = nullptr;  // pairs written by the counting sort (device)
  const uint64_t* list_pts = nullptr;  // after affine rounds: the points the final list indexes
  if (p.counting_sort) {
    uint32_t* counts = reinterpret_cast<uint32_t*>(ws + p.off_counts);
    uint32_t* offsets = reinterpret_cast<uint32_t*>(ws + p.off_offsets);
    {
      ProfSpan span("msm_digits", s);
      ZKB_TRY(check_cuda(cudaMemsetAsync(counts, 0, (size_t)(p.keys_used + 1) * 4, s), "msm count reset"));
      k_msm_bucket_digits<false><<<grid_for(p.n, 256), 256, 0, s>>>(J, p.w, p.W, p.none, p.table, counts,
                                                                     nullptr);
      ZKB_TRY(check_launch("msm digit count"));
      if (!p.table) {
        k_msm_phi<<<grid_for(p.n, 256), 256, 0, s>>>(J);
        ZKB_TRY(check_launch("msm phi points"));
      }
    }
    ProfSpan span("msm_sort", s);
    size_t scan_bytes = p.cub_bytes;
    ZKB_TRY(check_cuda(cub::DeviceScan::ExclusiveSum(ws + p.off_cub, scan_bytes, counts, offsets,
                                                     (int)(p.keys_used + 1), s),
                       "msm bucket offsets"));
    // offsets[keys_used] = the pair count; no key reaches it, so it survives the scatter
    // the interleaved (key, value) words take the space of keys0 and keys1 (2 x 4 E bytes)
    uint2* pairs = reinterpret_cast<uint2*>(keys0);
    k_msm_bucket_digits<true><<<grid_for(p.n, 256), 256, 0, s>>>(J, p.w, p.W, p.none, p.table, offsets,
                                                                  pairs);
    ZKB_TRY(check_launch("msm digit scatter"));
    e_dev = offsets + p.keys_used;
    skeys = keys0;
    svals = keys0 + 1;
    st = 2;
    if (p.aff_rounds > 0) {
      // after the scatter, offsets[b] is the end of bucket b's pairs
      ProfSpan aspan("msm_affine_rounds", s);
      const int keys = (int)p.keys_used;
      const uint32_t* in_ends = offsets;
      const uint64_t* in_pts = nullptr;
      uint32_t* ends[2] = {reinterpret_cast<uint32_t*>(ws + p.off_aff_ends0),
                           reinterpret_cast<uint32_t*>(ws + p.off_aff_ends1)};
      uint64_t* pts[2] = {reinterpret_cast<uint64_t*>(ws + p.off_aff_pts0),
                          reinterpret_cast<uint64_t*>(ws + p.off_aff_pts1)};
      uint32_t* half = reinterpret_cast<uint32_t*>(ws + p.off_aff_half);
      uint64_t* scratch = reinterpret_cast<uint64_t*>(ws + p.off_aff_scratch);
      AffMeta* meta = reinterpret_cast<AffMeta*>(ws + p.off_aff_meta);
      // the final list's (bucket, entry) pairs take the space of the unused value arrays
      uint2* final_pairs = reinterpret_cast<uint2*>(ws + p.off_vals0);
      for (int r = 0; r < p.aff_rounds; ++r) {
        uint32_t* out_ends = ends[r & 1];
        k_msm_half_counts<<<grid_for(keys, 256), 256, 0, s>>>(in_ends, keys, half);
        ZKB_TRY(check_launch("msm affine round counts"));
        size_t scan_bytes2 = p.cub_bytes;
        ZKB_TRY(check_cuda(cub::DeviceScan::InclusiveSum(ws + p.off_cub, scan_bytes2, half, out_ends, keys, s),
                           "msm affine round layout"));
        const int64_t blocks = aff_blocks(p.aff_bound[r + 1], p.aff_k);
        uint2* op = r + 1 == p.aff_rounds ? final_pairs : nullptr;
        if (r == 0) {
          auto kern = p.call_products ? k_msm_affine_round<true, CallMul> : k_msm_affine_round<true, InlineMul>;
          kern<<<(unsigned)blocks, kAffThreads, 0, s>>>(J, pairs, in_pts, in_ends, out_ends, keys, p.aff_k, pts[0],
                                                         scratch, meta, op);
        } else {
          auto kern = p.call_products ? k_msm_affine_round<false, CallMul> : k_msm_affine_round<false, InlineMul>;
          kern<<<(unsigned)blocks, kAffThreads, 0, s>>>(J, nullptr, in_pts, in_ends, out_ends, keys, p.aff_k,
                                                         pts[r & 1], scratch, meta, op);
        }
        ZKB_TRY(check_launch("msm affine round"));
        in_ends = out_ends;
        in_pts = pts[r & 1];
      }
      // the XYZZ levels take the last round's points as one point array
      list_pts = in_pts;
      skeys = reinterpret_cast<const uint32_t*>(final_pairs);
      svals = skeys + 1;
      e_dev = in_ends + keys - 1;
    }
  } else {
    {
      ProfSpan span("msm_digits", s);
      k_msm_digits<<<grid_for(p.n, 256), 256, 0, s>>>(J, p.w, p.W, p.none, keys0, vals0);
      ZKB_TRY(check_launch("msm digits"));
      k_msm_phi<<<grid_for(p.n, 256), 256, 0, s>>>(J);
      ZKB_TRY(check_launch("msm phi points"));
    }
    cub::DoubleBuffer<uint32_t> kb(keys0, keys1), vb(vals0, vals1);
    size_t cub_bytes = p.cub_bytes;
    ProfSpan span("msm_sort", s);
    ZKB_TRY(check_cuda(cub::DeviceRadixSort::SortPairs(ws + p.off_cub, cub_bytes, kb, vb, (int)p.E,
                                                       0, p.key_bits, s),
                       "msm sort"));
    skeys = kb.Current();
    svals = vb.Current();
  }

  // 3. buckets
  const int64_t nbuckets = windows * p.nb;
  k_xyzz_fill_identity<<<grid_for(nbuckets, 256), 256, 0, s>>>(buckets, nbuckets);
  ZKB_TRY(check_launch("msm bucket init"));
  uint32_t* sk[2] = {reinterpret_cast<uint32_t*>(ws + p.off_slot_keys_a),
                     reinterpret_cast<uint32_t*>(ws + p.off_slot_keys_b)};
  uint64_t* sp[2] = {reinterpret_cast<uint64_t*>(ws + p.off_slot_pts_a),
                     reinterpret_cast<uint64_t*>(ws + p.off_slot_pts_b)};
  {
    ProfSpan span("msm_acc_points", s);
    const unsigned grid = (unsigned)((p.T1 + 127) / 128);
    if (list_pts) {
      // one point array for every job: the one-job kernel over a job table whose
      // only entry is that array
      MsmJobs L = J;
      L.count = 1;
      L.points[0] = list_pts;
      L.phi[0] = nullptr;
      L.pts_n[0] = INT64_MAX;
      auto kern = p.call_products ? k_msm_acc_points<CallMul> : k_msm_acc_points<InlineMul>;
      kern<<<grid, 128, 0, s>>>(L, skeys, svals, st, p.E_list, e_dev, p.k1, p.none, buckets, sk[0], sp[0]);
    } else if (p.count > 1) {
      auto kern = p.call_products ? k_msm_acc_points_batch<CallMul> : k_msm_acc_points_batch<InlineMul>;
      kern<<<grid, 128, 0, s>>>(J, skeys, svals, st, p.E, e_dev, p.k1, p.none, buckets, sk[0], sp[0]);
    } else {
      auto kern = p.call_products ? k_msm_acc_points<CallMul> : k_msm_acc_points<InlineMul>;
      kern<<<grid, 128, 0, s>>>(J, skeys, svals, st, p.E, e_dev, p.k1, p.none, buckets, sk[0], sp[0]);
    }
    ZKB_TRY(check_launch("msm bucket accumulation"));
  }
  {
    ProfSpan span("msm_acc_merge", s);
    int cur = 0;
    int64_t M = 2 * p.T1;
    for (size_t lvl = 0; lvl < p.slot_levels.size(); ++lvl) {
      const int64_t T = p.slot_levels[lvl];
      const unsigned grid = (unsigned)((T + 127) / 128);
      auto kern = p.call_products ? k_msm_acc_slots<CallMul> : k_msm_acc_slots<InlineMul>;
      kern<<<grid, 128, 0, s>>>(sk[cur], sp[cur], M, p.k2, p.none, buckets,
                                           sk[cur ^ 1], sp[cur ^ 1]);
      ZKB_TRY(check_launch("msm bucket merge"));
      cur ^= 1;
      M = 2 * T;
    }
  }

  // 4. window reduction
  uint64_t* rs[2] = {reinterpret_cast<uint64_t*>(ws + p.off_red_s0),
                     reinterpret_cast<uint64_t*>(ws + p.off_red_s1)};
  uint64_t* ru[2] = {reinterpret_cast<uint64_t*>(ws + p.off_red_u0),
                     reinterpret_cast<uint64_t*>(ws + p.off_red_u1)};
  uint64_t* wsum = reinterpret_cast<uint64_t*>(ws + p.off_wsum);
  {
    ProfSpan span("msm_reduce", s);
    auto red = p.call_products ? k_msm_reduce<CallMul> : k_msm_reduce<InlineMul>;
    const uint64_t* A = buckets;
    const uint64_t* T = nullptr;
    int64_t G = p.nb;
    int lL = p.log_l, r = 0;
    for (;;) {
      const int64_t per = (int64_t)32 << lL;
      const int64_t chunks = (G + per - 1) / per;
      const bool last = chunks == 1;
      const int64_t total = windows * chunks;
      red<<<(unsigned)((total * 32 + 127) / 128), 128, 0, s>>>(A, T, G, lL, chunks, total,
                                                                last ? wsum : rs[r], last ? nullptr : ru[r]);
      ZKB_TRY(check_launch(last ? "msm window sums" : "msm window reduction"));
      if (last) break;
      A = rs[r];
      T = ru[r];
      r ^= 1;
      G = chunks;
      // the next level: the fewest items a lane that finish the window, at most 16
      lL = 0;
      while (lL < 4 && ((int64_t)32 << lL) < G) ++lL;
    }
  }

  // 5. finalize
  ProfSpan fin_span("msm_finalize", s);
  auto fin = p.call_products ? k_msm_finalize<CallMul> : k_msm_finalize<InlineMul>;
  // with tables there is one window sum per job: nothing to combine
  fin<<<1, p.count < 32 ? 32 : p.count, 0, s>>>(J, wsum, p.table ? 1 : p.W, p.w);
  return check_launch("msm finalize");
}

// ---- batches of jobs --------------------------------------------------------

// Jobs with the same window share one pipeline run (a chunk), at most
// kMsmMaxBatch jobs and 2^31 sorted pairs per chunk; chunks run concurrently
// on side streams, each in its own slice of the workspace.
struct MsmChunk {
  int w = 0;
  std::vector<int> jobs;  // indices into the caller's job array
  MsmPlan plan;
  size_t offset = 0;
};

static int validate_job(const zkb_msm_job& j, int index, int table) {
  if (j.n < 0) return fail(ZKB_EINVAL, "job %d: negative point count", index);
  if (j.n >= (1ll << 30)) return fail(ZKB_EINVAL, "job %d: at most 2^30 - 1 points per MSM", index);
  if (!table && (j.window_size < 0 || j.window_size > kMsmMaxWindow)) {
    return fail(ZKB_EINVAL, "job %d: window_size must be in 1..%d (or 0 for the default), got %d",
                index, kMsmMaxWindow, j.window_size);
  }
  if (!j.result) return fail(ZKB_EINVAL, "job %d: null result buffer", index);
  ZKB_TRY(check_align(j.result, 8, "result"));
  if (j.n == 0) return ZKB_OK;
  if (!j.points || !j.scalars) return fail(ZKB_EINVAL, "job %d: null buffer", index);
  ZKB_TRY(check_align(j.points, 16, "points"));
  ZKB_TRY(check_align(j.scalars, 16, "scalars"));
  return ZKB_OK;
}

static int plan_batch(const zkb_msm_job* jobs, int count, std::vector<MsmChunk>& chunks,
                      size_t& total, int table = 0) {
  chunks.clear();
  total = 0;
  if (count < 0) return fail(ZKB_EINVAL, "negative job count");
  if (count > 0 && !jobs) return fail(ZKB_EINVAL, "null job array");
  std::vector<int> order;
  for (int i = 0; i < count; ++i) {
    ZKB_TRY(validate_job(jobs[i], i, table));
    if (table && (jobs[i].window_size < kTableMinWindow || jobs[i].window_size > kTableMaxWindow)) {
      return fail(ZKB_EINVAL, "job %d: a fixed-base table's window must be %d..%d, got %d", i,
                  kTableMinWindow, kTableMaxWindow, jobs[i].window_size);
    }
    if (jobs[i].n > 0) order.push_back(i);
  }
  auto window_of = [&](int i) {
    return jobs[i].window_size ? jobs[i].window_size : default_window(jobs[i].n);
  };
  // by window, then by size (largest first) so each chunk's sort stays in range
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const int wa = window_of(a), wb = window_of(b);
    return wa != wb ? wa < wb : jobs[a].n > jobs[b].n;
  });
  for (int i : order) {
    const int w = window_of(i);
    const int64_t pairs = 2 * (int64_t)num_windows(w) * jobs[i].n;
    if (pairs >= (1ll << 31)) {
      return fail(ZKB_EINVAL, "%lld points at window %d exceed the sort's 2^31 pairs",
                  (long long)jobs[i].n, w);
    }
    bool fits = !chunks.empty() && chunks.back().w == w &&
                (int)chunks.back().jobs.size() < kMsmMaxBatch;
    if (fits) {
      int64_t cur = 0;
      for (int k : chunks.back().jobs) cur += 2 * (int64_t)num_windows(w) * jobs[k].n;
      fits = cur + pairs < (1ll << 31);
    }
    if (!fits) {
      chunks.emplace_back();
      chunks.back().w = w;
    }
    chunks.back().jobs.push_back(i);
  }
  for (auto& c : chunks) {
    std::vector<int64_t> sizes;
    for (int k : c.jobs) sizes.push_back(jobs[k].n);
    ZKB_TRY(make_plan(sizes.data(), (int)sizes.size(), c.w, c.plan, table));
    c.offset = total;
    total += align256(c.plan.total);
  }
  return ZKB_OK;
}

// One MSM through the batch pipeline.
static int run_single(const uint64_t* points, const uint64_t* scalars, uint64_t* result,
                      const MsmPlan& p, char* ws, cudaStream_t s) {
  const MsmJobs J = job_table(p, &points, &scalars, &result, ws);
  return run_msm(J, p, ws, s);
}

// A batch of MSM jobs (zkb_msm_batch), or of MSMs over fixed-base tables.
int msm_batch(const zkb_msm_job* jobs, int count, void* workspace, size_t workspace_bytes, void* stream,
              int table);

}  // namespace zkb

using namespace zkb;

extern "C" {

int zkb_msm_default_window(int64_t n) { return zkb::default_window(n); }

size_t zkb_msm_workspace_bytes(int64_t n, int window_size) {
  set_error("%s", "");
  if (n <= 0) return 0;
  const int w = window_size ? window_size : default_window(n);
  if (w < 1 || w > kMsmMaxWindow) return 0;
  MsmPlan p;
  if (make_plan(&n, 1, w, p, 0, 0, 0, single_call_pairs_cap()) != ZKB_OK) return 0;
  return p.total;
}

int zkb_msm(const uint64_t* points, const uint64_t* scalars, int64_t n, int window_size,
            uint64_t* result, void* workspace, size_t workspace_bytes, void* stream) {
  set_error("%s", "");
  if (n < 0) return fail(ZKB_EINVAL, "negative point count");
  if (n >= (1ll << 30)) return fail(ZKB_EINVAL, "at most 2^30 - 1 points per MSM");
  if (window_size < 0 || window_size > kMsmMaxWindow) {
    return fail(ZKB_EINVAL, "window_size must be in 1..%d (or 0 for the default), got %d",
                kMsmMaxWindow, window_size);
  }
  if (!result) return fail(ZKB_EINVAL, "null result buffer");
  ZKB_TRY(check_align(result, 8, "result"));
  cudaStream_t s = as_stream(stream);
  if (n == 0) {
    k_msm_identity_result<<<1, 1, 0, s>>>(result);
    return check_launch("msm identity");
  }
  if (!points || !scalars) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(points, 16, "points"));
  ZKB_TRY(check_align(scalars, 16, "scalars"));
  ZKB_TRY(check_align(workspace, 256, "workspace"));
  const int w = window_size ? window_size : default_window(n);
  MsmPlan p;
  ZKB_TRY(make_plan(&n, 1, w, p, 0, 0, 0, single_call_pairs_cap()));
  if ((int64_t)p.E >= (1ll << 31)) {
    return fail(ZKB_EINVAL, "%lld points at window %d exceed the sort's 2^31 pairs",
                (long long)n, w);
  }
  if (!workspace || workspace_bytes < p.total) {
    return fail(ZKB_EWORKSPACE, "MSM of %lld points at window %d needs %zu workspace bytes, got %zu",
                (long long)n, w, p.total, workspace_bytes);
  }
  return run_single(points, scalars, result, p, reinterpret_cast<char*>(workspace), s);
}

size_t zkb_msm_batch_workspace_bytes(const zkb_msm_job* jobs, int count) {
  set_error("%s", "");
  std::vector<MsmChunk> chunks;
  size_t total = 0;
  if (plan_batch(jobs, count, chunks, total) != ZKB_OK) return 0;
  return total;
}

int zkb_msm_batch(const zkb_msm_job* jobs, int count, void* workspace, size_t workspace_bytes,
                  void* stream) {
  return zkb::msm_batch(jobs, count, workspace, workspace_bytes, stream, 0);
}

size_t zkb_msm_table_bytes(int64_t n, int window_size) {
  if (n <= 0 || window_size < kTableMinWindow || window_size > kTableMaxWindow) return 0;
  return (size_t)n * 2 * num_windows(window_size) * 64;
}

int zkb_msm_table_build(const uint64_t* points, int64_t n, int window_size, uint64_t* table,
                        void* stream) {
  set_error("%s", "");
  if (window_size < kTableMinWindow || window_size > kTableMaxWindow) {
    return fail(ZKB_EINVAL, "a fixed-base table's window must be %d..%d, got %d", kTableMinWindow,
                kTableMaxWindow, window_size);
  }
  const int W = num_windows(window_size);
  if (n < 0 || n >= (1ll << 30) || 2 * (int64_t)W * n >= (1ll << 31)) {
    return fail(ZKB_EINVAL, "%lld points do not fit a table at window %d", (long long)n, window_size);
  }
  if (n == 0) return ZKB_OK;
  if (!points || !table) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(points, 16, "points"));
  ZKB_TRY(check_align(table, 16, "table"));
  k_msm_table_build<<<(unsigned)((n + 127) / 128), 128, 0, as_stream(stream)>>>(points, n, window_size, W,
                                                                                 table);
  return check_launch("msm fixed-base table");
}

size_t zkb_msm_fixed_batch_workspace_bytes(const zkb_msm_job* jobs, int count) {
  set_error("%s", "");
  std::vector<MsmChunk> chunks;
  size_t total = 0;
  if (plan_batch(jobs, count, chunks, total, 1) != ZKB_OK) return 0;
  return total;
}

int zkb_msm_fixed_batch(const zkb_msm_job* jobs, int count, void* workspace, size_t workspace_bytes,
                        void* stream) {
  return zkb::msm_batch(jobs, count, workspace, workspace_bytes, stream, 1);
}

}  // extern "C"

namespace zkb {

int msm_batch(const zkb_msm_job* jobs, int count, void* workspace, size_t workspace_bytes, void* stream,
              int table) {
  set_error("%s", "");
  std::vector<MsmChunk> chunks;
  size_t total = 0;
  ZKB_TRY(plan_batch(jobs, count, chunks, total, table));
  if (total > 0) {
    ZKB_TRY(check_align(workspace, 256, "workspace"));
    if (!workspace || workspace_bytes < total) {
      return fail(ZKB_EWORKSPACE, "MSM batch of %d jobs needs %zu workspace bytes, got %zu", count,
                  total, workspace_bytes);
    }
  }
  cudaStream_t s = as_stream(stream);
  for (int i = 0; i < count; ++i) {
    if (jobs[i].n == 0) {
      k_msm_identity_result<<<1, 1, 0, s>>>(jobs[i].result);
      ZKB_TRY(check_launch("msm identity"));
    }
  }
  auto run_chunk = [&](const MsmChunk& c, cudaStream_t cs) {
    std::vector<const uint64_t*> pts, scs;
    std::vector<uint64_t*> res;
    for (int k : c.jobs) {
      pts.push_back(jobs[k].points);
      scs.push_back(jobs[k].scalars);
      res.push_back(jobs[k].result);
    }
    char* ws = reinterpret_cast<char*>(workspace) + c.offset;
    const MsmJobs J = job_table(c.plan, pts.data(), scs.data(), res.data(), ws);
    return run_msm(J, c.plan, ws, cs);
  };
  if (chunks.size() == 1) return run_chunk(chunks[0], s);
  if (chunks.empty()) return ZKB_OK;
  Fanout fan;
  const int sides = (int)std::min<size_t>(chunks.size(), Fanout::kMaxSides);
  ZKB_TRY(fan.fork(s, sides));
  for (size_t c = 0; c < chunks.size(); ++c) {
    const int rc = run_chunk(chunks[c], fan.side((int)c));
    if (rc != ZKB_OK) {
      fan.join(s);
      return rc;
    }
  }
  return fan.join(s);
}

}  // namespace zkb

extern "C" {

}  // extern "C"

// ---------------------------------------------------------------------------
// MSM without any allocation: scratch in a fixed device array
// ---------------------------------------------------------------------------
//
// zkb_msm takes its scratch memory from the caller. Some callers have no way
// to hand over device memory at call time: a plugin running inside another
// framework whose device memory is all reserved up front by that framework's
// own allocator, or a latency-critical serving loop that must never reach
// cudaMalloc (which can synchronise the whole device and stall every other
// stream). zkb_msm_no_alloc serves them: it runs the very same MSM pipeline on
// a scratch array that is part of the library itself.
//
// The array below is a file-scope device variable: every GPU on which the
// library is loaded holds these 64 MiB until the process exits, whether or
// not the entry point is ever called. That is enough scratch for 2^16 points
// at the default window; larger problems are refused with ZKB_EWORKSPACE.
// All calls share the one array per device, so two calls whose work overlaps
// on the GPU (different streams, or different host threads) corrupt each
// other's results: callers must order them, for example on one stream.
// Every buffer the pipeline reads is fully rewritten by the call itself (the
// buckets are reset to the identity, every key and slot is written before it
// is read), so a call never depends on what the previous one left behind.

namespace zkb {

static constexpr size_t kNoAllocScratchBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_msm_static_scratch[kNoAllocScratchBytes];
// The sort's key and value arrays take 16 bytes per digit pair, so no plan that
// fits the array can reach the 2^31 pairs the sort indexes (checked again below).
static_assert(kNoAllocScratchBytes < (1ull << 31) * 16, "the fixed scratch could hold 2^31 sort pairs");

// Device address of g_msm_static_scratch for the current device and context.
// In host code the array's name is only a host-side stand-in; the address a
// kernel may use comes from cudaGetSymbolAddress with the device current. It is
// looked up on every call (a table lookup in the runtime, no allocation) rather
// than cached per device index: after cudaDeviceReset, or under another context
// on the same device, a cached address would point into a module that no longer
// exists. The first lookup on a device also loads the library's module there.
static int static_scratch_address(void** out) {
  void* ptr = nullptr;
  ZKB_TRY(check_cuda(cudaGetSymbolAddress(&ptr, g_msm_static_scratch),
                     "cudaGetSymbolAddress(static MSM scratch)"));
  if (!ptr) return fail(ZKB_ECUDA, "cudaGetSymbolAddress returned no address for the static MSM scratch");
  *out = ptr;
  return ZKB_OK;
}

}  // namespace zkb

extern "C" {

size_t zkb_msm_no_alloc_capacity(void) { return zkb::kNoAllocScratchBytes; }

int zkb_msm_no_alloc(const uint64_t* points, const uint64_t* scalars, int64_t n, int window_size,
                     uint64_t* result, void* stream) {
  set_error("%s", "");
  if (n < 0) return fail(ZKB_EINVAL, "negative point count");
  if (n >= (1ll << 30)) return fail(ZKB_EINVAL, "at most 2^30 - 1 points per MSM");
  if (window_size < 0 || window_size > kMsmMaxWindow) {
    return fail(ZKB_EINVAL, "window_size must be in 1..%d (or 0 for the default), got %d",
                kMsmMaxWindow, window_size);
  }
  if (!result) return fail(ZKB_EINVAL, "null result buffer");
  ZKB_TRY(check_align(result, 8, "result"));
  cudaStream_t s = as_stream(stream);
  if (n == 0) {
    k_msm_identity_result<<<1, 1, 0, s>>>(result);
    return check_launch("msm identity");
  }
  if (!points || !scalars) return fail(ZKB_EINVAL, "null buffer");
  ZKB_TRY(check_align(points, 16, "points"));
  ZKB_TRY(check_align(scalars, 16, "scalars"));
  const int w = window_size ? window_size : default_window(n);
  MsmPlan p;
  ZKB_TRY(make_plan(&n, 1, w, p, 0, 0, 0, single_call_pairs_cap()));
  // short bucket chains and short first-level reduction runs, which suit small
  // MSMs, take more scratch: when the plan does not fit the fixed scratch, the
  // compact shape (at least 64 pairs per thread, at least 4 buckets a lane) may
  if (p.total > kNoAllocScratchBytes && (p.k1 < 64 || p.log_l < 2)) {
    ZKB_TRY(make_plan(&n, 1, w, p, 0, p.k1 > 64 ? p.k1 : 64, p.log_l > 2 ? p.log_l : 2));
  }
  if (p.total > kNoAllocScratchBytes) {
    return fail(ZKB_EWORKSPACE,
                "MSM of %lld points at window %d needs %zu bytes of scratch; the library's fixed "
                "scratch holds %zu bytes (use zkb_msm with a caller-provided workspace)",
                (long long)n, w, p.total, kNoAllocScratchBytes);
  }
  if ((int64_t)p.E >= (1ll << 31)) {
    return fail(ZKB_EINVAL, "%lld points at window %d exceed the sort's 2^31 pairs", (long long)n, w);
  }
  void* scratch = nullptr;
  ZKB_TRY(static_scratch_address(&scratch));
  return run_single(points, scalars, result, p, reinterpret_cast<char*>(scratch), s);
}

}  // extern "C"
