// runtime.cu — error reporting, version, and the host side of field set-up.
#include <atomic>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "field_host.h"
#include "tma.cuh"

namespace zkb {

static thread_local char g_last_error[1024] = "";
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ---- tuning knobs -----------------------------------------------------------
// name, default, min, max. Read by the planners at each call, so a change
// applies to the next call (and to the workspace size queries).
struct Knob {
  const char* name;
  int value, lo, hi;
};
static Knob g_knobs[] = {
    {"msm.pairs_per_thread", 0, 0, 4096},    // sorted pairs each bucket thread adds (8..4096; 0 = by size)
    {"msm.slots_per_thread", 8, 4, 4096},    // partial sums each merge thread adds
    {"msm.reduce_log_segment", 4, 0, 8},     // log2 of the buckets a lane sums in the first reduction level
    {"msm.call_pairs_cap", 16, 8, 64},       // longest automatic bucket run of a one-MSM call
    {"msm.call_products", 1, 0, 1},          // bucket kernels call one shared product (1) or inline all (0)
    {"msm.sort", 1, 0, 1},                   // pairs grouped by a counting sort (1) or a radix sort (0)
    {"msm.affine_rounds", 0, -1, 8},         // affine rounds before the XYZZ levels (0 = none, -1 = by size)
    {"msm.affine_batch", 64, 8, 512},        // output entries per thread of an affine round
    {"ntt.max_log_radix", 0, 0, 12},         // largest sub-transform per pass (log2, 8..12; 0 = by size)
    {"ntt.cta_log_elems", 0, 0, 12},         // elements staged per CTA (log2, 9..12; 0 = by size)
    {"ntt.threads", 0, 0, 512},              // threads per NTT CTA (64..512; 0 = by tile)
    {"ntt.call_products", 0, 0, 1},          // pass kernels call one shared product (1) or inline all (0)
    {"ntt.full_table_mb", 4096, 0, 65536},   // budget of expanded NTT tables (MiB; 0 = two-level only)
    {"ntt.batch_spin_limit", 0, 0, 1 << 30},  // polls before a batch tile's dependency wait gives up (0 = 2^22)
    {"ntt.tma", 1, 0, 1},                    // multi-pass transforms: TMA-fed persistent passes (1) or per-thread gathers (0)
    {"ntt.lazy", 1, 0, 1},                   // TMA passes: values in [0, 2p) between butterfly rounds (p < 2^254)
    {"ntt.tma_grid", 1, 0, 1},               // TMA passes: one persistent wave (0) or one tile per block (1)
    {"ntt.tma_blocks_per_sm", 0, 0, 6},      // TMA passes of 128-thread blocks: registers capped for 5 or 6 blocks (0 = no cap)
    {"ntt64.first_col_log", -1, -1, 6},      // int64 NTT first pass: log2 of input words per row (-1 = by size)
    {"ntt64.first_max_k", 0, 0, 10},         // int64 NTT first pass: stages (4..10; 0 = by size)
    {"ntt64.col_log", 0, 0, 6},              // int64 NTT later passes: log2 of words per row (1..6; 0 = by size)
    {"ntt64.max_k", 0, 0, 10},               // int64 NTT later passes: most stages (2..10; 0 = by size)
};
static std::mutex g_knob_mutex;

static Knob* find_knob(const char* key) {
  if (!key) return nullptr;
  for (auto& k : g_knobs)
    if (std::strcmp(k.name, key) == 0) return &k;
  return nullptr;
}

int tune_get(const char* key) {
  std::lock_guard<std::mutex> lock(g_knob_mutex);
  Knob* k = find_knob(key);
  return k ? k->value : 0;
}

// ---- per-size tuning tables ---------------------------------------------------
// Choices that depend on the problem size, set per log2 size (an autotuner's
// measured table); 0 = no entry, the planner's own rule applies.
struct SizedKnob {
  const char* name;
  int lo, hi;
  int value[kMaxSizedLog + 1];
};
static SizedKnob g_sized[] = {
    {"msm.window", 1, 20, {}},          // MSM window for ceil(log2 n) = log
    {"ntt.max_log_radix", 8, 12, {}},   // largest pass radix for an NTT of 2^log rows
    {"ntt.cta_log_elems", 9, 12, {}},   // rows per NTT block
    {"ntt.threads", 64, 512, {}},       // threads per NTT block
};

static SizedKnob* find_sized(const char* key) {
  if (!key) return nullptr;
  for (auto& k : g_sized)
    if (std::strcmp(k.name, key) == 0) return &k;
  return nullptr;
}

int tune_get_sized(const char* key, int log_n) {
  if (log_n < 0 || log_n > kMaxSizedLog) return 0;
  std::lock_guard<std::mutex> lock(g_knob_mutex);
  SizedKnob* k = find_sized(key);
  return k ? k->value[log_n] : 0;
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof g_last_error, fmt, ap);
  va_end(ap);
}

// ---- 256-bit host helpers (little-endian uint64 limbs) ----------------------

static bool u256_ge(const uint64_t a[4], const uint64_t b[4]) {
  for (int j = 3; j >= 0; --j) {
    if (a[j] != b[j]) return a[j] > b[j];
  }
  return true;
}

static void u256_sub(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]) {
  unsigned __int128 borrow = 0;
  for (int j = 0; j < 4; ++j) {
    unsigned __int128 d = (unsigned __int128)a[j] - b[j] - borrow;
    r[j] = (uint64_t)d;
    borrow = (d >> 64) ? 1 : 0;
  }
}

// r = 2r mod p for r < p < 2^255 (2r < 2^256, no fifth limb needed).
static void u256_double_mod(uint64_t r[4], const uint64_t p[4]) {
  uint64_t carry = 0;
  for (int j = 0; j < 4; ++j) {
    uint64_t next = r[j] >> 63;
    r[j] = (r[j] << 1) | carry;
    carry = next;
  }
  if (u256_ge(r, p)) u256_sub(r, r, p);
}

static const uint64_t kBn254R[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull,
                                    0xb85045b68181585dull, 0x30644e72e131a029ull};
static const uint64_t kBn254P[4] = {0x3c208c16d87cfd47ull, 0x97816a916871ca8dull,
                                    0xb85045b68181585dull, 0x30644e72e131a029ull};

int field_init(zkb_field* f, const uint64_t modulus[4]) {
  if (!f || !modulus) return fail(ZKB_EINVAL, "zkb_field_init: null pointer");
  // odd and in [3, 2^255) (zkgpu/field256_gpu.py:278-280)
  bool small = modulus[3] == 0 && modulus[2] == 0 && modulus[1] == 0 && modulus[0] < 3;
  if ((modulus[0] & 1) == 0 || small || (modulus[3] >> 63) != 0) {
    return fail(ZKB_EINVAL, "modulus must be odd and in [3, 2^255)");
  }
  std::memset(f, 0, sizeof *f);
  std::memcpy(f->modulus, modulus, sizeof f->modulus);
  // R mod p: 1 doubled 256 times; R^2 mod p: 256 more doublings.
  uint64_t r[4] = {1, 0, 0, 0};
  if (u256_ge(r, modulus)) u256_sub(r, r, modulus);
  for (int i = 0; i < 256; ++i) u256_double_mod(r, modulus);
  std::memcpy(f->one, r, sizeof r);
  for (int i = 0; i < 256; ++i) u256_double_mod(r, modulus);
  std::memcpy(f->r2, r, sizeof r);
  // p^-1 mod 2^64 by Newton's iteration (each step doubles the correct bits;
  // x = p is already correct to 3 bits for odd p), then negate.
  uint64_t x = modulus[0];
  for (int i = 0; i < 6; ++i) x *= 2 - modulus[0] * x;
  f->ninv = (uint64_t)0 - x;
  if (std::memcmp(modulus, kBn254R, sizeof kBn254R) == 0) {
    f->kind = ZKB_FIELD_BN254_FR;
  } else if (std::memcmp(modulus, kBn254P, sizeof kBn254P) == 0) {
    f->kind = ZKB_FIELD_BN254_FQ;
  } else {
    f->kind = ZKB_FIELD_GENERIC;
  }
  return ZKB_OK;
}

FieldRT to_rt(const zkb_field& f) {
  FieldRT rt;
  for (int j = 0; j < 4; ++j) {
    rt.P[2 * j] = (uint32_t)f.modulus[j];
    rt.P[2 * j + 1] = (uint32_t)(f.modulus[j] >> 32);
    rt.ONE[2 * j] = (uint32_t)f.one[j];
    rt.ONE[2 * j + 1] = (uint32_t)(f.one[j] >> 32);
    rt.R2[2 * j] = (uint32_t)f.r2[j];
    rt.R2[2 * j + 1] = (uint32_t)(f.r2[j] >> 32);
  }
  rt.NINV = (uint32_t)f.ninv;
  return rt;
}

int check_field(const zkb_field* f) {
  if (!f) return fail(ZKB_EINVAL, "null field");
  if (f->kind != ZKB_FIELD_GENERIC && f->kind != ZKB_FIELD_BN254_FR && f->kind != ZKB_FIELD_BN254_FQ) {
    return fail(ZKB_EINVAL, "field not initialised by zkb_field_init");
  }
  return ZKB_OK;
}

// ---- tensor maps --------------------------------------------------------------
// cuTensorMapEncodeTiled is a driver entry point; the runtime hands out its
// address, so the library needs no link against the driver library.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess) {
      fn = reinterpret_cast<EncodeTiledFn>(p);
    }
  });
  return fn;
}

int encode_tensor_map_u64(CUtensorMap* map, const void* base, int rank, const uint64_t* dims,
                          const uint64_t* strides_bytes, const uint32_t* box) {
  EncodeTiledFn fn = encode_tiled_fn();
  if (!fn) return fail(ZKB_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
  if (rank < 2 || rank > 5) return fail(ZKB_EINVAL, "tensor map rank %d out of 2..5", rank);
  if (reinterpret_cast<uintptr_t>(base) & 15) return fail(ZKB_EINVAL, "tensor map base must be 16-byte aligned");
  cuuint64_t gdim[5], gstride[4];
  cuuint32_t bdim[5], estride[5];
  for (int i = 0; i < rank; ++i) {
    gdim[i] = dims[i];
    bdim[i] = box[i];
    estride[i] = 1;
    if (box[i] < 1 || box[i] > 256 || box[i] > dims[i]) {
      return fail(ZKB_EINVAL, "tensor map box dimension %d (%u) out of range", i, box[i]);
    }
  }
  if ((box[0] * 8u) % 16u) return fail(ZKB_EINVAL, "tensor map box inner extent must be a multiple of 16 bytes");
  for (int i = 0; i + 1 < rank; ++i) {
    gstride[i] = strides_bytes[i];
    if (strides_bytes[i] % 16) return fail(ZKB_EINVAL, "tensor map stride %d not a multiple of 16 bytes", i);
  }
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, (cuuint32_t)rank, const_cast<void*>(base), gdim,
                        gstride, bdim, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ZKB_ECUDA, "cuTensorMapEncodeTiled failed (CUresult %d)", (int)r);
  return ZKB_OK;
}

}  // namespace zkb

extern "C" {

const char* zkb_last_error(void) { return zkb::g_last_error; }

int zkb_version(void) { return 100; }

uint64_t zkb_launch_count(void) { return zkb::g_launches.load(); }

int zkb_tune_set(const char* key, int value) {
  zkb::set_error("%s", "");
  std::lock_guard<std::mutex> lock(zkb::g_knob_mutex);
  zkb::Knob* k = zkb::find_knob(key);
  if (!k) return zkb::fail(ZKB_EINVAL, "unknown tuning knob '%s'", key ? key : "(null)");
  if (value < k->lo || value > k->hi) {
    return zkb::fail(ZKB_EINVAL, "%s must be in %d..%d, got %d", k->name, k->lo, k->hi, value);
  }
  k->value = value;
  return ZKB_OK;
}

int zkb_tune_set_sized(const char* key, int log_n, int value) {
  zkb::set_error("%s", "");
  std::lock_guard<std::mutex> lock(zkb::g_knob_mutex);
  zkb::SizedKnob* k = zkb::find_sized(key);
  if (!k) return zkb::fail(ZKB_EINVAL, "unknown per-size tuning table '%s'", key ? key : "(null)");
  if (log_n < 0 || log_n > zkb::kMaxSizedLog) {
    return zkb::fail(ZKB_EINVAL, "log2 size must be in 0..%d, got %d", zkb::kMaxSizedLog, log_n);
  }
  if (value != 0 && (value < k->lo || value > k->hi)) {
    return zkb::fail(ZKB_EINVAL, "%s must be 0 (no entry) or in %d..%d, got %d", k->name, k->lo, k->hi,
                     value);
  }
  k->value[log_n] = value;
  return ZKB_OK;
}

int zkb_tune_get_sized(const char* key, int log_n, int* value) {
  zkb::set_error("%s", "");
  std::lock_guard<std::mutex> lock(zkb::g_knob_mutex);
  zkb::SizedKnob* k = zkb::find_sized(key);
  if (!k || !value) return zkb::fail(ZKB_EINVAL, "unknown per-size tuning table '%s'", key ? key : "(null)");
  if (log_n < 0 || log_n > zkb::kMaxSizedLog) {
    return zkb::fail(ZKB_EINVAL, "log2 size must be in 0..%d, got %d", zkb::kMaxSizedLog, log_n);
  }
  *value = k->value[log_n];
  return ZKB_OK;
}

int zkb_tune_get(const char* key, int* value) {
  zkb::set_error("%s", "");
  std::lock_guard<std::mutex> lock(zkb::g_knob_mutex);
  zkb::Knob* k = zkb::find_knob(key);
  if (!k || !value) return zkb::fail(ZKB_EINVAL, "unknown tuning knob '%s'", key ? key : "(null)");
  *value = k->value;
  return ZKB_OK;
}

int zkb_field_init(zkb_field* f, const uint64_t modulus[4]) {
  zkb::set_error("%s", "");
  return zkb::field_init(f, modulus);
}

}  // extern "C"
