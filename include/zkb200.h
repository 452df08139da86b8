/*
 * zkb200.h — C ABI of libzkb200.so, the B200 (sm_100a) BN254 prover hot path.
 *
 * Every buffer argument is a DEVICE pointer unless stated otherwise; `stream`
 * is a cudaStream_t (NULL = the legacy default stream). Calls are
 * stream-ordered and return as soon as the work is queued; a result is ready
 * once the stream has reached it. Every call returns ZKB_OK or an error code
 * and leaves a message for zkb_last_error() (thread-local).
 *
 * Data layout (the reference's, zkgpu/field256_gpu.py:12-20 and
 * zkgpu/curve_gpu.py:15-26):
 *   field element  4 x uint64, little-endian limbs, Montgomery form a*2^256 mod p,
 *                  canonical (< p); 32 bytes per row.
 *   Jacobian point (X, Y, Z), 3 field elements (96 bytes); Z = 0 is the identity,
 *                  stored as (ONE, ONE, 0).
 *   affine point   (x, y), 2 field elements (64 bytes); never the identity.
 *
 * Each entry point below names the reference interface it replaces. The
 * reference has no native FFI: its GPU path launches CuPy RawKernels from
 * Python, so these functions take the place of those launches together with
 * the host-side argument handling around them.
 */
#ifndef ZKB200_H
#define ZKB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define ZKB_OK 0
#define ZKB_EINVAL 1      /* bad argument value (Python: ValueError) */
#define ZKB_ETYPE 2       /* bad buffer shape or type (Python: TypeError) */
#define ZKB_ECUDA 3       /* CUDA error (Python: RuntimeError) */
#define ZKB_ENOTONCURVE 4 /* an input point is not on y^2 = x^3 + 3 (ValueError) */
#define ZKB_EWORKSPACE 5  /* workspace too small (ValueError) */
#define ZKB_ETIMEOUT 6    /* a bounded device wait gave up (RuntimeError) */

/* Message of the last failing call on this thread ("" if none). */
const char* zkb_last_error(void);

/* ABI version of this library (major * 100 + minor). */
int zkb_version(void);

/* ---- fields --------------------------------------------------------------- */

/* A prime field's Montgomery parameters. Plain data: filled by zkb_field_init,
 * copied by value, never freed. */
typedef struct zkb_field {
  uint64_t modulus[4]; /* p, odd, 3 <= p < 2^255 */
  uint64_t one[4];     /* R mod p, R = 2^256 (Montgomery one) */
  uint64_t r2[4];      /* R^2 mod p (converts into Montgomery form) */
  uint64_t ninv;       /* -p^-1 mod 2^64 (the reference's ZK_NINV) */
  int32_t kind;        /* ZKB_FIELD_GENERIC, ZKB_FIELD_BN254_FR or ZKB_FIELD_BN254_FQ */
  int32_t reserved;
} zkb_field;

#define ZKB_FIELD_GENERIC 0
#define ZKB_FIELD_BN254_FR 1
#define ZKB_FIELD_BN254_FQ 2

/* Replaces Field256.__init__ (zkgpu/field256_gpu.py:277-288): validates the
 * modulus (odd, in [3, 2^255); ZKB_EINVAL otherwise) and computes R mod p,
 * R^2 mod p and -p^-1 mod 2^64 on the host. Host pointers. */
int zkb_field_init(zkb_field* f, const uint64_t modulus[4]);

/* Replaces the zk256_mul / zk256_add / zk256_sub launches with their
 * single-row broadcast (zkgpu/field256_gpu.py:172-191, :466-473):
 * out[i] = a[i * a_step] OP b[i * b_step] for i < n, where a_step and b_step
 * are 1, or 0 to broadcast one row. n = 0 is a no-op. out may alias a or b.
 * zkb_field_mul with a == b and equal steps squares (36 word products in
 * place of 64; the same rows). */
int zkb_field_mul(const zkb_field* f, const uint64_t* a, int64_t a_step, const uint64_t* b,
                  int64_t b_step, uint64_t* out, int64_t n, void* stream);
int zkb_field_add(const zkb_field* f, const uint64_t* a, int64_t a_step, const uint64_t* b,
                  int64_t b_step, uint64_t* out, int64_t n, void* stream);
int zkb_field_sub(const zkb_field* f, const uint64_t* a, int64_t a_step, const uint64_t* b,
                  int64_t b_step, uint64_t* out, int64_t n, void* stream);

/* Replaces Field256.from_ints' device step (zkgpu/field256_gpu.py:307-310):
 * out[i] = Montgomery form of the plain value in[i]. For BN254 fields any
 * 256-bit value is accepted and reduced mod p on the device; for other moduli
 * in[i] must already be below p. */
int zkb_field_to_mont(const zkb_field* f, const uint64_t* in, uint64_t* out, int64_t n,
                      void* stream);

/* Replaces Field256.to_ints' device step (zkgpu/field256_gpu.py:318-319):
 * out[i] = the plain canonical value of Montgomery row in[i]. */
int zkb_field_from_mont(const zkb_field* f, const uint64_t* in, uint64_t* out, int64_t n,
                        void* stream);

/* ---- NTT ------------------------------------------------------------------ */

/* Device workspace (bytes) zkb_ntt needs for a transform of n rows. */
size_t zkb_ntt_workspace_bytes(int64_t n);

/* Number of NTT pass tiles on the current device, since the library loaded,
 * whose bounded wait for their TMA loads gave up (each such block stops early
 * and that transform's output is incomplete); 0 in a healthy run. It has no
 * counterpart in the reference. Synchronous; ~0 if the device cannot be read. */
uint64_t zkb_ntt_wait_timeouts(void);

/* Replaces Field256.ntt / _ntt_on_gpu (zkgpu/field256_gpu.py:347-387) and the
 * GPU coset form of Radix2Domain.coset_fft / coset_ifft (zkgpu/domain.py:122-135):
 *   forward:  out[k] = sum_j in[j] * g^j * w^(j k)
 *   inverse:  out[j] = n^-1 * g^-j * sum_k in[k] * w^(-j k)
 * in natural order, with w a primitive n-th root of unity and g the coset
 * offset (g = 1 when `coset` is NULL). n must be a power of two, 1 <= n <= 2^28.
 * `omega` (host, plain canonical value of w) may be NULL for BN254 Fr, which
 * then uses 5^((r-1)/n) (zkgpu/ntt.py:98-124). `coset` is a host pointer to g's
 * plain value, or NULL. `in` is not modified; out must not alias in. */
int zkb_ntt(const zkb_field* f, const uint64_t* in, uint64_t* out, int64_t n, int invert,
            const uint64_t* omega, const uint64_t* coset, void* workspace,
            size_t workspace_bytes, void* stream);

/* One transform of a batch (device pointers). */
typedef struct zkb_ntt_job {
  const uint64_t* in; /* (n, 4) Montgomery rows; not modified */
  uint64_t* out;      /* (n, 4); must not alias any input of the batch */
  int64_t n;          /* a power of two, 0 <= n <= 2^28 */
  int32_t invert;     /* nonzero: inverse transform */
  int32_t has_coset;  /* nonzero: coset transform with offset `coset` */
  uint64_t coset[4];  /* plain value of the coset offset g */
} zkb_ntt_job;

/* Device workspace (bytes) zkb_ntt_batch needs for these jobs (host array). */
size_t zkb_ntt_batch_workspace_bytes(const zkb_ntt_job* jobs, int count);

/* Batched form of zkb_ntt over BN254 Fr (built-in roots 5^((r-1)/n)): up to 64
 * independent transforms of any sizes in ONE persistent kernel launch. The
 * launch's CTAs take CTA-sized tiles from a device counter, first passes of
 * all transforms before second passes; a tile of a later pass waits for the
 * previous pass of its own transform (a bounded wait). Each job's output is
 * bit-identical to zkb_ntt's for the same arguments. `status` (device int32,
 * may be NULL) receives ZKB_OK, or ZKB_ETIMEOUT if a wait gave up (outputs
 * are then incomplete). `jobs` is a host array, read during the call. */
int zkb_ntt_batch(const zkb_field* f, const zkb_ntt_job* jobs, int count, void* workspace,
                  size_t workspace_bytes, int32_t* status, void* stream);

/* The cross-part step of one BN254 Fr NTT of n rows split over `parts` GPUs
 * (parts = G, a power of 2 in 2..16; G^2 <= n). It has no counterpart in the
 * reference, which runs on one GPU; it is the step that makes the single
 * transform of zkb_ntt shard (the four-step decomposition n = G m, m = n / G).
 * With the input in block layout (part r holds x[r m .. r m + m)), a first
 * exchange gives part s the rows x[j1 m + s c + i] of every j1 < G (c = m / G),
 * stored as `in` = (G, c): block j1 from part j1. This call writes `out` =
 * (G, c), block k1 bound for part k1:
 *   out[k1][i] = post[k1] w_n^(j2 k1) sum_j1 in[j1][i] w_G^(j1 k1),  j2 = s c + i,
 * with w^-1 when `invert`, and x[j] pre-scaled by g^j for a forward coset
 * transform (`coset`: host pointer to g's plain value, or NULL). `post` is a
 * device array of G Montgomery rows, or NULL for 1: G^-1 for an inverse
 * transform (times g^-k1 for an inverse coset). After a second exchange part t
 * holds the rows for k1 = t of every part in order, and zkb_ntt of size m
 * (inverse ones with coset offset g^G) yields y[t + k2 G] for k2 < m: cyclic
 * layout. zkgpu/sharded.py drives the whole transform over torch.distributed. */
int zkb_ntt_cross_step(const zkb_field* f, const uint64_t* in, uint64_t* out, int64_t n, int parts,
                       int part, int invert, const uint64_t* coset, const uint64_t* post,
                       void* stream);

/* Replaces the quotient step of the reference's GPU prover,
 * Fr.mul(Fr.sub(Fr.mul(a, b), c), z_inv) (demo/prover_simulation.py:148):
 * out[i] = (a[i] b[i] - c[i]) z over BN254 Fr, in one pass. a, b, c, out are
 * (n, 4) Montgomery rows; z points to ONE device row holding z's plain value
 * (e.g. 1 / (g^n - 1)), so that the call reads nothing from the host. out may
 * alias a, b or c. */
int zkb_quotient_pointwise(const uint64_t* a, const uint64_t* b, const uint64_t* c,
                           const uint64_t* z, uint64_t* out, int64_t n, void* stream);

/* ---- fields of one 64-bit word (moduli below 2^63) ------------------------ */

/* Replace gpu_batch_mul / gpu_batch_add (zkgpu/field_gpu.py:147-196):
 * out[i] = (a[i] OP b[i]) mod `mod`, for 2 <= mod < 2^63 (ZKB_EINVAL
 * otherwise). Inputs are any int64 values, reduced into [0, mod) first (so
 * negative ones land in the field); outputs lie in [0, mod). Device arrays of
 * n int64; out may alias a or b. */
int zkb_u64_mul(const int64_t* a, const int64_t* b, int64_t* out, int64_t n, int64_t mod, void* stream);
int zkb_u64_add(const int64_t* a, const int64_t* b, int64_t* out, int64_t n, int64_t mod, void* stream);

/* Replaces gpu_batch_pow (zkgpu/field_gpu.py:199-230) for a non-negative
 * exponent: out[i] = bases[i]^e mod `mod`, e given as `words` little-endian
 * 64-bit words in DEVICE memory (any size; words = 0 is e = 0). */
int zkb_u64_pow(const int64_t* bases, int64_t* out, int64_t n, const uint64_t* exp_words, int words,
                int64_t mod, void* stream);

/* Device workspace (bytes) zkb_ntt64 needs for n words. */
size_t zkb_ntt64_workspace_bytes(int64_t n);

/* Replaces ntt_gpu (zkgpu/ntt_gpu.py:86-155): the natural-order NTT (or, with
 * invert, its inverse scaled by n^-1) of n int64 values over an odd prime
 * mod < 2^63, with omega the primitive n-th root of unity the caller derives
 * (g^((mod-1)/n) for the smallest non-residue g, as zkgpu/ntt.py:98-124).
 * Inputs are reduced into [0, mod) first; n a power of 2 up to 2^30; in and
 * out must not overlap (ZKB_EINVAL). The workspace holds the stage twiddle
 * table (16 KiB for any n). */
int zkb_ntt64(const int64_t* in, int64_t* out, int64_t n, int64_t mod, int64_t omega, int invert,
              void* workspace, size_t workspace_bytes, void* stream);

/* ---- BN254 G1 ------------------------------------------------------------- */

/* Replace the zk_g1_add / zk_g1_add_affine / zk_g1_double launches
 * (zkgpu/curve_gpu.py:236-274, :394-414, :446-462): EFD add-2007-bl,
 * madd-2007-bl and dbl-2009-l with the reference's special cases, so the
 * Jacobian coordinates are exactly the reference's. a_step / b_step as for
 * the field ops. out may alias the inputs. */
int zkb_g1_add(const uint64_t* a, int64_t a_step, const uint64_t* b, int64_t b_step,
               uint64_t* out, int64_t n, void* stream);
int zkb_g1_add_affine(const uint64_t* a, int64_t a_step, const uint64_t* b, int64_t b_step,
                      uint64_t* out, int64_t n, void* stream);
int zkb_g1_double(const uint64_t* a, uint64_t* out, int64_t n, void* stream);

/* Replaces the device half of curve_gpu.from_device and curve.from_jacobian
 * (zkgpu/curve_gpu.py:384-386, zkgpu/curve.py:221-233): out is (n, 2, 4)
 * plain canonical affine coordinates, with (0, 0) for the identity. */
int zkb_g1_to_affine(const uint64_t* jac, uint64_t* out, int64_t n, void* stream);

/* Fixed-base scalar multiplication k_i G for the generator G = (1, 2), the
 * reference's Point.__mul__ (zkgpu/curve.py:153-159) used to build base sets:
 * k is (n, 4) plain 256-bit scalars (not 0 mod r), out is (n, 2, 4) affine
 * rows in Montgomery form. */
int zkb_g1_mul_generator(const uint64_t* k, uint64_t* out, int64_t n, void* stream);

/* Replaces the on-curve validation that Point() performs for every MSM input
 * (zkgpu/msm_gpu.py:441-442, zkgpu/curve.py:69-79), on the device:
 * points is (n, 2, 4) affine in Montgomery form; *first_bad (a device int64)
 * receives the smallest index whose point is off the curve, or -1. */
int zkb_g1_check_affine(const uint64_t* points, int64_t n, int64_t* first_bad, void* stream);

/* ---- MSM ------------------------------------------------------------------ */

/* The library's default window size for n points. */
int zkb_msm_default_window(int64_t n);

/* Device workspace (bytes) zkb_msm needs for n points at window size w
 * (w = 0: the default). */
size_t zkb_msm_workspace_bytes(int64_t n, int window_size);

/* Replaces msm_pippenger_gpu's device path (zkgpu/msm_gpu.py:336-377, :447-449)
 * including the final window combination and affine conversion, which the
 * reference runs on the CPU (zkgpu/msm.py:156-169, zkgpu/curve.py:221-233).
 *   points   (n, 2, 4) affine BN254 G1 points in Montgomery form (valid points;
 *            see zkb_g1_check_affine)
 *   scalars  (n, 4) plain little-endian 256-bit integers; reduced mod r on the
 *            device (the reference reduces mod r on the host)
 *   result   device buffer of 9 uint64: x (4 limbs), y (4 limbs), both plain
 *            canonical, then 1 if the sum is the point at infinity (x = y = 0)
 *            else 0.
 * window_size is in 1..20, or 0 for zkb_msm_default_window(n). Digits are
 * signed, so a window of w bits has 2^(w-1) buckets. n = 0 gives infinity. */
int zkb_msm(const uint64_t* points, const uint64_t* scalars, int64_t n, int window_size,
            uint64_t* result, void* workspace, size_t workspace_bytes, void* stream);

/* MSM for callers that cannot allocate device memory at call time: a plugin
 * living inside a framework that owns all device memory through its own
 * allocator, or a serving loop that must never reach cudaMalloc because it
 * can synchronise the whole device. It has no counterpart in the reference.
 * Same inputs, result and result layout as zkb_msm, but no workspace: the
 * scratch is a fixed 64 MiB array inside the library (zkb_msm_no_alloc_capacity()),
 * which every GPU that loads the library keeps until the process exits. That
 * covers 2^16 points at the default window; a problem that needs more returns
 * ZKB_EWORKSPACE. Each call looks up the array's device address for the
 * current device; the first call on a device also loads the library's code
 * there, so make that first call before any stream capture. A problem of 2^31
 * or more digit pairs is refused with ZKB_EINVAL, as by zkb_msm (the 64 MiB
 * limit refuses it first). All calls share the array, so calls whose work overlaps on the GPU
 * (other streams or other host threads) race: order them, e.g. on one stream.
 * Nothing is allocated or freed. */
int zkb_msm_no_alloc(const uint64_t* points, const uint64_t* scalars, int64_t n, int window_size,
                     uint64_t* result, void* stream);

/* Size in bytes of the fixed scratch array zkb_msm_no_alloc works in. */
size_t zkb_msm_no_alloc_capacity(void);

/* One MSM of a batch: the arguments of zkb_msm (device pointers). */
typedef struct zkb_msm_job {
  const uint64_t* points;  /* (n, 2, 4) affine, Montgomery form */
  const uint64_t* scalars; /* (n, 4) plain 256-bit integers */
  int64_t n;               /* 0 <= n < 2^30; n = 0 gives infinity */
  uint64_t* result;        /* 9 uint64, laid out as zkb_msm's */
  int32_t window_size;     /* 1..20, or 0 for zkb_msm_default_window(n) */
  int32_t reserved;
} zkb_msm_job;

/* Device workspace (bytes) zkb_msm_batch needs for these jobs (host array). */
size_t zkb_msm_batch_workspace_bytes(const zkb_msm_job* jobs, int count);

/* Batched form of msm_pippenger_gpu (zkgpu/msm_gpu.py:398-449) for many
 * independent MSMs of uneven sizes, e.g. the four G1 MSMs of a Groth16 proof
 * (demo/prover_simulation.py:94-98) or MSMs over prefixes of one resident
 * base set. Each job's result is exactly zkb_msm's for the same arguments.
 * Jobs with the same window size run through one pipeline (one sort, one
 * bucket pass, one reduction and one finalize for all of them, up to 64 jobs
 * and 2^31 digit pairs per group); groups of different window sizes run
 * concurrently on library-owned side streams that fork from and join back to
 * `stream`. `jobs` is a host array; nothing is copied from it after the call
 * returns. */
int zkb_msm_batch(const zkb_msm_job* jobs, int count, void* workspace, size_t workspace_bytes,
                  void* stream);

/* ---- MSMs over a resident base set (fixed-base tables) ------------------- */

/* These have no counterpart in the reference, whose MSM takes its points with
 * every call. A prover that runs many MSMs over one resident base set (an SRS)
 * builds a table once: for each point P_i its 2 W rows 2^(w win) P_i and
 * phi(2^(w win) P_i), win < W = ceil(128 / w), affine Montgomery (64 bytes a
 * row). An MSM over the table adds every window's digits into one set of
 * 2^(w-1) buckets: fewer buckets to reduce, no doublings in the final
 * combination, and room for larger windows, i.e. fewer mixed additions. The
 * result equals zkb_msm's over the same points at any window. */

/* Device bytes of the table of n points at window w (8..24): n * 2W * 64;
 * 0 for an invalid window or n <= 0. */
size_t zkb_msm_table_bytes(int64_t n, int window_size);

/* Builds the table of `points` ((n, 2, 4) affine Montgomery rows on the curve,
 * not the identity) at window w (8..24) into `table` (zkb_msm_table_bytes).
 * A table of N points also serves every prefix of them: its first n * 2W rows
 * are the table of the first n points. */
int zkb_msm_table_build(const uint64_t* points, int64_t n, int window_size, uint64_t* table,
                        void* stream);

/* zkb_msm_batch over tables: jobs[j].points is a table built at window
 * jobs[j].window_size (required, 8..24) of at least jobs[j].n points, and the
 * job sums s_i P_i over its first n points. Results as zkb_msm_batch's. */
size_t zkb_msm_fixed_batch_workspace_bytes(const zkb_msm_job* jobs, int count);
int zkb_msm_fixed_batch(const zkb_msm_job* jobs, int count, void* workspace, size_t workspace_bytes,
                        void* stream);

/* ---- measurement -------------------------------------------------------- */

/* Tuning knobs, read by each call when it plans its work (so they also change
 * the workspace size queries): "msm.pairs_per_thread" (sorted pairs a bucket
 * thread adds in turn, 8..4096; default 0 = by size: the pair bound over 2^19,
 * as a power of two within 8..64, or within 8..16 for zkb_msm and
 * zkb_msm_no_alloc), "msm.call_pairs_cap" (16: that upper limit for the
 * one-MSM calls, 8..64; shorter bucket blocks let work on other streams reach
 * the SMs sooner), "msm.slots_per_thread" (8), "msm.reduce_log_segment" (4: the
 * first reduction level sums 16 buckets a lane, 512 a warp), "msm.sort" (1:
 * pairs grouped by a counting sort that skips zero digits; 0: a radix sort
 * of all pairs; the same points either way),
 * "ntt.max_log_radix" (log2 of the largest sub-transform one NTT pass does,
 * 8..12; default 0 = by size: three passes from 2^19 rows, else up to 12),
 * "ntt.cta_log_elems" (log2 of the rows staged per NTT block, 9..12; default
 * 0 = 9: a block holds one sub-transform once those reach 512 rows),
 * "ntt.threads" (threads per NTT block, 64..512; default 0 = by the block's
 * rows: 128 up to 512, 256 up to 2048, 512 for 4096); the int64 NTT's tile shapes
 * "ntt64.first_col_log" (input words per row of a first-pass tile, log2, 0..6;
 * -1 = by size), "ntt64.first_max_k" (first-pass stages, 4..10; 0 = by size),
 * "ntt64.col_log" (words per row of a later-pass tile, log2, 1..6; 0 = by size),
 * "ntt64.max_k" (most stages of a later pass, 2..10; 0 = by size);
 * "ntt.full_table_mb" (MiB the library may hold in expanded NTT tables: per
 * pass shape and direction the boundary twiddles of a non-last pass, per
 * coset transform its n scale factors, each saving one product per row;
 * default 4096, 0 = none);
 * "ntt.tma" (1: transforms of two or more passes run TMA-fed pass kernels;
 * 0: the per-thread gather form; the same rows either way), "ntt.tma_grid"
 * (1: one tile per block; 0: one persistent wave of double-buffered blocks),
 * "ntt.tma_blocks_per_sm" (0, or 5 / 6: the pass kernel of 128-thread blocks
 * with its registers capped for that many blocks per SM), "ntt.lazy" (1:
 * inside a TMA pass, values stay in [0, 2p) between butterfly rounds and are
 * made canonical at the store, for moduli below 2^254; 0: canonical after
 * every operation; the same rows either way);
 * "msm.affine_rounds" (rounds in which every bucket's list is halved by affine
 * additions sharing one inversion per block, before the XYZZ levels; 0 = none,
 * the default; -1 = by size; 1..8 forced), "msm.affine_batch" (output entries
 * per thread of such a round, 8..512; default 64);
 * "ntt.batch_spin_limit" (polls, each after a sleep of at least 256 ns, before
 * a tile of zkb_ntt_batch gives up waiting for the previous pass of its
 * transform and reports ZKB_ETIMEOUT through the status word; 0 = the default
 * 2^22, about a second).
 * ZKB_EINVAL for an unknown name or a value out of range. Process-wide, not
 * per stream. */
int zkb_tune_set(const char* key, int value);
int zkb_tune_get(const char* key, int* value);

/* Per-size tuning tables, one entry per log2 problem size (0..32): what an
 * autotuner measured best (zkgpu/autotune.py fills and caches them). It
 * replaces the reference's addition-count window model
 * (pippenger_window_size, zkgpu/msm.py:112-121) with measured choices.
 * Tables: "msm.window" (1..20; the default window of an MSM whose point count
 * rounds up to 2^log_n), "ntt.max_log_radix" (8..12), "ntt.cta_log_elems"
 * (9..12), "ntt.threads" (64..512) for an NTT of 2^log_n rows. value = 0
 * clears an entry. An entry takes precedence over the process-wide knob of
 * the same name. Tables are read when a call plans its work: change them
 * between a workspace-size query and the call it sizes and the two disagree. */
int zkb_tune_set_sized(const char* key, int log_n, int value);
int zkb_tune_get_sized(const char* key, int log_n, int* value);

/* Measured issue rates on the current device: loops of independent
 * mad.lo.u32, of mad.wide.u32 (32 x 32 -> 64-bit multiply-add) and of this
 * library's 256-bit Montgomery product over BN254's base field, each one
 * launch of as many 256-thread blocks as fit the SMs at once. *_per_clk_sm is
 * operations per SM per SM clock (from the SMs' cycle counters, independent
 * of the clock), *_per_s per second over the whole GPU (CUDA events), *_mhz
 * the SM clock that the two imply. They are the measured denominators of the
 * integer rooflines; the IMAD pipe peak at clock f is sms * madlo_per_clk_sm
 * * f. Takes a few tens of milliseconds and synchronises the stream. */
typedef struct zkb_int_peaks {
  double madlo_per_clk_sm, madlo_per_s, madlo_mhz;
  double madwide_per_clk_sm, madwide_per_s, madwide_mhz;
  double montmul_per_clk_sm, montmul_per_s, montmul_mhz;
  int32_t sms;
  int32_t reserved;
} zkb_int_peaks;

int zkb_measure_int_peaks(zkb_int_peaks* out, void* stream);

/* Number of this library's own kernels launched so far in this process
 * (sorting kernels of the CUB library are not counted). */
uint64_t zkb_launch_count(void);

/* Per-stage timing with CUDA events on the launching stream. on = 1 clears
 * the record and starts recording the MSM and NTT stages; 0 stops. */
void zkb_profile_enable(int on);

/* Waits for the recorded events and writes one line per stage,
 * "name count total_ms", into buf (host, len bytes, NUL-terminated).
 * Returns the length the full report needs, including the NUL. */
int zkb_profile_report(char* buf, size_t len);

#ifdef __cplusplus
}
#endif

#endif /* ZKB200_H */
