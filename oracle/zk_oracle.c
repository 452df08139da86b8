/*
 * zk_oracle.c — the reference's BN254 CPU algorithms restated in C.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for libzkb200.so and the timed CPU
 * baseline; never linked into the product. Built by oracle/Makefile into
 * oracle/libzk_oracle.so and called through oracle/c_oracle.py.
 *
 * Arithmetic follows the reference file by file:
 *   field   Montgomery CIOS on 4 x 64-bit limbs, R = 2^256, five words of state
 *           (zkgpu/field256_gpu.py:65-169)
 *   NTT     bit-reversed copy, then iterative radix-2 DIT stages with the
 *           twiddle w_len^j (zkgpu/ntt.py:132-203); inverse scales by n^-1;
 *           coset scaling by g^j / g^-j (zkgpu/domain.py:33-39, :122-135)
 *   curve   EFD dbl-2009-l, add-2007-bl, madd-2007-bl with the reference's
 *           special cases (zkgpu/curve.py:236-303), from_jacobian with one
 *           inversion (:221-233), double-and-add (:306-324)
 *   MSM     unsigned w-bit windows, buckets by mixed addition, the running-sum
 *           trick, Horner over windows (zkgpu/msm.py:156-207)
 * Rows use the reference's layout: little-endian 64-bit limbs, Montgomery
 * form for field elements and curve coordinates.
 *
 * Threads: the MSM splits windows across threads, the NTT splits each
 * stage's butterflies, base generation splits points. Results do not depend
 * on the thread count.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

typedef struct {
  uint64_t p[4];
  uint64_t one[4];
  uint64_t r2[4];
  uint64_t ninv; /* -p^-1 mod 2^64 */
} zo_field;

/* BN254 scalar field r and base field p (zkgpu/field.py:17, zkgpu/curve.py:29) */
static const zo_field FR = {
    {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull, 0x30644e72e131a029ull},
    {0xac96341c4ffffffbull, 0x36fc76959f60cd29ull, 0x666ea36f7879462eull, 0x0e0a77c19a07df2full},
    {0x1bb8e645ae216da7ull, 0x53fe3ab1e35c59e3ull, 0x8c49833d53bb8085ull, 0x0216d0b17f4e44a5ull},
    0xc2e1f593efffffffull};
static const zo_field FQ = {
    {0x3c208c16d87cfd47ull, 0x97816a916871ca8dull, 0xb85045b68181585dull, 0x30644e72e131a029ull},
    {0xd35d438dc58f0d9dull, 0x0a78eb28f5c70b3dull, 0x666ea36f7879462cull, 0x0e0a77c19a07df2full},
    {0xf32cfc5b538afa89ull, 0xb5e71911d44501fbull, 0x47ab1eff0a417ff6ull, 0x06d89f71cab8351full},
    0x87d20782e4866389ull};

static const zo_field* field_of(int fid) { return fid == 0 ? &FR : &FQ; }

/* ---- field ----------------------------------------------------------------- */

static int geq(const uint64_t a[4], const uint64_t b[4]) {
  for (int j = 3; j >= 0; --j)
    if (a[j] != b[j]) return a[j] > b[j];
  return 1;
}

static void sub4(uint64_t r[4], const uint64_t a[4], const uint64_t b[4]) {
  uint64_t borrow = 0;
  for (int j = 0; j < 4; ++j) {
    u128 d = (u128)a[j] - b[j] - borrow;
    r[j] = (uint64_t)d;
    borrow = (uint64_t)(d >> 64) & 1;
  }
}

static void reduce_once(uint64_t t[4], const zo_field* f) {
  if (geq(t, f->p)) sub4(t, t, f->p);
}

/* CIOS: t < 2p between steps, so five words of state (zkgpu/field256_gpu.py:96-128). */
static void fmul(uint64_t r[4], const uint64_t a[4], const uint64_t b[4], const zo_field* f) {
  uint64_t t[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < 4; ++i) {
    u128 c = 0;
    for (int j = 0; j < 4; ++j) {
      c += (u128)a[j] * b[i] + t[j];
      t[j] = (uint64_t)c;
      c >>= 64;
    }
    t[4] = (uint64_t)c;
    uint64_t m = t[0] * f->ninv;
    c = ((u128)m * f->p[0] + t[0]) >> 64;
    for (int j = 1; j < 4; ++j) {
      c += (u128)m * f->p[j] + t[j];
      t[j - 1] = (uint64_t)c;
      c >>= 64;
    }
    t[3] = t[4] + (uint64_t)c;
  }
  reduce_once(t, f);
  memcpy(r, t, 32);
}

static void fadd(uint64_t r[4], const uint64_t a[4], const uint64_t b[4], const zo_field* f) {
  uint64_t s[4], carry = 0;
  for (int j = 0; j < 4; ++j) {
    u128 x = (u128)a[j] + b[j] + carry;
    s[j] = (uint64_t)x;
    carry = (uint64_t)(x >> 64);
  }
  reduce_once(s, f);
  memcpy(r, s, 32);
}

static void fsub(uint64_t r[4], const uint64_t a[4], const uint64_t b[4], const zo_field* f) {
  uint64_t s[4], borrow = 0;
  for (int j = 0; j < 4; ++j) {
    u128 d = (u128)a[j] - b[j] - borrow;
    s[j] = (uint64_t)d;
    borrow = (uint64_t)(d >> 64) & 1;
  }
  if (borrow) {
    uint64_t carry = 0;
    for (int j = 0; j < 4; ++j) {
      u128 x = (u128)s[j] + f->p[j] + carry;
      s[j] = (uint64_t)x;
      carry = (uint64_t)(x >> 64);
    }
  }
  memcpy(r, s, 32);
}

static int fis_zero(const uint64_t a[4]) { return (a[0] | a[1] | a[2] | a[3]) == 0; }

static void fto_mont(uint64_t r[4], const uint64_t a[4], const zo_field* f) { fmul(r, a, f->r2, f); }

static void ffrom_mont(uint64_t r[4], const uint64_t a[4], const zo_field* f) {
  const uint64_t one[4] = {1, 0, 0, 0};
  fmul(r, a, one, f);
}

/* a^e for a 256-bit plain exponent, a in Montgomery form. */
static void fpow(uint64_t r[4], const uint64_t a[4], const uint64_t e[4], const zo_field* f) {
  uint64_t acc[4], base[4];
  memcpy(acc, f->one, 32);
  memcpy(base, a, 32);
  for (int w = 3; w >= 0; --w)
    for (int bit = 63; bit >= 0; --bit) {
      fmul(acc, acc, acc, f);
      if ((e[w] >> bit) & 1) fmul(acc, acc, base, f);
    }
  memcpy(r, acc, 32);
}

static void fpow_u64(uint64_t r[4], const uint64_t a[4], uint64_t e, const zo_field* f) {
  const uint64_t ee[4] = {e, 0, 0, 0};
  fpow(r, a, ee, f);
}

static void finv(uint64_t r[4], const uint64_t a[4], const zo_field* f) {
  uint64_t e[4];
  memcpy(e, f->p, 32);
  e[0] -= 2; /* p odd, p > 2: no borrow */
  fpow(r, a, e, f);
}

/* reduce any 256-bit value mod a BN254 modulus (p > 2^253: at most 5 subtractions) */
static void freduce_full(uint64_t a[4], const zo_field* f) {
  while (geq(a, f->p)) sub4(a, a, f->p);
}

/* ---- threads ----------------------------------------------------------------- */

typedef void (*range_fn)(void* ctx, int64_t lo, int64_t hi);

typedef struct {
  range_fn fn;
  void* ctx;
  int64_t lo, hi;
} range_job;

static void* range_worker(void* arg) {
  range_job* j = (range_job*)arg;
  j->fn(j->ctx, j->lo, j->hi);
  return NULL;
}

/* fn(ctx, lo, hi) over [0, n) split into `threads` contiguous pieces */
static void parallel_for(int64_t n, int threads, range_fn fn, void* ctx) {
  if (threads < 1) threads = 1;
  if (threads > n) threads = (int)(n > 0 ? n : 1);
  if (threads == 1) {
    fn(ctx, 0, n);
    return;
  }
  pthread_t* tid = (pthread_t*)malloc(sizeof(pthread_t) * threads);
  range_job* jobs = (range_job*)malloc(sizeof(range_job) * threads);
  for (int t = 0; t < threads; ++t) {
    jobs[t].fn = fn;
    jobs[t].ctx = ctx;
    jobs[t].lo = n * t / threads;
    jobs[t].hi = n * (t + 1) / threads;
    pthread_create(&tid[t], NULL, range_worker, &jobs[t]);
  }
  for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
  free(tid);
  free(jobs);
}

/* ---- exported field ops (Montgomery rows) ------------------------------------ */

void zo_field_mul(int fid, const uint64_t* a, const uint64_t* b, uint64_t* out, int64_t n) {
  const zo_field* f = field_of(fid);
  for (int64_t i = 0; i < n; ++i) fmul(out + 4 * i, a + 4 * i, b + 4 * i, f);
}
void zo_field_add(int fid, const uint64_t* a, const uint64_t* b, uint64_t* out, int64_t n) {
  const zo_field* f = field_of(fid);
  for (int64_t i = 0; i < n; ++i) fadd(out + 4 * i, a + 4 * i, b + 4 * i, f);
}
void zo_field_sub(int fid, const uint64_t* a, const uint64_t* b, uint64_t* out, int64_t n) {
  const zo_field* f = field_of(fid);
  for (int64_t i = 0; i < n; ++i) fsub(out + 4 * i, a + 4 * i, b + 4 * i, f);
}
void zo_to_mont(int fid, const uint64_t* in, uint64_t* out, int64_t n) {
  const zo_field* f = field_of(fid);
  for (int64_t i = 0; i < n; ++i) {
    uint64_t v[4];
    memcpy(v, in + 4 * i, 32);
    freduce_full(v, f);
    fto_mont(out + 4 * i, v, f);
  }
}
void zo_from_mont(int fid, const uint64_t* in, uint64_t* out, int64_t n) {
  const zo_field* f = field_of(fid);
  for (int64_t i = 0; i < n; ++i) ffrom_mont(out + 4 * i, in + 4 * i, f);
}

/* ---- NTT over Fr (zkgpu/ntt.py:149-203) ------------------------------------------ */

/* w_{2^28} = 5^((r-1)/2^28) (plain), the root all sizes derive from */
static const uint64_t ROOT28[4] = {0x9bd61b6e725b19f0ull, 0x402d111e41112ed4ull,
                                   0x00e0a7eb8ef62abcull, 0x2a3c09f0a58a7e85ull};

typedef struct {
  uint64_t* a;
  const uint64_t* tw; /* tw[j] = w_len^j for j < half */
  int64_t half, n;
} stage_ctx;

static void stage_range(void* vctx, int64_t lo, int64_t hi) {
  stage_ctx* c = (stage_ctx*)vctx;
  /* butterfly index k in [lo, hi): group k / half, position j = k % half */
  for (int64_t k = lo; k < hi; ++k) {
    int64_t j = k % c->half;
    int64_t i0 = (k / c->half) * 2 * c->half + j;
    int64_t i1 = i0 + c->half;
    uint64_t v[4];
    fmul(v, c->a + 4 * i1, c->tw + 4 * j, &FR);
    uint64_t u[4];
    memcpy(u, c->a + 4 * i0, 32);
    fadd(c->a + 4 * i0, u, v, &FR);
    fsub(c->a + 4 * i1, u, v, &FR);
  }
}

typedef struct {
  uint64_t* a;
  const uint64_t* g_lo;
  const uint64_t* g_hi;
  int gs;
  const uint64_t* scale;
} scale_ctx;

static void scale_range(void* vctx, int64_t lo, int64_t hi) {
  scale_ctx* c = (scale_ctx*)vctx;
  for (int64_t i = lo; i < hi; ++i) {
    if (c->g_lo) {
      uint64_t g[4];
      fmul(g, c->g_lo + 4 * (i & ((1ll << c->gs) - 1)), c->g_hi + 4 * (i >> c->gs), &FR);
      fmul(c->a + 4 * i, c->a + 4 * i, g, &FR);
    }
    if (c->scale) fmul(c->a + 4 * i, c->a + 4 * i, c->scale, &FR);
  }
}

typedef struct {
  const uint64_t* in;
  uint64_t* out;
  int log_n;
  const uint64_t* g_lo; /* forward coset: out[bitrev(i)] = in[i] g^i, else plain copy */
  const uint64_t* g_hi;
  int gs;
} bitrev_ctx;

static void bitrev_range(void* vctx, int64_t lo, int64_t hi) {
  bitrev_ctx* c = (bitrev_ctx*)vctx;
  for (int64_t i = lo; i < hi; ++i) {
    int64_t r = 0;
    for (int b = 0; b < c->log_n; ++b) r |= ((i >> b) & 1) << (c->log_n - 1 - b);
    if (c->g_lo) {
      uint64_t g[4];
      fmul(g, c->g_lo + 4 * (i & ((1ll << c->gs) - 1)), c->g_hi + 4 * (i >> c->gs), &FR);
      fmul(c->out + 4 * r, c->in + 4 * i, g, &FR);
    } else {
      memcpy(c->out + 4 * r, c->in + 4 * i, 32);
    }
  }
}

/* tab[i] = base^i for i < count (Montgomery) */
static void power_table(uint64_t* tab, const uint64_t base[4], int64_t count) {
  if (count <= 0) return;
  memcpy(tab, FR.one, 32);
  for (int64_t i = 1; i < count; ++i) fmul(tab + 4 * i, tab + 4 * (i - 1), base, &FR);
}

/*
 * out = NTT(in) over BN254 Fr on Montgomery rows, natural order. coset (plain
 * g, or NULL): forward scales input j by g^j first, inverse scales output j by
 * g^-j. Only stages [stage_lo, stage_hi) of the log2 n run (for timing a
 * sample); pass 0 and 64 for the full transform. Returns 0, or -1 for a bad n.
 */
int zo_ntt(const uint64_t* in, uint64_t* out, int64_t n, int invert, const uint64_t* coset,
           int threads, int stage_lo, int stage_hi) {
  if (n <= 0 || (n & (n - 1)) || n > (1ll << 28)) return -1;
  int log_n = 0;
  while ((1ll << log_n) < n) ++log_n;
  uint64_t g_m[4], t[4];
  uint64_t *g_lo = NULL, *g_hi = NULL;
  int gs = (log_n + 1) / 2;
  if (coset) {
    /* g^j for the forward transform (applied to the input, so before the
       bit reversal: scale out[bitrev(j)] by g^j is the same as scaling in[j]) */
    memcpy(t, coset, 32);
    fto_mont(g_m, t, &FR);
    if (invert) finv(g_m, g_m, &FR);
    g_lo = (uint64_t*)malloc((size_t)32 << gs);
    g_hi = (uint64_t*)malloc((size_t)32 << (log_n - gs));
    power_table(g_lo, g_m, 1ll << gs);
    uint64_t step[4];
    fpow_u64(step, g_m, 1ull << gs, &FR);
    power_table(g_hi, step, 1ll << (log_n - gs));
  }
  /* bit-reversed copy (zkgpu/ntt.py:132-141), with the forward coset scaling
     x_j g^j (zkgpu/domain.py:33-39) applied on the way */
  {
    const int fwd_coset = coset && !invert;
    bitrev_ctx c = {in, out, log_n, fwd_coset ? g_lo : NULL, fwd_coset ? g_hi : NULL, gs};
    parallel_for(n, threads, bitrev_range, &c);
  }
  /* omega_n = w28^(2^28 / n), inverted for the inverse transform */
  uint64_t w[4];
  fto_mont(t, ROOT28, &FR);
  fpow_u64(w, t, (1ull << 28) >> log_n, &FR);
  if (invert) finv(w, w, &FR);
  uint64_t* tw = (uint64_t*)malloc((size_t)32 * (n / 2 > 0 ? n / 2 : 1));
  for (int s = 0; s < log_n; ++s) {
    int64_t half = 1ll << s;
    if (s < stage_lo || s >= stage_hi) continue;
    /* w_len = omega^(n / length), length = 2 half (zkgpu/ntt.py:184-195) */
    uint64_t wl[4];
    fpow_u64(wl, w, (uint64_t)(n >> (s + 1)), &FR);
    power_table(tw, wl, half);
    stage_ctx c = {out, tw, half, n};
    parallel_for(n / 2, threads, stage_range, &c);
  }
  free(tw);
  if (invert) {
    uint64_t nv[4] = {(uint64_t)n, 0, 0, 0}, nm[4], ninv[4];
    fto_mont(nm, nv, &FR);
    finv(ninv, nm, &FR);
    scale_ctx c = {out, coset ? g_lo : NULL, g_hi, gs, ninv};
    parallel_for(n, threads, scale_range, &c);
  }
  free(g_lo);
  free(g_hi);
  return 0;
}

/* ---- G1 (zkgpu/curve.py:236-324) --------------------------------------------- */

typedef struct {
  uint64_t x[4], y[4], z[4];
} jac;

static void jset_identity(jac* r) {
  memcpy(r->x, FQ.one, 32);
  memcpy(r->y, FQ.one, 32);
  memset(r->z, 0, 32);
}

static void jdouble(jac* r, const jac* p) {
  const zo_field* f = &FQ;
  if (fis_zero(p->z) || fis_zero(p->y)) {
    jset_identity(r);
    return;
  }
  uint64_t a[4], b[4], c[4], d[4], e[4], t[4], x3[4], y3[4], z3[4];
  fmul(a, p->x, p->x, f);
  fmul(b, p->y, p->y, f);
  fmul(c, b, b, f);
  fadd(t, p->x, b, f);
  fmul(t, t, t, f);
  fsub(t, t, a, f);
  fsub(t, t, c, f);
  fadd(d, t, t, f);
  fadd(e, a, a, f);
  fadd(e, e, a, f);
  fmul(x3, e, e, f);
  fadd(t, d, d, f);
  fsub(x3, x3, t, f);
  fsub(t, d, x3, f);
  fmul(y3, e, t, f);
  fadd(t, c, c, f);
  fadd(t, t, t, f);
  fadd(t, t, t, f);
  fsub(y3, y3, t, f);
  fmul(t, p->y, p->z, f);
  fadd(z3, t, t, f);
  memcpy(r->x, x3, 32);
  memcpy(r->y, y3, 32);
  memcpy(r->z, z3, 32);
}

static void jadd(jac* r, const jac* p, const jac* q) {
  const zo_field* f = &FQ;
  if (fis_zero(p->z)) {
    *r = *q;
    return;
  }
  if (fis_zero(q->z)) {
    *r = *p;
    return;
  }
  uint64_t z1z1[4], z2z2[4], u1[4], u2[4], s1[4], s2[4], h[4], rr[4], i[4], j[4], v[4], t[4];
  fmul(z1z1, p->z, p->z, f);
  fmul(z2z2, q->z, q->z, f);
  fmul(u1, p->x, z2z2, f);
  fmul(u2, q->x, z1z1, f);
  fmul(s1, p->y, q->z, f);
  fmul(s1, s1, z2z2, f);
  fmul(s2, q->y, p->z, f);
  fmul(s2, s2, z1z1, f);
  fsub(h, u2, u1, f);
  fsub(rr, s2, s1, f);
  fadd(rr, rr, rr, f);
  if (fis_zero(h)) {
    if (fis_zero(rr))
      jdouble(r, p);
    else
      jset_identity(r);
    return;
  }
  fadd(t, h, h, f);
  fmul(i, t, t, f);
  fmul(j, h, i, f);
  fmul(v, u1, i, f);
  uint64_t x3[4], y3[4], z3[4];
  fmul(x3, rr, rr, f);
  fsub(x3, x3, j, f);
  fadd(t, v, v, f);
  fsub(x3, x3, t, f);
  fsub(t, v, x3, f);
  fmul(y3, rr, t, f);
  fmul(t, s1, j, f);
  fadd(t, t, t, f);
  fsub(y3, y3, t, f);
  fadd(t, p->z, q->z, f);
  fmul(z3, t, t, f);
  fsub(z3, z3, z1z1, f);
  fsub(z3, z3, z2z2, f);
  fmul(z3, z3, h, f);
  memcpy(r->x, x3, 32);
  memcpy(r->y, y3, 32);
  memcpy(r->z, z3, 32);
}

static void jadd_affine(jac* r, const jac* p, const uint64_t qx[4], const uint64_t qy[4]) {
  const zo_field* f = &FQ;
  if (fis_zero(p->z)) {
    memcpy(r->x, qx, 32);
    memcpy(r->y, qy, 32);
    memcpy(r->z, f->one, 32);
    return;
  }
  uint64_t z1z1[4], u2[4], s2[4], h[4], hh[4], i[4], j[4], rr[4], v[4], t[4];
  fmul(z1z1, p->z, p->z, f);
  fmul(u2, qx, z1z1, f);
  fmul(s2, qy, p->z, f);
  fmul(s2, s2, z1z1, f);
  fsub(h, u2, p->x, f);
  fsub(rr, s2, p->y, f);
  fadd(rr, rr, rr, f);
  if (fis_zero(h)) {
    if (fis_zero(rr))
      jdouble(r, p);
    else
      jset_identity(r);
    return;
  }
  fmul(hh, h, h, f);
  fadd(i, hh, hh, f);
  fadd(i, i, i, f);
  fmul(j, h, i, f);
  fmul(v, p->x, i, f);
  uint64_t x3[4], y3[4], z3[4];
  fmul(x3, rr, rr, f);
  fsub(x3, x3, j, f);
  fadd(t, v, v, f);
  fsub(x3, x3, t, f);
  fsub(t, v, x3, f);
  fmul(y3, rr, t, f);
  fmul(t, p->y, j, f);
  fadd(t, t, t, f);
  fsub(y3, y3, t, f);
  fadd(t, p->z, h, f);
  fmul(z3, t, t, f);
  fsub(z3, z3, z1z1, f);
  fsub(z3, z3, hh, f);
  memcpy(r->x, x3, 32);
  memcpy(r->y, y3, 32);
  memcpy(r->z, z3, 32);
}

/* affine plain (x, y) and an infinity flag for a Jacobian point (zkgpu/curve.py:221-233) */
static void jto_affine_plain(const jac* p, uint64_t out[9]) {
  const zo_field* f = &FQ;
  memset(out, 0, 72);
  if (fis_zero(p->z)) {
    out[8] = 1;
    return;
  }
  uint64_t zi[4], zi2[4], x[4], y[4];
  finv(zi, p->z, f);
  fmul(zi2, zi, zi, f);
  fmul(x, p->x, zi2, f);
  fmul(zi2, zi2, zi, f);
  fmul(y, p->y, zi2, f);
  ffrom_mont(out, x, f);
  ffrom_mont(out + 4, y, f);
}

void zo_g1_add(const uint64_t* a, const uint64_t* b, uint64_t* out, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    jac p, q, r;
    memcpy(&p, a + 12 * i, 96);
    memcpy(&q, b + 12 * i, 96);
    jadd(&r, &p, &q);
    memcpy(out + 12 * i, &r, 96);
  }
}

void zo_g1_add_affine(const uint64_t* a, const uint64_t* b, uint64_t* out, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    jac p, r;
    memcpy(&p, a + 12 * i, 96);
    jadd_affine(&r, &p, b + 8 * i, b + 8 * i + 4);
    memcpy(out + 12 * i, &r, 96);
  }
}

void zo_g1_double(const uint64_t* a, uint64_t* out, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    jac p, r;
    memcpy(&p, a + 12 * i, 96);
    jdouble(&r, &p);
    memcpy(out + 12 * i, &r, 96);
  }
}

void zo_g1_to_affine(const uint64_t* a, uint64_t* out9, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    jac p;
    memcpy(&p, a + 12 * i, 96);
    jto_affine_plain(&p, out9 + 9 * i);
  }
}

/* k G by left-to-right double-and-add (zkgpu/curve.py:306-324), G = (1, 2). */
static void gen_mul(jac* acc, const uint64_t k[4]) {
  uint64_t one[4] = {1, 0, 0, 0}, two[4] = {2, 0, 0, 0}, gx[4], gy[4];
  fto_mont(gx, one, &FQ);
  fto_mont(gy, two, &FQ);
  jset_identity(acc);
  int started = 0;
  for (int w = 3; w >= 0; --w)
    for (int bit = 63; bit >= 0; --bit) {
      if (started) jdouble(acc, acc);
      if ((k[w] >> bit) & 1) {
        jadd_affine(acc, acc, gx, gy);
        started = 1;
      }
    }
}

typedef struct {
  const uint64_t* k;
  uint64_t* out;
} gen_ctx;

static void gen_range(void* vctx, int64_t lo, int64_t hi) {
  gen_ctx* c = (gen_ctx*)vctx;
  for (int64_t i = lo; i < hi; ++i) {
    jac acc;
    gen_mul(&acc, c->k + 4 * i);
    uint64_t a9[9];
    jto_affine_plain(&acc, a9);
    /* affine Montgomery rows (the identity, k = 0 mod r, is not a valid base) */
    fto_mont(c->out + 8 * i, a9, &FQ);
    fto_mont(c->out + 8 * i + 4, a9 + 4, &FQ);
  }
}

/* out (n, 2, 4): affine Montgomery rows of k_i G for plain scalars k_i in [1, r). */
void zo_g1_mul_generator(const uint64_t* k, uint64_t* out, int64_t n, int threads) {
  gen_ctx c = {k, out};
  parallel_for(n, threads, gen_range, &c);
}

/* ---- MSM (zkgpu/msm.py:156-207) ------------------------------------------------ */

typedef struct {
  const uint64_t* pts;   /* (n, 2, 4) affine Montgomery */
  const uint64_t* sc;    /* (n, 4) plain, reduced mod r */
  int64_t n;
  int w, win_lo;
  jac* sums;             /* one per window in [win_lo, win_hi) */
} msm_ctx;

static uint32_t window_digit(const uint64_t s[4], int win, int w) {
  int shift = win * w, limb = shift >> 6, off = shift & 63;
  if (limb >= 4) return 0;
  uint64_t v = s[limb] >> off;
  if (off + w > 64 && limb + 1 < 4) v |= s[limb + 1] << (64 - off);
  return (uint32_t)(v & ((1ull << w) - 1));
}

static void msm_windows(void* vctx, int64_t lo, int64_t hi) {
  msm_ctx* c = (msm_ctx*)vctx;
  int64_t nb = 1ll << c->w;
  jac* buckets = (jac*)malloc(sizeof(jac) * (size_t)nb);
  for (int64_t wi = lo; wi < hi; ++wi) {
    int win = c->win_lo + (int)wi;
    for (int64_t b = 0; b < nb; ++b) jset_identity(&buckets[b]);
    for (int64_t i = 0; i < c->n; ++i) {
      uint32_t d = window_digit(c->sc + 4 * i, win, c->w);
      if (d) jadd_affine(&buckets[d], &buckets[d], c->pts + 8 * i, c->pts + 8 * i + 4);
    }
    jac running, total;
    jset_identity(&running);
    jset_identity(&total);
    for (int64_t k = nb - 1; k > 0; --k) {
      jadd(&running, &running, &buckets[k]);
      jadd(&total, &total, &running);
    }
    c->sums[wi] = total;
  }
  free(buckets);
}

/*
 * Window sums win_lo .. win_hi - 1 of the reference's Pippenger, as Jacobian
 * Montgomery rows (out: (win_hi - win_lo, 3, 4)). scalars: plain, any 256-bit
 * value (reduced mod r here).
 */
int zo_msm_window_sums(const uint64_t* points, const uint64_t* scalars, int64_t n, int w,
                       int win_lo, int win_hi, int threads, uint64_t* out) {
  if (w < 1 || w > 20 || win_hi < win_lo) return -1;
  uint64_t* sc = (uint64_t*)malloc((size_t)32 * (n > 0 ? n : 1));
  for (int64_t i = 0; i < n; ++i) {
    memcpy(sc + 4 * i, scalars + 4 * i, 32);
    freduce_full(sc + 4 * i, &FR);
  }
  jac* sums = (jac*)malloc(sizeof(jac) * (size_t)(win_hi - win_lo > 0 ? win_hi - win_lo : 1));
  msm_ctx c = {points, sc, n, w, win_lo, sums};
  parallel_for(win_hi - win_lo, threads, msm_windows, &c);
  memcpy(out, sums, sizeof(jac) * (size_t)(win_hi - win_lo));
  free(sums);
  free(sc);
  return 0;
}

/* The full MSM: window sums, Horner (zkgpu/msm.py:180-193), affine result out9. */
int zo_msm(const uint64_t* points, const uint64_t* scalars, int64_t n, int w, int threads,
           uint64_t* out9) {
  if (n == 0) {
    memset(out9, 0, 72);
    out9[8] = 1;
    return 0;
  }
  int W = (254 + w - 1) / w;
  jac* sums = (jac*)malloc(sizeof(jac) * (size_t)W);
  if (zo_msm_window_sums(points, scalars, n, w, 0, W, threads, (uint64_t*)sums) != 0) {
    free(sums);
    return -1;
  }
  jac acc = sums[W - 1];
  for (int win = W - 2; win >= 0; --win) {
    for (int k = 0; k < w; ++k) jdouble(&acc, &acc);
    jadd(&acc, &acc, &sums[win]);
  }
  jto_affine_plain(&acc, out9);
  free(sums);
  return 0;
}
