// curve.cuh — BN254 G1 (y^2 = x^3 + 3 over Fq) point arithmetic.
//
// Two coordinate systems:
//   * Jacobian (X, Y, Z), affine (X/Z^2, Y/Z^3), Z = 0 the identity stored as
//     (ONE, ONE, 0). The element-wise point API must reproduce the
//     reference's exact Jacobian coordinates, so these formulas are the EFD
//     ones the reference uses (zkgpu/curve.py:236-303), with its special
//     cases, evaluated to the same field values.
//   * XYZZ (X, Y, ZZ, ZZZ), affine (X/ZZ, Y/ZZZ), ZZ^3 = ZZZ^2, ZZ = 0 the
//     identity. Used inside the MSM, whose output is compared only as an
//     affine point: mixed addition costs 8M + 2S instead of Jacobian's 7M + 4S
//     and full addition 12M + 2S instead of 11M + 5S (EFD "xyzz" formulas
//     madd-2008-s, add-2008-s, dbl-2008-s-1, mdbl-2008-s-1 with a = 0).
#pragma once
#include "field.cuh"

namespace zkb {

using G1F = FqP;

struct Jac {
  uint32_t x[8], y[8], z[8];
};
struct Aff {
  uint32_t x[8], y[8];
};
struct Xyzz {
  uint32_t x[8], y[8], zz[8], zzz[8];
};

// ---- loads and stores (Montgomery rows, 32 bytes per coordinate) ----------

__device__ __forceinline__ void jac_load(Jac& p, const uint64_t* src) {
  fe_load(p.x, src);
  fe_load(p.y, src + 4);
  fe_load(p.z, src + 8);
}
__device__ __forceinline__ void jac_store(uint64_t* dst, const Jac& p) {
  fe_store(dst, p.x);
  fe_store(dst + 4, p.y);
  fe_store(dst + 8, p.z);
}
__device__ __forceinline__ void aff_load(Aff& p, const uint64_t* src) {
  fe_load(p.x, src);
  fe_load(p.y, src + 4);
}
__device__ __forceinline__ void aff_load_nc(Aff& p, const uint64_t* src) {
  fe_load_nc(p.x, src);
  fe_load_nc(p.y, src + 4);
}
__device__ __forceinline__ void xyzz_load(Xyzz& p, const uint64_t* src) {
  fe_load(p.x, src);
  fe_load(p.y, src + 4);
  fe_load(p.zz, src + 8);
  fe_load(p.zzz, src + 12);
}
__device__ __forceinline__ void xyzz_store(uint64_t* dst, const Xyzz& p) {
  fe_store(dst, p.x);
  fe_store(dst + 4, p.y);
  fe_store(dst + 8, p.zz);
  fe_store(dst + 12, p.zzz);
}

// ---- Jacobian (reference formulas) -----------------------------------------

__device__ __forceinline__ void jac_set_identity(Jac& r) {
  G1F f;
  fe_one(r.x, f);
  fe_one(r.y, f);
  fe_zero(r.z);
}

// 2P, EFD dbl-2009-l (zkgpu/curve.py:236-252): A = X1^2, B = Y1^2, C = B^2,
// D = 2((X1 + B)^2 - A - C), E = 3A, F = E^2, X3 = F - 2D,
// Y3 = E (D - X3) - 8C, Z3 = 2 Y1 Z1. Z1 = 0 or Y1 = 0 gives the identity.
static __device__ __noinline__ void jac_double(Jac& r, const Jac& p) {
  G1F f;
  if (fe_is_zero(p.z) || fe_is_zero(p.y)) {
    jac_set_identity(r);
    return;
  }
  uint32_t a[8], b[8], c[8], d[8], e[8], t[8], x3[8], y3[8], z3[8];
  fe_sqr(a, p.x, f);
  fe_sqr(b, p.y, f);
  fe_sqr(c, b, f);
  fe_add(t, p.x, b, f);
  fe_sqr(t, t, f);
  fe_sub(t, t, a, f);
  fe_sub(t, t, c, f);
  fe_dbl(d, t, f);
  fe_dbl(e, a, f);
  fe_add(e, e, a, f);
  fe_sqr(x3, e, f);      // F
  fe_dbl(t, d, f);
  fe_sub(x3, x3, t, f);  // X3 = F - 2D
  fe_sub(t, d, x3, f);
  fe_mul(y3, e, t, f);
  fe_dbl(t, c, f);       // 2C
  fe_dbl(t, t, f);       // 4C
  fe_dbl(t, t, f);       // 8C
  fe_sub(y3, y3, t, f);
  fe_mul(t, p.y, p.z, f);
  fe_dbl(z3, t, f);
  fe_copy(r.x, x3);
  fe_copy(r.y, y3);
  fe_copy(r.z, z3);
}

// P + Q, EFD add-2007-bl (zkgpu/curve.py:255-281): Z1Z1 = Z1^2, Z2Z2 = Z2^2,
// U1 = X1 Z2Z2, U2 = X2 Z1Z1, S1 = Y1 Z2 Z2Z2, S2 = Y2 Z1 Z1Z1, H = U2 - U1,
// I = (2H)^2, J = H I, r = 2(S2 - S1), V = U1 I, X3 = r^2 - J - 2V,
// Y3 = r (V - X3) - 2 S1 J, Z3 = ((Z1 + Z2)^2 - Z1Z1 - Z2Z2) H.
// H = 0: equal points double, inverse points give the identity.
static __device__ __noinline__ void jac_add(Jac& r, const Jac& p, const Jac& q) {
  G1F f;
  if (fe_is_zero(p.z)) {
    r = q;
    return;
  }
  if (fe_is_zero(q.z)) {
    r = p;
    return;
  }
  uint32_t z1z1[8], z2z2[8], u1[8], u2[8], s1[8], s2[8], h[8], rr[8], i[8], j[8], v[8], t[8];
  fe_sqr(z1z1, p.z, f);
  fe_sqr(z2z2, q.z, f);
  fe_mul(u1, p.x, z2z2, f);
  fe_mul(u2, q.x, z1z1, f);
  fe_mul(s1, p.y, q.z, f);
  fe_mul(s1, s1, z2z2, f);
  fe_mul(s2, q.y, p.z, f);
  fe_mul(s2, s2, z1z1, f);
  fe_sub(h, u2, u1, f);
  fe_sub(rr, s2, s1, f);
  fe_dbl(rr, rr, f);
  if (fe_is_zero(h)) {
    if (fe_is_zero(rr)) {
      jac_double(r, p);
    } else {
      jac_set_identity(r);
    }
    return;
  }
  fe_dbl(t, h, f);
  fe_sqr(i, t, f);
  fe_mul(j, h, i, f);
  fe_mul(v, u1, i, f);
  uint32_t x3[8], y3[8], z3[8];
  fe_sqr(x3, rr, f);
  fe_sub(x3, x3, j, f);
  fe_dbl(t, v, f);
  fe_sub(x3, x3, t, f);
  fe_sub(t, v, x3, f);
  fe_mul(y3, rr, t, f);
  fe_mul(t, s1, j, f);
  fe_dbl(t, t, f);
  fe_sub(y3, y3, t, f);
  fe_add(t, p.z, q.z, f);
  fe_sqr(z3, t, f);
  fe_sub(z3, z3, z1z1, f);
  fe_sub(z3, z3, z2z2, f);
  fe_mul(z3, z3, h, f);
  fe_copy(r.x, x3);
  fe_copy(r.y, y3);
  fe_copy(r.z, z3);
}

// P + (x2, y2) for an affine, non-identity Q, EFD madd-2007-bl
// (zkgpu/curve.py:284-303): Z1Z1 = Z1^2, U2 = x2 Z1Z1, S2 = y2 Z1 Z1Z1,
// H = U2 - X1, HH = H^2, I = 4 HH, J = H I, r = 2(S2 - Y1), V = X1 I,
// X3 = r^2 - J - 2V, Y3 = r (V - X3) - 2 Y1 J, Z3 = (Z1 + H)^2 - Z1Z1 - HH.
// Z1 = 0 gives (x2, y2, ONE).
static __device__ __noinline__ void jac_add_affine(Jac& r, const Jac& p, const Aff& q) {
  G1F f;
  if (fe_is_zero(p.z)) {
    fe_copy(r.x, q.x);
    fe_copy(r.y, q.y);
    fe_one(r.z, f);
    return;
  }
  uint32_t z1z1[8], u2[8], s2[8], h[8], hh[8], i[8], j[8], rr[8], v[8], t[8];
  fe_sqr(z1z1, p.z, f);
  fe_mul(u2, q.x, z1z1, f);
  fe_mul(s2, q.y, p.z, f);
  fe_mul(s2, s2, z1z1, f);
  fe_sub(h, u2, p.x, f);
  fe_sub(rr, s2, p.y, f);
  fe_dbl(rr, rr, f);
  if (fe_is_zero(h)) {
    if (fe_is_zero(rr)) {
      jac_double(r, p);
    } else {
      jac_set_identity(r);
    }
    return;
  }
  fe_sqr(hh, h, f);
  fe_dbl(i, hh, f);
  fe_dbl(i, i, f);
  fe_mul(j, h, i, f);
  fe_mul(v, p.x, i, f);
  uint32_t x3[8], y3[8], z3[8];
  fe_sqr(x3, rr, f);
  fe_sub(x3, x3, j, f);
  fe_dbl(t, v, f);
  fe_sub(x3, x3, t, f);
  fe_sub(t, v, x3, f);
  fe_mul(y3, rr, t, f);
  fe_mul(t, p.y, j, f);
  fe_dbl(t, t, f);
  fe_sub(y3, y3, t, f);
  fe_add(t, p.z, h, f);
  fe_sqr(z3, t, f);
  fe_sub(z3, z3, z1z1, f);
  fe_sub(z3, z3, hh, f);
  fe_copy(r.x, x3);
  fe_copy(r.y, y3);
  fe_copy(r.z, z3);
}

// ---- XYZZ (MSM internals) ---------------------------------------------------

__device__ __forceinline__ void xyzz_set_identity(Xyzz& r) {
  fe_zero(r.x);
  fe_zero(r.y);
  fe_zero(r.zz);
  fe_zero(r.zzz);
}

__device__ __forceinline__ bool xyzz_is_identity(const Xyzz& p) { return fe_is_zero(p.zz); }

__device__ __forceinline__ void xyzz_from_affine(Xyzz& r, const Aff& q) {
  G1F f;
  fe_copy(r.x, q.x);
  fe_copy(r.y, q.y);
  fe_one(r.zz, f);
  fe_one(r.zzz, f);
}

// Products in the XYZZ formulas go through a policy M: InlineMul expands
// every Montgomery product in place; CallMul calls one shared copy of it.
// The bucket kernels run one mixed addition per sorted pair in a loop; with
// its ten products (and the rare doubling path's eight) expanded, the loop
// body outgrows the SM's instruction cache and warps stall on instruction
// fetch. With CallMul the body calls one shared copy of the product
// (fe_mul_shared).
struct InlineMul {
  __device__ __forceinline__ static void mul(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
    fe_mul(r, a, b, G1F{});
  }
  __device__ __forceinline__ static void sqr(uint32_t r[8], const uint32_t a[8]) { fe_sqr(r, a, G1F{}); }
  // r = a b + c d (one Montgomery reduction, fe_mul2)
  __device__ __forceinline__ static void mul2(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                              const uint32_t c[8], const uint32_t d[8]) {
    fe_mul2(r, a, b, c, d, G1F{});
  }
};

struct CallMul {
  __device__ __forceinline__ static void mul(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
    fe_mul_shared(r, a, b, G1F{});
  }
  __device__ __forceinline__ static void sqr(uint32_t r[8], const uint32_t a[8]) {
    fe_sqr_shared(r, a, G1F{});
  }
  __device__ __forceinline__ static void mul2(uint32_t r[8], const uint32_t a[8], const uint32_t b[8],
                                              const uint32_t c[8], const uint32_t d[8]) {
    fe_mul2_shared(r, a, b, c, d, G1F{});
  }
};

// 2(x, y) for an affine point, mdbl-2008-s-1: U = 2y, V = U^2, W = U V,
// S = x V, M = 3 x^2, X3 = M^2 - 2S, Y3 = M (S - X3) - W y, ZZ3 = V, ZZZ3 = W.
template <class M = InlineMul>
__device__ __forceinline__ void xyzz_mdbl(Xyzz& r, const Aff& q) {
  G1F f;
  uint32_t u[8], v[8], w[8], s[8], m[8], t[8];
  fe_dbl(u, q.y, f);
  M::sqr(v, u);
  M::mul(w, u, v);
  M::mul(s, q.x, v);
  M::sqr(m, q.x);
  fe_dbl(t, m, f);
  fe_add(m, m, t, f);
  M::sqr(r.x, m);
  fe_dbl(t, s, f);
  fe_sub(r.x, r.x, t, f);
  fe_sub(t, s, r.x, f);
  fe_p_minus(u, q.y, f);
  M::mul2(r.y, m, t, w, u);  // M (S - X3) - W y
  fe_copy(r.zz, v);
  fe_copy(r.zzz, w);
}

// 2P, dbl-2008-s-1 (a = 0): U = 2Y, V = U^2, W = U V, S = X V, M = 3 X^2,
// X3 = M^2 - 2S, Y3 = M (S - X3) - W Y, ZZ3 = V ZZ, ZZZ3 = W ZZZ.
template <class M = InlineMul>
__device__ __forceinline__ void xyzz_dbl(Xyzz& r, const Xyzz& p) {
  G1F f;
  if (fe_is_zero(p.zz) || fe_is_zero(p.y)) {
    xyzz_set_identity(r);
    return;
  }
  uint32_t u[8], v[8], w[8], s[8], m[8], t[8];
  fe_dbl(u, p.y, f);
  M::sqr(v, u);
  M::mul(w, u, v);
  M::mul(s, p.x, v);
  M::sqr(m, p.x);
  fe_dbl(t, m, f);
  fe_add(m, m, t, f);
  uint32_t x3[8], y3[8];
  M::sqr(x3, m);
  fe_dbl(t, s, f);
  fe_sub(x3, x3, t, f);
  fe_sub(t, s, x3, f);
  fe_p_minus(u, p.y, f);
  M::mul2(y3, m, t, w, u);  // M (S - X3) - W Y
  M::mul(r.zz, v, p.zz);
  M::mul(r.zzz, w, p.zzz);
  fe_copy(r.x, x3);
  fe_copy(r.y, y3);
}

// 2P in Jacobian coordinates with the products of M: dbl-2009-l as
// jac_double (2 products and 5 squarings, against 6 and 3 for xyzz_dbl).
// For a chain of doublings on one thread (the MSM's final combination).
template <class M>
__device__ __forceinline__ void jac_dbl_m(Jac& r, const Jac& p) {
  G1F f;
  if (fe_is_zero(p.z) || fe_is_zero(p.y)) {
    jac_set_identity(r);
    return;
  }
  uint32_t a[8], b[8], c[8], d[8], e[8], t[8], x3[8], y3[8], z3[8];
  M::sqr(a, p.x);
  M::sqr(b, p.y);
  M::sqr(c, b);
  fe_add(t, p.x, b, f);
  M::sqr(t, t);
  fe_sub(t, t, a, f);
  fe_sub(t, t, c, f);
  fe_dbl(d, t, f);
  fe_dbl(e, a, f);
  fe_add(e, e, a, f);
  M::sqr(x3, e);
  fe_dbl(t, d, f);
  fe_sub(x3, x3, t, f);
  fe_sub(t, d, x3, f);
  M::mul(y3, e, t);
  fe_dbl(t, c, f);
  fe_dbl(t, t, f);
  fe_dbl(t, t, f);
  fe_sub(y3, y3, t, f);
  M::mul(t, p.y, p.z);
  fe_dbl(z3, t, f);
  fe_copy(r.x, x3);
  fe_copy(r.y, y3);
  fe_copy(r.z, z3);
}

// XYZZ (x = X / ZZ, y = Y / ZZZ, ZZ^3 = ZZZ^2) to Jacobian: (X ZZ^2, Y ZZ^3, ZZZ),
// since (X ZZ^2) / ZZZ^2 = X / ZZ and (Y ZZ^3) / ZZZ^3 = Y / ZZZ. No inversion.
template <class M>
__device__ __forceinline__ void xyzz_to_jac(Jac& r, const Xyzz& p) {
  if (xyzz_is_identity(p)) {
    jac_set_identity(r);
    return;
  }
  uint32_t zz2[8], zz3[8];
  M::sqr(zz2, p.zz);
  M::mul(zz3, zz2, p.zz);
  M::mul(r.x, p.x, zz2);
  M::mul(r.y, p.y, zz3);
  fe_copy(r.z, p.zzz);
}

// Jacobian to XYZZ: (X, Y, Z^2, Z^3).
template <class M>
__device__ __forceinline__ void jac_to_xyzz(Xyzz& r, const Jac& p) {
  if (fe_is_zero(p.z)) {
    xyzz_set_identity(r);
    return;
  }
  M::sqr(r.zz, p.z);
  M::mul(r.zzz, r.zz, p.z);
  fe_copy(r.x, p.x);
  fe_copy(r.y, p.y);
}

// P += (x2, y2), madd-2008-s: P' = x2 ZZ1 - X1, R = y2 ZZZ1 - Y1, PP = P'^2,
// PPP = P' PP, Q = X1 PP, X3 = R^2 - PPP - 2Q, Y3 = R (Q - X3) - Y1 PPP,
// ZZ3 = ZZ1 PP, ZZZ3 = ZZZ1 PPP. Special cases: P the identity gives Q;
// P' = 0 means equal x: doubling (R = 0) or the identity (R != 0).
template <class M = InlineMul>
__device__ __forceinline__ void xyzz_add_affine(Xyzz& acc, const Aff& q) {
  G1F f;
  if (fe_is_zero(acc.zz)) {
    xyzz_from_affine(acc, q);
    return;
  }
  uint32_t pp[8], r[8], t[8];
  M::mul(pp, q.x, acc.zz);
  fe_sub(pp, pp, acc.x, f);   // P'
  M::mul(r, q.y, acc.zzz);
  fe_sub(r, r, acc.y, f);     // R
  if (fe_is_zero(pp)) {
    if (fe_is_zero(r)) {
      xyzz_mdbl<M>(acc, q);
    } else {
      xyzz_set_identity(acc);
    }
    return;
  }
  uint32_t ppp[8], qq[8];
  M::sqr(t, pp);           // PP
  M::mul(ppp, pp, t);      // PPP
  M::mul(qq, acc.x, t);    // Q
  M::mul(acc.zz, acc.zz, t);
  M::mul(acc.zzz, acc.zzz, ppp);
  M::sqr(t, r);
  fe_sub(t, t, ppp, f);
  fe_sub(t, t, qq, f);
  fe_sub(t, t, qq, f);        // X3
  fe_sub(qq, qq, t, f);        // Q - X3
  fe_p_minus(acc.y, acc.y, f);  // -Y1 as p - Y1
  M::mul2(acc.y, r, qq, acc.y, ppp);  // R (Q - X3) - Y1 PPP
  fe_copy(acc.x, t);
}

// r = P + Q, add-2008-s: U1 = X1 ZZ2, U2 = X2 ZZ1, S1 = Y1 ZZZ2, S2 = Y2 ZZZ1,
// P' = U2 - U1, R = S2 - S1, PP = P'^2, PPP = P' PP, Q = U1 PP,
// X3 = R^2 - PPP - 2Q, Y3 = R (Q - X3) - S1 PPP, ZZ3 = ZZ1 ZZ2 PP,
// ZZZ3 = ZZZ1 ZZZ2 PPP. r may alias p or q.
template <class M = InlineMul>
__device__ __forceinline__ void xyzz_add(Xyzz& r, const Xyzz& p, const Xyzz& q) {
  G1F f;
  if (fe_is_zero(q.zz)) {
    r = p;
    return;
  }
  if (fe_is_zero(p.zz)) {
    r = q;
    return;
  }
  uint32_t u1[8], s1[8], pp[8], rr[8], t[8];
  M::mul(u1, p.x, q.zz);
  M::mul(pp, q.x, p.zz);
  fe_sub(pp, pp, u1, f);      // P'
  M::mul(s1, p.y, q.zzz);
  M::mul(rr, q.y, p.zzz);
  fe_sub(rr, rr, s1, f);      // R
  if (fe_is_zero(pp)) {
    if (fe_is_zero(rr)) {
      xyzz_dbl<M>(r, p);
    } else {
      xyzz_set_identity(r);
    }
    return;
  }
  uint32_t ppp[8], qq[8], zz[8], zzz[8];
  M::sqr(t, pp);           // PP
  M::mul(ppp, pp, t);      // PPP
  M::mul(qq, u1, t);       // Q
  M::mul(zz, p.zz, q.zz);
  M::mul(zz, zz, t);
  M::mul(zzz, p.zzz, q.zzz);
  M::mul(zzz, zzz, ppp);
  M::sqr(t, rr);
  fe_sub(t, t, ppp, f);
  fe_sub(t, t, qq, f);
  fe_sub(t, t, qq, f);        // X3
  fe_sub(qq, qq, t, f);        // Q - X3
  fe_p_minus(s1, s1, f);       // -S1 as p - S1
  M::mul2(r.y, rr, qq, s1, ppp);  // R (Q - X3) - S1 PPP
  fe_copy(r.x, t);
  fe_copy(r.zz, zz);
  fe_copy(r.zzz, zzz);
}

// The MSM's affine bucket lists mark the point at infinity by bit 255 of x,
// which a canonical coordinate (below q < 2^254) never sets.
__device__ __forceinline__ bool aff_is_inf(const Aff& p) { return (p.x[7] >> 31) != 0; }

// Negate an affine point: (x, -y).
__device__ __forceinline__ void aff_neg(Aff& q) {
  G1F f;
  fe_neg(q.y, q.y, f);
}

// y^2 == x^3 + 3 for an affine point in Montgomery form.
__device__ __forceinline__ bool aff_on_curve(const Aff& q) {
  G1F f;
  uint32_t lhs[8], rhs[8], three[8];
  fe_sqr(lhs, q.y, f);
  fe_sqr(rhs, q.x, f);
  fe_mul(rhs, rhs, q.x, f);
  fe_one(three, f);
  fe_add(three, three, three, f);  // 2
  uint32_t one[8];
  fe_one(one, f);
  fe_add(three, three, one, f);    // 3
  fe_add(rhs, rhs, three, f);
  return fe_eq(lhs, rhs);
}

}  // namespace zkb
