// G1 point arithmetic for BN254 and BLS12-381 (short Weierstrass, a = 0) on the device.
//
// Buckets accumulate in extended Jacobian "XYZZ" coordinates (x = X/ZZ, y = Y/ZZZ,
// ZZ^3 = ZZZ^2), formulas madd-2008-s, add-2008-s, dbl-2008-s-1 and mdbl-2008-s-1 from the
// Explicit-Formulas Database. The reference accumulates in homogeneous projective
// coordinates (lib/cbits/curves/g1/proj/bn128_G1_proj.c:333-373 madd, :272-313 add); both
// compute the same group element, and every output is converted to the canonical
// representation the reference produces, so results are bit-identical.
//
// Special cases mirror the reference's madd (bn128_G1_proj.c:334-358): an empty bucket takes
// the point, an affine (0,0) input is the identity and is skipped, equal points double,
// opposite points give the identity.
#pragma once
#include "zkb_field.cuh"

namespace zkb {

struct BN254 {
  using Fp = BnFp;
  using Fr = BnFr;
  static constexpr int FP_WORDS = 8;      // 32-bit words per Fp element
  static constexpr int SCALAR_BITS = 254; // r < 2^254
  static constexpr int ID = 0;
};
struct BLS12_381 {
  using Fp = BlsFp;
  using Fr = BlsFr;
  static constexpr int FP_WORDS = 12;
  static constexpr int SCALAR_BITS = 255; // r < 2^255
  static constexpr int ID = 1;
};

template <class F>
struct Affine {
  Fe<F> x, y;
};

template <class F>
struct Xyzz {
  Fe<F> X, Y, ZZ, ZZZ;   // ZZ == 0 encodes the identity
};

template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_inf() {
  Xyzz<F> r;
  r.X = fe_zero<F>(); r.Y = fe_zero<F>(); r.ZZ = fe_zero<F>(); r.ZZZ = fe_zero<F>();
  return r;
}
// The identity is ZZ == 0 exactly, also on a redundant-range field: it is only ever set by
// xyzz_inf(), and no formula produces a ZZ that is 0 mod p otherwise (ZZ3 is a product of
// non-zero factors; neither curve group has a point with y = 0), so a ZZ equal to p cannot occur.
template <class F>
__device__ __forceinline__ bool xyzz_is_inf(const Xyzz<F>& p) { return fe_is_zero(p.ZZ); }

template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_from_affine(const Affine<F>& a) {
  Xyzz<F> r;
  r.X = a.x; r.Y = a.y; r.ZZ = fe_one<F>(); r.ZZZ = fe_one<F>();
  return r;
}

// 2*(x, y) for an affine point, mdbl-2008-s-1 (a = 0); rare inside bucket sums, kept out of line
template <class F>
__device__ __noinline__ Xyzz<F> xyzz_dbl_affine(const Affine<F>& a) {
  const Fe<F> U = fe_dbl(a.y);
  const Fe<F> V = fe_sqr(U);
  const Fe<F> W = fe_mul(U, V);
  const Fe<F> S = fe_mul(a.x, V);
  const Fe<F> xx = fe_sqr(a.x);
  const Fe<F> M = fe_add(fe_dbl(xx), xx);
  Xyzz<F> r;
  r.X = fe_sub(fe_sqr(M), fe_dbl(S));
  r.Y = fe_sub(fe_mul(M, fe_sub(S, r.X)), fe_mul(W, a.y));
  r.ZZ = V;
  r.ZZZ = W;
  return r;
}

// 2*P, dbl-2008-s-1 (a = 0); the identity maps to itself (ZZ3 = V*ZZ1 = 0); out of line
template <class F>
__device__ __noinline__ Xyzz<F> xyzz_dbl(const Xyzz<F>& p) {
  const Fe<F> U = fe_dbl(p.Y);
  const Fe<F> V = fe_sqr(U);
  const Fe<F> W = fe_mul(U, V);
  const Fe<F> S = fe_mul(p.X, V);
  const Fe<F> xx = fe_sqr(p.X);
  const Fe<F> M = fe_add(fe_dbl(xx), xx);
  Xyzz<F> r;
  r.X = fe_sub(fe_sqr(M), fe_dbl(S));
  r.Y = fe_sub(fe_mul(M, fe_sub(S, r.X)), fe_mul(W, p.Y));
  r.ZZ = fe_mul(V, p.ZZ);
  r.ZZZ = fe_mul(W, p.ZZZ);
  return r;
}

// acc += a for an affine a that is not (0, 0); madd-2008-s with exact special cases
template <class F>
__device__ __forceinline__ void xyzz_madd(Xyzz<F>& acc, const Affine<F>& a) {
  if (xyzz_is_inf(acc)) { acc = xyzz_from_affine(a); return; }
  Fe<F> U2, S2;
  fe_mul2(U2, a.x, acc.ZZ, S2, a.y, acc.ZZZ);
  const Fe<F> P = fe_sub(U2, acc.X);
  const Fe<F> R = fe_sub(S2, acc.Y);
  if (fe_is_zero_mod(P)) {
    if (fe_is_zero_mod(R)) acc = xyzz_dbl_affine(a);
    else acc = xyzz_inf<F>();
    return;
  }
  Fe<F> PP, RR, PPP, Q;
  fe_sqr2(PP, P, RR, R);
  fe_mul2(PPP, P, PP, Q, acc.X, PP);
  const Fe<F> X3 = fe_sub(fe_sub(RR, PPP), fe_dbl(Q));
  Fe<F> t1, t2;
  fe_mul2(t1, R, fe_sub(Q, X3), t2, acc.Y, PPP);
  fe_mul2(acc.ZZ, acc.ZZ, PP, acc.ZZZ, acc.ZZZ, PPP);
  acc.X = X3;
  acc.Y = fe_sub(t1, t2);
}

// acc += q, add-2008-s with exact special cases (single products: pairing them was measured 15%
// slower in the group FFT's scalar multiplications)
template <class F>
__device__ __forceinline__ void xyzz_add(Xyzz<F>& acc, const Xyzz<F>& q) {
  if (xyzz_is_inf(q)) return;
  if (xyzz_is_inf(acc)) { acc = q; return; }
  const Fe<F> U1 = fe_mul(acc.X, q.ZZ);
  const Fe<F> U2 = fe_mul(q.X, acc.ZZ);
  const Fe<F> S1 = fe_mul(acc.Y, q.ZZZ);
  const Fe<F> S2 = fe_mul(q.Y, acc.ZZZ);
  const Fe<F> P = fe_sub(U2, U1);
  const Fe<F> R = fe_sub(S2, S1);
  if (fe_is_zero_mod(P)) {
    if (fe_is_zero_mod(R)) acc = xyzz_dbl(acc);
    else acc = xyzz_inf<F>();
    return;
  }
  const Fe<F> PP = fe_sqr(P);
  const Fe<F> PPP = fe_mul(P, PP);
  const Fe<F> Q = fe_mul(U1, PP);
  Fe<F> X3 = fe_sub(fe_sub(fe_sqr(R), PPP), fe_dbl(Q));
  const Fe<F> Y3 = fe_sub(fe_mul(R, fe_sub(Q, X3)), fe_mul(S1, PPP));
  acc.ZZ = fe_mul(fe_mul(acc.ZZ, q.ZZ), PP);
  acc.ZZZ = fe_mul(fe_mul(acc.ZZZ, q.ZZZ), PPP);
  acc.X = X3;
  acc.Y = Y3;
}

// canonical coordinates (values in [0, p)) of a point whose field keeps a redundant range
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_canon(const Xyzz<F>& p) {
  Xyzz<F> r;
  r.X = fe_canon(p.X); r.Y = fe_canon(p.Y); r.ZZ = fe_canon(p.ZZ); r.ZZZ = fe_canon(p.ZZZ);
  return r;
}

// acc += q with the independent products in pairs (one call computes two, interleaving their
// reduction chains): the MSM's bucket merge and reduction kernels, whose short sequential chains
// of additions run at low occupancy, where the halved dependency depth pays
template <class F>
__device__ __forceinline__ void xyzz_add_paired(Xyzz<F>& acc, const Xyzz<F>& q) {
  if (xyzz_is_inf(q)) return;
  if (xyzz_is_inf(acc)) { acc = q; return; }
  Fe<F> U1, U2, S1, S2;
  fe_mul2(U1, acc.X, q.ZZ, U2, q.X, acc.ZZ);
  fe_mul2(S1, acc.Y, q.ZZZ, S2, q.Y, acc.ZZZ);
  const Fe<F> P = fe_sub(U2, U1);
  const Fe<F> R = fe_sub(S2, S1);
  if (fe_is_zero_mod(P)) {
    if (fe_is_zero_mod(R)) acc = xyzz_dbl(acc);
    else acc = xyzz_inf<F>();
    return;
  }
  Fe<F> PP, RR, PPP, Q, zz, zzz;
  fe_sqr2(PP, P, RR, R);
  fe_mul2(PPP, P, PP, Q, U1, PP);
  const Fe<F> X3 = fe_sub(fe_sub(RR, PPP), fe_dbl(Q));
  Fe<F> t1, t2;
  fe_mul2(t1, R, fe_sub(Q, X3), t2, S1, PPP);
  fe_mul2(zz, acc.ZZ, q.ZZ, zzz, acc.ZZZ, q.ZZZ);
  fe_mul2(acc.ZZ, zz, PP, acc.ZZZ, zzz, PPP);
  acc.X = X3;
  acc.Y = fe_sub(t1, t2);
}

template <class F>
__device__ __forceinline__ Affine<F> affine_neg(const Affine<F>& a) {
  Affine<F> r;
  r.x = a.x;
  r.y = fe_neg(a.y);
  return r;
}

// ------------------------------------------------------------------------ memory layout
// affine: x | y (2*FP_WORDS words, the reference's layout); XYZZ: X | Y | ZZ | ZZZ.
template <class F>
__device__ __forceinline__ Affine<F> affine_load(const uint32_t* __restrict__ p) {
  Affine<F> a;
  a.x = fe_load_nc<F>(p);
  a.y = fe_load_nc<F>(p + F::N);
  return a;
}
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_load(const uint32_t* __restrict__ p) {
  Xyzz<F> r;
  r.X = fe_load<F>(p);
  r.Y = fe_load<F>(p + F::N);
  r.ZZ = fe_load<F>(p + 2 * F::N);
  r.ZZZ = fe_load<F>(p + 3 * F::N);
  return r;
}
template <class F>
__device__ __forceinline__ void xyzz_store(uint32_t* __restrict__ p, const Xyzz<F>& a) {
  fe_store<F>(p, a.X);
  fe_store<F>(p + F::N, a.Y);
  fe_store<F>(p + 2 * F::N, a.ZZ);
  fe_store<F>(p + 3 * F::N, a.ZZZ);
}

}  // namespace zkb
