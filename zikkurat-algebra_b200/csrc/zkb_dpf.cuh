// Prime-field multiplication on the FP64 pipe: Montgomery products over 52-bit limbs held as
// exact integers in doubles.
//
// The 32-bit-limb product of zkb_field.cuh spends most of its ~590 instructions on carry
// propagation in the integer ALU. Here an element is L limbs of 52 bits (L = 5 for 254/255-bit
// fields, 8 for BLS12-381 Fp) and the Montgomery radix is R' = 2^(52 L). A 52 x 52-bit limb
// product is split exactly into high and low 52-bit halves with two fused multiply-adds:
//     h = fma_rz(a, b, 2^104)       = 2^104 + H 2^52     (rounding toward zero drops L)
//     l = fma_rn(a, b, 2^104 + 2^52 - h) = L + 2^52      (exact: the true value fits 53 bits)
// and the bit patterns of h and l carry H and L in their mantissas. Column sums of those bit
// patterns (minus the known exponent bits) accumulate in 64-bit integers without overflow
// (at most 4L + 1 terms of < 2^52 per column), followed by the usual word-by-word Montgomery
// reduction: the digits m_i = (t_i * (-p^-1)) mod 2^52 come from a 64-bit integer product, the
// products m_i * p from the same FMA split. Squarings take each cross product once, doubled.
//
// Bounds: inputs in [0, p) (canonical). Then a b + m p < p^2 + R' p, so
// (a b + m p) / R' < p (p / R' + 1) < 2p and one conditional subtraction gives the canonical
// result. Lazy field types (LAZY = true, zkb_field.cuh) take inputs in [0, 2p): then
// (a b + m p) / R' < p (4p / R' + 1) < 2p as well (R' >= 2^6 p for every field here), so the
// product stays in [0, 2p) without the subtraction. Every operation is an exact modular operation, so
// values converted back to the 32-bit-limb Montgomery form (radix R = 2^(32 N)) are the same
// field elements; conversions: into the FP64 form mont'(x R, R'^2 / R), back mont'(x R', R).
#pragma once
#include <mutex>

#include "zkb_curve.cuh"
#include "zkb_field.cuh"
#include "zkb_host_ec.h"

namespace zkb {

template <class P>
struct D52 {
  static constexpr int L = P::N == 8 ? 5 : 8;   // 52-bit limbs: 260 bits for 254/255-bit p, 416 for 381-bit p
  static constexpr uint64_t MASK = (1ull << 52) - 1;
  // bits [52k, 52k + 52) of p
  __host__ __device__ static constexpr uint64_t plimb(int k) {
    uint64_t r = 0;
    for (int b = 0; b < 52; b++) {
      const int bit = 52 * k + b;
      const int w = bit >> 5;
      if (w < P::N && ((P::mod(w) >> (bit & 31)) & 1u)) r |= 1ull << b;
    }
    return r;
  }
  // -p^-1 mod 2^52 (Newton iteration for the inverse mod 2^64)
  __host__ __device__ static constexpr uint64_t pinv() {
    const uint64_t p0 = (uint64_t)P::mod(0) | ((uint64_t)P::mod(1) << 32);
    uint64_t x = 1;
    for (int i = 0; i < 7; i++) x = x * (2 - p0 * x);
    return (0 - x) & MASK;
  }
};

template <class P>
struct FeD {
  uint64_t v[D52<P>::L];   // limbs < 2^52, value in [0, p)
};

static constexpr uint64_t DPF_B52 = 0x4330000000000000ull;    // bits of 2^52
static constexpr uint64_t DPF_B104 = 0x4670000000000000ull;   // bits of 2^104

// a * b = H 2^52 + L for 52-bit integers a, b held in doubles; returns the bit patterns
// bits(2^104) + H and bits(2^52) + L
__device__ __forceinline__ void dpf_split(double a, double b, uint64_t& hb, uint64_t& lb) {
  const double h = __fma_rz(a, b, 0x1p104);
  const double c = __dsub_rn(0x1.0000000000001p104, h);   // 2^104 + 2^52 - h = (1 - H) 2^52, exact
  const double l = __fma_rn(a, b, c);                      // L + 2^52, exact
  hb = (uint64_t)__double_as_longlong(h);
  lb = (uint64_t)__double_as_longlong(l);
}
__device__ __forceinline__ double dpf_to_double(uint64_t x) {   // x < 2^52
  return __dsub_rn(__longlong_as_double((long long)(x | DPF_B52)), 0x1p52);
}

// r - p if r >= p (r < 2p), limb-wise with borrows
template <class P>
__device__ __forceinline__ void fd_reduce_once(uint64_t (&r)[D52<P>::L]) {
  constexpr int L = D52<P>::L;
  uint64_t t[L];
  int64_t borrow = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const int64_t d = (int64_t)r[k] - (int64_t)D52<P>::plimb(k) - borrow;
    borrow = d < 0 ? 1 : 0;
    t[k] = (uint64_t)d & D52<P>::MASK;
  }
  if (!borrow) {
#pragma unroll
    for (int k = 0; k < L; k++) r[k] = t[k];
  }
}

// Field types with EXACT = true run their products on the FP64 pipe in the reference's own
// Montgomery radix R = 2^(32 N) instead of R' = 2^(52 L): the last reduction digit is
// 32 N - 52 (L - 1) bits wide (48 for 254/255-bit fields, 20 for BLS12-381 Fp), so the product
// is a drop-in for the 32-bit-limb one and data need no radix conversion.
template <class P, class = void>
struct ExactOf { static constexpr bool value = false; };
template <class P>
struct ExactOf<P, decltype((void)P::EXACT)> { static constexpr bool value = P::EXACT; };
template <class P>
inline constexpr bool exact_v = ExactOf<P>::value;

// Montgomery reduction of the 2L + 1 columns of a product (column k: sum of 52-bit pieces of
// weight 2^(52 k), < 2^57), word by word with 52-bit digits (the last one narrower for an EXACT
// field); canonical result (in [0, 2p) for a lazy field).
template <class P>
__device__ __forceinline__ FeD<P> fd_reduce(uint64_t (&col)[2 * D52<P>::L + 1]) {
  constexpr int L = D52<P>::L;
  constexpr uint64_t M = D52<P>::MASK;
  constexpr bool EX = exact_v<P>;
  constexpr int LD = EX ? 32 * P::N - 52 * (L - 1) : 52;   // width of the last digit
  uint64_t carry = 0;
#pragma unroll
  for (int i = 0; i < L; i++) {
    const bool narrow = EX && i == L - 1;
    const uint64_t dm = narrow ? ((1ull << LD) - 1) : M;
    const uint64_t v = col[i] + carry;
    // m_i = (t_i * (-p^-1)) mod 2^52 (2^LD for a narrow digit): a 64-bit integer product (IMAD
    // pipe, otherwise idle here)
    const double m = dpf_to_double(((v & dm) * D52<P>::pinv()) & dm);
    uint64_t hb, lb;
    uint64_t hprev;
    dpf_split(m, (double)D52<P>::plimb(0), hprev, lb);
    if (narrow) col[i] = v + lb - DPF_B52;          // low LD bits zero; bits LD.. are the result's
    else carry = (v + lb - DPF_B52) >> 52;          // the low 52 bits are zero now
#pragma unroll
    for (int j = 1; j < L; j++) {
      dpf_split(m, (double)D52<P>::plimb(j), hb, lb);
      col[i + j] += lb + hprev - (DPF_B52 + DPF_B104);
      hprev = hb;
    }
    col[i + L] += hprev - DPF_B104;
  }
  uint64_t r[L];
  if constexpr (EX) {
    // columns L-1 .. 2L-1 into 52-bit limbs, then the result is those bits from bit LD on
    uint64_t nl[L + 1];
    uint64_t c = 0;
#pragma unroll
    for (int k = 0; k <= L; k++) {
      const uint64_t v = col[L - 1 + k] + c;
      nl[k] = k < L ? (v & M) : v;
      c = v >> 52;
    }
#pragma unroll
    for (int k = 0; k < L; k++) r[k] = (nl[k] >> LD) | ((nl[k + 1] << (52 - LD)) & (k < L - 1 ? M : ~0ull));
  } else {
    uint64_t c = carry;
#pragma unroll
    for (int k = 0; k < L; k++) {
      const uint64_t v = col[L + k] + c;
      r[k] = k < L - 1 ? (v & M) : v;
      c = v >> 52;
    }
  }
  if constexpr (!lazy_v<P>) fd_reduce_once<P>(r);   // a lazy field keeps (ab + mp) / R < 2p
  FeD<P> out;
#pragma unroll
  for (int k = 0; k < L; k++) out.v[k] = r[k];
  return out;
}

template <class P>
__device__ __forceinline__ FeD<P> fd_mul_inl(const FeD<P>& ai, const FeD<P>& bi) {
  constexpr int L = D52<P>::L;
  double a[L], b[L];
#pragma unroll
  for (int k = 0; k < L; k++) { a[k] = dpf_to_double(ai.v[k]); b[k] = dpf_to_double(bi.v[k]); }
  uint64_t col[2 * L + 1];
#pragma unroll
  for (int k = 0; k < 2 * L + 1; k++) col[k] = 0;
  // product scanning: diagonal d holds products (i, d - i); low halves -> column d, high -> d + 1
#pragma unroll
  for (int d = 0; d <= 2 * L - 2; d++) {
    uint64_t slo = 0, shi = 0, blo = 0, bhi = 0;
#pragma unroll
    for (int i = 0; i < L; i++) {
      const int j = d - i;
      if (j < 0 || j >= L) continue;
      uint64_t hb, lb;
      dpf_split(a[i], b[j], hb, lb);
      slo += lb; shi += hb; blo += DPF_B52; bhi += DPF_B104;
    }
    col[d] += slo - blo;
    col[d + 1] += shi - bhi;
  }
  return fd_reduce<P>(col);
}

// a^2: each cross product a_i a_j (i < j) once, doubled; L (L + 1) / 2 limb products instead of L^2
template <class P>
__device__ __forceinline__ FeD<P> fd_sqr_inl(const FeD<P>& ai) {
  constexpr int L = D52<P>::L;
  double a[L];
#pragma unroll
  for (int k = 0; k < L; k++) a[k] = dpf_to_double(ai.v[k]);
  uint64_t col[2 * L + 1];
#pragma unroll
  for (int k = 0; k < 2 * L + 1; k++) col[k] = 0;
#pragma unroll
  for (int d = 0; d <= 2 * L - 2; d++) {
    uint64_t xlo = 0, xhi = 0, bx = 0;   // cross terms (doubled below)
    uint64_t slo = 0, shi = 0;           // the square term a_{d/2}^2
#pragma unroll
    for (int i = 0; i < L; i++) {
      const int j = d - i;
      if (j < i || j >= L) continue;
      uint64_t hb, lb;
      dpf_split(a[i], a[j], hb, lb);
      if (i == j) { slo = lb - DPF_B52; shi = hb - DPF_B104; }
      else { xlo += lb; xhi += hb; bx += 1; }
    }
    col[d] += 2 * (xlo - bx * DPF_B52) + slo;
    col[d + 1] += 2 * (xhi - bx * DPF_B104) + shi;
  }
  return fd_reduce<P>(col);
}

// Out of line for the same reason as fe_mul_call (instruction-cache footprint of point formulas).
template <class P>
__device__ __noinline__ FeD<P> fd_mul_call(const FeD<P> a, const FeD<P> b) { return fd_mul_inl<P>(a, b); }
template <class P>
__device__ __forceinline__ FeD<P> fd_mul(const FeD<P>& a, const FeD<P>& b) { return fd_mul_call<P>(a, b); }
template <class P>
__device__ __forceinline__ FeD<P> fd_sqr(const FeD<P>& a) { return fd_mul<P>(a, a); }

template <class P>
__device__ __forceinline__ FeD<P> fd_zero() {
  FeD<P> r;
#pragma unroll
  for (int k = 0; k < D52<P>::L; k++) r.v[k] = 0;
  return r;
}
template <class P>
__device__ __forceinline__ bool fd_is_zero(const FeD<P>& a) {
  uint64_t o = 0;
#pragma unroll
  for (int k = 0; k < D52<P>::L; k++) o |= a.v[k];
  return o == 0;
}

template <class P>
__device__ __forceinline__ FeD<P> fd_add(const FeD<P>& a, const FeD<P>& b) {
  constexpr int L = D52<P>::L;
  uint64_t r[L];
  uint64_t c = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const uint64_t s = a.v[k] + b.v[k] + c;
    r[k] = s & D52<P>::MASK;
    c = s >> 52;
  }
  r[L - 1] |= c << 52;   // a + b < 2p fits the top limb's spare bits
  fd_reduce_once<P>(r);
  FeD<P> out;
#pragma unroll
  for (int k = 0; k < L; k++) out.v[k] = r[k];
  return out;
}

template <class P>
__device__ __forceinline__ FeD<P> fd_sub(const FeD<P>& a, const FeD<P>& b) {
  constexpr int L = D52<P>::L;
  uint64_t r[L];
  int64_t borrow = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const int64_t d = (int64_t)a.v[k] - (int64_t)b.v[k] - borrow;
    borrow = d < 0 ? 1 : 0;
    r[k] = (uint64_t)d & D52<P>::MASK;
  }
  if (borrow) {   // a - b + p
    uint64_t c = 0;
#pragma unroll
    for (int k = 0; k < L; k++) {
      const uint64_t s = r[k] + D52<P>::plimb(k) + c;
      r[k] = s & D52<P>::MASK;
      c = s >> 52;
    }
  }
  FeD<P> out;
#pragma unroll
  for (int k = 0; k < L; k++) out.v[k] = r[k];
  return out;
}

template <class P>
__device__ __forceinline__ FeD<P> fd_dbl(const FeD<P>& a) { return fd_add<P>(a, a); }
template <class P>
__device__ __forceinline__ FeD<P> fd_neg(const FeD<P>& a) { return fd_sub<P>(fd_zero<P>(), a); }

// 32-bit words (N of them, value < 2^(32 N)) <-> 52-bit limbs, exact repacking
template <class P>
__device__ __forceinline__ FeD<P> fd_from_words(const Fe<P>& x) {
  constexpr int L = D52<P>::L;
  FeD<P> r;
#pragma unroll
  for (int k = 0; k < L; k++) {
    uint64_t acc = 0;
#pragma unroll
    for (int w = 0; w < P::N; w++) {
      const int lo = 32 * w - 52 * k;   // position of word w's bit 0 inside limb k
      if (lo <= -32 || lo >= 52) continue;
      const uint64_t word = x.v[w];
      acc |= lo >= 0 ? (word << lo) : (word >> (-lo));
    }
    r.v[k] = acc & D52<P>::MASK;
  }
  return r;
}
template <class P>
__device__ __forceinline__ Fe<P> fd_to_words(const FeD<P>& a) {
  constexpr int L = D52<P>::L;
  Fe<P> r;
#pragma unroll
  for (int w = 0; w < P::N; w++) {
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < L; k++) {
      const int lo = 52 * k - 32 * w;   // position of limb k's bit 0 inside word w
      if (lo >= 32 || lo <= -52) continue;
      acc |= lo >= 0 ? (a.v[k] << lo) : (a.v[k] >> (-lo));
    }
    r.v[w] = (uint32_t)acc;
  }
  return r;
}

// ------------------------------------------------------------ the FP64 flavour of a field
// BnFpD / BlsFpD have the modulus and word layout of BnFp / BlsFp, but Montgomery radix
// R' = 2^(52 L): values are x R' mod p in N 32-bit words (canonical), so additions, subtractions,
// comparisons and the point formulas of zkb_curve.cuh run unchanged on the integer pipes, and
// fe_mul dispatches to the FP64 product below (words repacked into 52-bit limbs and back).
// one / r2 are R' and R'^2 mod p.
#define ZKB_DPF_TABLE(name, n, ...)                                               \
  __host__ __device__ static constexpr uint32_t name(int i) {                    \
    constexpr uint32_t t[n] = {__VA_ARGS__};                                      \
    return t[i];                                                                  \
  }

struct BnFpD {
  static constexpr bool DPF = true;
  static constexpr int N = 8;
  static constexpr uint32_t n0 = BnFp::n0;
  __host__ __device__ static constexpr uint32_t mod(int i) { return BnFp::mod(i); }
  // 2^260 mod p, 2^520 mod p
  ZKB_DPF_TABLE(one, 8, 0xf6fce4b4u, 0x45520880u, 0xbaa989a8u, 0x49890849u, 0x818f014au, 0x85a9201du, 0x1bb7724fu, 0x1f16424eu)
  ZKB_DPF_TABLE(r2, 8, 0x1966eb04u, 0xb868a81du, 0x95018016u, 0x98e61561u, 0x0b4f898cu, 0xbfd53160u, 0x0d3a9969u, 0x0a8469a3u)
};
struct BlsFpD {
  static constexpr bool DPF = true;
  static constexpr int N = 12;
  static constexpr uint32_t n0 = BlsFp::n0;
  __host__ __device__ static constexpr uint32_t mod(int i) { return BlsFp::mod(i); }
  // 2^416 mod p, 2^832 mod p
  ZKB_DPF_TABLE(one, 12, 0xa8e9b9afu, 0x44f6480eu, 0x766c8fe4u, 0xa96f7d65u, 0x28b540feu, 0xe82efd42u, 0xade53b2eu, 0x6723e5f0u, 0xfdd4230au, 0x25ff6eb6u, 0xef23c24au, 0x14c8ee06u)
  ZKB_DPF_TABLE(r2, 12, 0xcb89af51u, 0x1a2a5bf4u, 0xfbba7ca3u, 0xec71f13au, 0x32646160u, 0x71046590u, 0x8311a84du, 0x480a4a18u, 0x7ad91f53u, 0x6698e590u, 0x5d745072u, 0x08746207u)
};

struct BnFrD {
  static constexpr bool DPF = true;
  static constexpr int N = 8;
  static constexpr uint32_t n0 = BnFr::n0;
  __host__ __device__ static constexpr uint32_t mod(int i) { return BnFr::mod(i); }
  // 2^260 mod r, 2^520 mod r
  ZKB_DPF_TABLE(one, 8, 0x3fffffacu, 0xb9db6b75u, 0x0f271055u, 0xcef7c838u, 0x818f016eu, 0x85a9201du, 0x1bb7724fu, 0x1f16424eu)
  ZKB_DPF_TABLE(r2, 8, 0xd16da6f5u, 0xce30b852u, 0x21620cddu, 0x43ffb6c6u, 0x2af1b953u, 0x5e103e7cu, 0xa122c3c1u, 0x0281528fu)
};
struct BlsFrD {
  static constexpr bool DPF = true;
  static constexpr int N = 8;
  static constexpr uint32_t n0 = BlsFr::n0;
  __host__ __device__ static constexpr uint32_t mod(int i) { return BlsFr::mod(i); }
  // 2^260 mod r, 2^520 mod r
  ZKB_DPF_TABLE(one, 8, 0xffffffddu, 0x00000022u, 0x00396c23u, 0x8d129397u, 0xaedf7745u, 0xff1776e6u, 0x4f77df20u, 0x26821fa1u)
  ZKB_DPF_TABLE(r2, 8, 0xf29c6cf0u, 0x99e99103u, 0x927663d9u, 0x31138b57u, 0xba1c0ed6u, 0x9f7715f1u, 0xc0273c82u, 0x09ff646cu)
};

#undef ZKB_DPF_TABLE

// The MSM bucket pipeline's fields: FP64 products in radix R' on the redundant range [0, 2p)
// (no conditional subtraction per product; values are made canonical where the per-window sums
// leave the pipeline, k_msm_xyzz_from_dpf).
struct BnFpL : BnFpD {
  static constexpr bool LAZY = true;
};
struct BlsFpL : BlsFpD {
  static constexpr bool LAZY = true;
};

// Fr with FP64-pipe products in the reference's radix (the same elements and results as BnFr /
// BlsFr): the element-wise Fr operations.
struct BnFrE : BnFr {
  static constexpr bool DPF = true;
  static constexpr bool EXACT = true;
};
struct BlsFrE : BlsFr {
  static constexpr bool DPF = true;
  static constexpr bool EXACT = true;
};
struct BnFpE : BnFp {
  static constexpr bool DPF = true;
  static constexpr bool EXACT = true;
};
struct BlsFpE : BlsFp {
  static constexpr bool DPF = true;
  static constexpr bool EXACT = true;
};

// The FP64 twin of a field type (used where a kernel multiplies radix-R data by radix-R'
// constants: mont'(x R, w R') = (x w) R, so data stay in the reference's radix).
template <class P> struct DpfOf;
template <> struct DpfOf<BnFp> { using type = BnFpD; };
template <> struct DpfOf<BlsFp> { using type = BlsFpD; };
template <> struct DpfOf<BnFr> { using type = BnFrD; };
template <> struct DpfOf<BlsFr> { using type = BlsFrD; };

template <class P>
__device__ __noinline__ Fe<P> fe_mul_dpf_call(const Fe<P> a, const Fe<P> b) {
  return fd_to_words<P>(fd_mul_inl<P>(fd_from_words<P>(a), fd_from_words<P>(b)));
}
template <class P>
__device__ __noinline__ Fe2<P> fe_mul2_dpf_call(const Fe<P> a, const Fe<P> b, const Fe<P> c, const Fe<P> d) {
  Fe2<P> r;
  r.a = fd_to_words<P>(fd_mul_inl<P>(fd_from_words<P>(a), fd_from_words<P>(b)));
  r.b = fd_to_words<P>(fd_mul_inl<P>(fd_from_words<P>(c), fd_from_words<P>(d)));
  return r;
}
template <class P>
__device__ __noinline__ Fe2<P> fe_sqr2_dpf_call(const Fe<P> a, const Fe<P> c) {
  Fe2<P> r;
  r.a = fd_to_words<P>(fd_sqr_inl<P>(fd_from_words<P>(a)));
  r.b = fd_to_words<P>(fd_sqr_inl<P>(fd_from_words<P>(c)));
  return r;
}
template <class P>
__device__ __noinline__ Fe<P> fe_sqr_dpf_call(const Fe<P> a) {
  return fd_to_words<P>(fd_sqr_inl<P>(fd_from_words<P>(a)));
}


// Curve types over the FP64 fields: the same points, products on the FP64 pipe (radix R').
struct BN254D {
  using Fp = BnFpD;
  using Fr = BnFr;
  static constexpr int FP_WORDS = 8;
  static constexpr int SCALAR_BITS = 254;
  static constexpr int ID = 0;
};
struct BLS12_381D {
  using Fp = BlsFpD;
  using Fr = BlsFr;
  static constexpr int FP_WORDS = 12;
  static constexpr int SCALAR_BITS = 255;
  static constexpr int ID = 1;
};
template <class C> struct DpfCurve;
template <> struct DpfCurve<BN254> { using type = BN254D; };
template <> struct DpfCurve<BLS12_381> { using type = BLS12_381D; };

// True when a pipeline field keeps its data in a radix other than the reference's, so bases
// enter and sums leave it through conversion products.
template <class F>
inline constexpr bool radix_conv_v = F::DPF && !exact_v<F>;

// The MSM bucket pipeline's fields with the reference's own radix: FP64 products with the exact
// last digit on the redundant range [0, 2p); bases and sums need no conversion.
struct BnFpLE : BnFp {
  static constexpr bool DPF = true;
  static constexpr bool EXACT = true;
  static constexpr bool LAZY = true;
};
struct BlsFpLE : BlsFp {
  static constexpr bool DPF = true;
  static constexpr bool EXACT = true;
  static constexpr bool LAZY = true;
};
struct BN254E {
  using Fp = BnFpLE;
  using Fr = BnFr;
  static constexpr int FP_WORDS = 8;
  static constexpr int SCALAR_BITS = 254;
  static constexpr int ID = 0;
};
struct BLS12_381E {
  using Fp = BlsFpLE;
  using Fr = BlsFr;
  static constexpr int FP_WORDS = 12;
  static constexpr int SCALAR_BITS = 255;
  static constexpr int ID = 1;
};

// Curve types of the MSM bucket pipeline in radix R': FP64 products on the redundant range
// [0, 2p) (bases converted in, window sums converted out).
struct BN254L {
  using Fp = BnFpL;
  using Fr = BnFr;
  static constexpr int FP_WORDS = 8;
  static constexpr int SCALAR_BITS = 254;
  static constexpr int ID = 0;
};
struct BLS12_381L {
  using Fp = BlsFpL;
  using Fr = BlsFr;
  static constexpr int FP_WORDS = 12;
  static constexpr int SCALAR_BITS = 255;
  static constexpr int ID = 1;
};
template <class C> struct MsmCurve;
template <> struct MsmCurve<BN254> { using type = BN254E; };
template <> struct MsmCurve<BLS12_381> { using type = BLS12_381E; };


// kin = R'^2 / R = 2^(2 * 52 L - 32 N) mod p and kout = R = 2^(32 N) mod p as field words
// (standard integers: they are operands of mont'(., .), not values in either radix)
template <class CD, int NL>
inline void dpf_consts(const host::Field<NL>& F, Fe<typename CD::Fp>& kin, Fe<typename CD::Fp>& kout) {
  using FD = typename CD::Fp;
  constexpr int L = D52<FD>::L;
  auto pow2 = [&](int e, Fe<FD>& out) {
    host::El<NL> x = host::zero<NL>();
    x.v[0] = 1;
    for (int i = 0; i < e; i++) x = host::add(F, x, x);
    for (int w = 0; w < FD::N; w++) out.v[w] = (uint32_t)(x.v[w >> 1] >> (32 * (w & 1)));
  };
  pow2(2 * 52 * L - 32 * FD::N, kin);
  pow2(32 * FD::N, kout);
}
template <class CD>
inline void dpf_consts_for(Fe<typename CD::Fp>& kin, Fe<typename CD::Fp>& kout) {
  static Fe<typename CD::Fp> s_kin, s_kout;
  static std::once_flag once;
  std::call_once(once, [] {
    if constexpr (CD::ID == 0) dpf_consts<CD, 4>(host::BN_FP, s_kin, s_kout);
    else dpf_consts<CD, 6>(host::BLS_FP, s_kin, s_kout);
  });
  kin = s_kin;
  kout = s_kout;
}

template <class CD>
inline Fe<typename CD::Fp> dpf_kin() {
  Fe<typename CD::Fp> a, b;
  dpf_consts_for<CD>(a, b);
  return a;
}
template <class CD>
inline Fe<typename CD::Fp> dpf_kout() {
  Fe<typename CD::Fp> a, b;
  dpf_consts_for<CD>(a, b);
  return b;
}

}  // namespace zkb
