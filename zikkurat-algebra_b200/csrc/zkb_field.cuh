// Prime-field arithmetic for sm_100a: Montgomery multiplication over 32-bit limbs on the
// integer multiply-add pipe (IMAD), with PTX carry chains.
//
// Values are stored exactly like the reference's little-endian 64-bit limbs
// (lib/cbits/curves/fields/mont/*_mont.c): a 64-bit limb k is 32-bit limbs 2k (low) and 2k+1
// (high), so the Montgomery radix R = 2^(32*N) equals the reference's 2^(64*N/2) and a
// Montgomery value needs no conversion between the host and the device.
//
// Every operation returns a fully reduced value in [0, p); the reduced result of a
// modular operation is unique, so results are bit-identical to the reference's
// (bn128_Fr_mont.c:86-103 add/sub, :189 mul = bigint256_mul + REDC :140-169).
#pragma once
#include <cstdint>

namespace zkb {

// ------------------------------------------------------------------ carry-chain primitives
// One PTX instruction each. A chain is a run of these with no other carry-flag user in
// between; `asm volatile` keeps their relative order, and the carry flag is PTX state that
// ptxas tracks as a dependency.
__device__ __forceinline__ uint32_t add_cc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t addc_cc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t addc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("addc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t sub_cc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t subc_cc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t subc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("subc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t mad_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r; asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ uint32_t madc_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r; asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ uint32_t mad_hi_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r; asm volatile("mad.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ uint32_t madc_hi_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r; asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }

// ------------------------------------------------------------------------ field parameters
// p, n0 = -p^-1 mod 2^32, R mod p, R^2 mod p. Moduli: lib/cbits/curves/fields/mont/
// bn128_Fp_mont.c:20, bn128_Fr_mont.c:20, bls12_381_Fp_mont.c:20, bls12_381_Fr_mont.c:20
// (n0 is the low word of the reference's 64-bit constant at :145/:151).
#define ZKB_TABLE(name, n, ...)                                                   \
  __host__ __device__ static constexpr uint32_t name(int i) {                    \
    constexpr uint32_t t[n] = {__VA_ARGS__};                                      \
    return t[i];                                                                  \
  }

struct BnFp {
  static constexpr bool DPF = false;   // products on the integer pipes
  static constexpr int N = 8;
  static constexpr uint32_t n0 = 0xe4866389u;
  ZKB_TABLE(mod, 8, 0xd87cfd47u, 0x3c208c16u, 0x6871ca8du, 0x97816a91u, 0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u)
  ZKB_TABLE(one, 8, 0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u, 0x7879462cu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u)
  ZKB_TABLE(r2, 8, 0x538afa89u, 0xf32cfc5bu, 0xd44501fbu, 0xb5e71911u, 0x0a417ff6u, 0x47ab1effu, 0xcab8351fu, 0x06d89f71u)
};
struct BnFr {
  static constexpr bool DPF = false;   // products on the integer pipes
  static constexpr int N = 8;
  static constexpr uint32_t n0 = 0xefffffffu;
  ZKB_TABLE(mod, 8, 0xf0000001u, 0x43e1f593u, 0x79b97091u, 0x2833e848u, 0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u)
  ZKB_TABLE(one, 8, 0x4ffffffbu, 0xac96341cu, 0x9f60cd29u, 0x36fc7695u, 0x7879462eu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u)
  ZKB_TABLE(r2, 8, 0xae216da7u, 0x1bb8e645u, 0xe35c59e3u, 0x53fe3ab1u, 0x53bb8085u, 0x8c49833du, 0x7f4e44a5u, 0x0216d0b1u)
};
struct BlsFp {
  static constexpr bool DPF = false;   // products on the integer pipes
  static constexpr int N = 12;
  static constexpr uint32_t n0 = 0xfffcfffdu;
  ZKB_TABLE(mod, 12, 0xffffaaabu, 0xb9feffffu, 0xb153ffffu, 0x1eabfffeu, 0xf6b0f624u, 0x6730d2a0u, 0xf38512bfu, 0x64774b84u, 0x434bacd7u, 0x4b1ba7b6u, 0x397fe69au, 0x1a0111eau)
  ZKB_TABLE(one, 12, 0x0002fffdu, 0x76090000u, 0xc40c0002u, 0xebf4000bu, 0x53c758bau, 0x5f489857u, 0x70525745u, 0x77ce5853u, 0xa256ec6du, 0x5c071a97u, 0xfa80e493u, 0x15f65ec3u)
  ZKB_TABLE(r2, 12, 0x1c341746u, 0xf4df1f34u, 0x09d104f1u, 0x0a76e6a6u, 0x4c95b6d5u, 0x8de5476cu, 0x939d83c0u, 0x67eb88a9u, 0xb519952du, 0x9a793e85u, 0x92cae3aau, 0x11988fe5u)
};
struct BlsFr {
  static constexpr bool DPF = false;   // products on the integer pipes
  static constexpr int N = 8;
  static constexpr uint32_t n0 = 0xffffffffu;
  ZKB_TABLE(mod, 8, 0x00000001u, 0xffffffffu, 0xfffe5bfeu, 0x53bda402u, 0x09a1d805u, 0x3339d808u, 0x299d7d48u, 0x73eda753u)
  ZKB_TABLE(one, 8, 0xfffffffeu, 0x00000001u, 0x00034802u, 0x5884b7fau, 0xecbc4ff5u, 0x998c4fefu, 0xacc5056fu, 0x1824b159u)
  ZKB_TABLE(r2, 8, 0xf3f29c6du, 0xc999e990u, 0x87925c23u, 0x2b6cedcbu, 0x7254398fu, 0x05d31496u, 0x9f59ff11u, 0x0748d9d9u)
};
#undef ZKB_TABLE

// --------------------------------------------------------------------------- element type
template <class P>
struct Fe {
  uint32_t v[P::N];
};

template <class P>
__device__ __forceinline__ Fe<P> fe_zero() {
  Fe<P> r;
#pragma unroll
  for (int i = 0; i < P::N; i++) r.v[i] = 0;
  return r;
}
template <class P>
__device__ __forceinline__ Fe<P> fe_one() {
  Fe<P> r;
#pragma unroll
  for (int i = 0; i < P::N; i++) r.v[i] = P::one(i);
  return r;
}
template <class P>
__device__ __forceinline__ bool fe_is_zero(const Fe<P>& a) {
  uint32_t x = a.v[0];
#pragma unroll
  for (int i = 1; i < P::N; i++) x |= a.v[i];
  return x == 0;
}
template <class P>
__device__ __forceinline__ bool fe_eq(const Fe<P>& a, const Fe<P>& b) {
  uint32_t x = a.v[0] ^ b.v[0];
#pragma unroll
  for (int i = 1; i < P::N; i++) x |= a.v[i] ^ b.v[i];
  return x == 0;
}

// ------------------------------------------------------------- redundant representation
// A field type with LAZY = true keeps its values in [0, 2p) instead of [0, p): products skip
// their final conditional subtraction (zkb_dpf.cuh), and additions, subtractions and negations
// reduce modulo 2p. 4p must fit the N words (true for all four fields here: p < 2^254 in 8 words,
// p < 2^381 in 12). Tests for zero accept both representatives 0 and p; fe_canon brings a value
// into [0, p) where it leaves the pipeline. Fields without the flag are canonical everywhere.
template <class P, class = void>
struct LazyOf { static constexpr bool value = false; };
template <class P>
struct LazyOf<P, decltype((void)P::LAZY)> { static constexpr bool value = P::LAZY; };
template <class P>
inline constexpr bool lazy_v = LazyOf<P>::value;

// word i of the modulus the additions reduce by: p, or 2p for a lazy field
template <class P>
__host__ __device__ constexpr uint32_t red_mod(int i) {
  if constexpr (lazy_v<P>) return (P::mod(i) << 1) | (i > 0 ? P::mod(i - 1) >> 31 : 0u);
  else return P::mod(i);
}

// t (N words) plus a top word `hi` (0 or 1), known to be < 2m: return t mod m, where m is the
// reduction modulus of P (p, or 2p for a lazy field); TO_P = true reduces by p instead.
template <class P, bool TO_P = false>
__device__ __forceinline__ Fe<P> reduce_once(const uint32_t* t, uint32_t hi) {
  constexpr int N = P::N;
  auto m = [](int j) { return TO_P ? P::mod(j) : red_mod<P>(j); };
  uint32_t d[N];
  d[0] = sub_cc(t[0], m(0));
#pragma unroll
  for (int j = 1; j < N; j++) d[j] = subc_cc(t[j], m(j));
  const uint32_t top = subc(hi, 0);     // 0xffffffff exactly when t < m
  Fe<P> r;
#pragma unroll
  for (int j = 0; j < N; j++) r.v[j] = (top == 0xffffffffu) ? t[j] : d[j];
  return r;
}

// canonical representative in [0, p) (identity for fields that are canonical throughout)
template <class P>
__device__ __forceinline__ Fe<P> fe_canon(const Fe<P>& a) {
  if constexpr (lazy_v<P>) return reduce_once<P, true>(a.v, 0u);
  else return a;
}

// a == 0 mod p (lazy fields: a is 0 or p)
template <class P>
__device__ __forceinline__ bool fe_is_zero_mod(const Fe<P>& a) {
  if constexpr (lazy_v<P>) {
    uint32_t x = a.v[0], y = a.v[0] ^ P::mod(0);
#pragma unroll
    for (int i = 1; i < P::N; i++) { x |= a.v[i]; y |= a.v[i] ^ P::mod(i); }
    return x == 0 || y == 0;
  } else {
    return fe_is_zero(a);
  }
}

template <class P>
__device__ __forceinline__ Fe<P> fe_add(const Fe<P>& a, const Fe<P>& b) {
  constexpr int N = P::N;
  uint32_t t[N];
  t[0] = add_cc(a.v[0], b.v[0]);
#pragma unroll
  for (int j = 1; j < N; j++) t[j] = addc_cc(a.v[j], b.v[j]);
  const uint32_t hi = addc(0, 0);
  return reduce_once<P>(t, hi);
}

template <class P>
__device__ __forceinline__ Fe<P> fe_sub(const Fe<P>& a, const Fe<P>& b) {
  constexpr int N = P::N;
  uint32_t t[N];
  t[0] = sub_cc(a.v[0], b.v[0]);
#pragma unroll
  for (int j = 1; j < N; j++) t[j] = subc_cc(a.v[j], b.v[j]);
  const uint32_t bw = subc(0, 0);       // 0xffffffff on borrow
  Fe<P> r;
  r.v[0] = add_cc(t[0], red_mod<P>(0) & bw);
#pragma unroll
  for (int j = 1; j < N - 1; j++) r.v[j] = addc_cc(t[j], red_mod<P>(j) & bw);
  r.v[N - 1] = addc(t[N - 1], red_mod<P>(N - 1) & bw);
  return r;
}

template <class P>
__device__ __forceinline__ Fe<P> fe_neg(const Fe<P>& a) {
  constexpr int N = P::N;
  const uint32_t nz = fe_is_zero(a) ? 0u : 0xffffffffu;
  Fe<P> r;
  r.v[0] = sub_cc(red_mod<P>(0) & nz, a.v[0]);
#pragma unroll
  for (int j = 1; j < N - 1; j++) r.v[j] = subc_cc(red_mod<P>(j) & nz, a.v[j]);
  r.v[N - 1] = subc(red_mod<P>(N - 1) & nz, a.v[N - 1]);
  return r;
}

template <class P>
__device__ __forceinline__ Fe<P> fe_dbl(const Fe<P>& a) { return fe_add(a, a); }

// Montgomery product a*b*2^(-32N) mod p by coarsely integrated operand scanning:
// per word b_i, accumulate a*b_i (low halves, then high halves), pick m = t0*n0,
// accumulate m*p the same way, and drop the (now zero) low word.
// Cost: 4N^2 + N IMAD (264 for N=8, 588 for N=12) plus 6N carry-propagation adds.
template <class P>
__device__ __forceinline__ Fe<P> fe_mul_inl(const Fe<P>& a, const Fe<P>& b) {
  constexpr int N = P::N;
  uint32_t t[N + 2];
#pragma unroll
  for (int j = 0; j < N + 2; j++) t[j] = 0;
#pragma unroll
  for (int i = 0; i < N; i++) {
    const uint32_t bi = b.v[i];
    t[0] = mad_lo_cc(a.v[0], bi, t[0]);
#pragma unroll
    for (int j = 1; j < N; j++) t[j] = madc_lo_cc(a.v[j], bi, t[j]);
    t[N] = addc_cc(t[N], 0);
    t[N + 1] = addc(t[N + 1], 0);
    t[1] = mad_hi_cc(a.v[0], bi, t[1]);
#pragma unroll
    for (int j = 1; j < N; j++) t[j + 1] = madc_hi_cc(a.v[j], bi, t[j + 1]);
    t[N + 1] = addc(t[N + 1], 0);

    const uint32_t m = t[0] * P::n0;
    t[0] = mad_lo_cc(m, P::mod(0), t[0]);
#pragma unroll
    for (int j = 1; j < N; j++) t[j] = madc_lo_cc(m, P::mod(j), t[j]);
    t[N] = addc_cc(t[N], 0);
    t[N + 1] = addc(t[N + 1], 0);
    t[1] = mad_hi_cc(m, P::mod(0), t[1]);
#pragma unroll
    for (int j = 1; j < N; j++) t[j + 1] = madc_hi_cc(m, P::mod(j), t[j + 1]);
    t[N + 1] = addc(t[N + 1], 0);
#pragma unroll
    for (int j = 0; j <= N; j++) t[j] = t[j + 1];
    t[N + 1] = 0;
  }
  return reduce_once<P>(t, t[N]);
}

// One out-of-line copy of the product per field and kernel. A point addition chains 10-14
// products; expanded in place they make a ~60 KB loop body that misses the instruction cache
// (measured on B200: the BN254 bucket-accumulation kernel ran 17% slower inlined, BLS12-381 75%).
// Defining ZKB_MUL_INLINE expands every product in place instead.
template <class P>
__device__ __noinline__ Fe<P> fe_mul_call(const Fe<P> a, const Fe<P> b) { return fe_mul_inl(a, b); }

// Product on the FP64 pipe for fields flagged DPF (zkb_dpf.cuh: same words, Montgomery radix
// 2^(52 L) instead of 2^(32 N)); defined there.
template <class P>
__device__ __noinline__ Fe<P> fe_mul_dpf_call(const Fe<P> a, const Fe<P> b);

template <class P>
__device__ __forceinline__ Fe<P> fe_mul(const Fe<P>& a, const Fe<P>& b) {
  if constexpr (P::DPF) {
    return fe_mul_dpf_call<P>(a, b);
  } else {
#ifdef ZKB_MUL_INLINE
    return fe_mul_inl(a, b);
#else
    return fe_mul_call<P>(a, b);
#endif
  }
}

template <class P>
__device__ __noinline__ Fe<P> fe_sqr_dpf_call(const Fe<P> a);   // zkb_dpf.cuh

template <class P>
__device__ __forceinline__ Fe<P> fe_sqr(const Fe<P>& a) {
  if constexpr (P::DPF) return fe_sqr_dpf_call<P>(a);
  else return fe_mul(a, a);
}

// Two independent products in one call. On the FP64 pipe (254/255-bit fields) the two are
// interleaved, which doubles the instruction-level parallelism of the word-by-word reduction
// chain; for BLS12-381 Fp the pair does not fit the register budget and runs as two calls.
template <class P> struct Fe2 { Fe<P> a, b; };
template <class P>
__device__ __noinline__ Fe2<P> fe_mul2_dpf_call(const Fe<P> a, const Fe<P> b, const Fe<P> c, const Fe<P> d);
template <class P>
__device__ __noinline__ Fe2<P> fe_sqr2_dpf_call(const Fe<P> a, const Fe<P> c);

// r = a b, s = c d (r, s may alias any operand)
template <class P>
__device__ __forceinline__ void fe_mul2(Fe<P>& r, const Fe<P>& a, const Fe<P>& b, Fe<P>& s,
                                        const Fe<P>& c, const Fe<P>& d) {
  if constexpr (P::DPF && P::N == 8) {   // 8-limb (BLS12-381 Fp) pairs spill: measured slower
    const Fe2<P> t = fe_mul2_dpf_call<P>(a, b, c, d);
    r = t.a;
    s = t.b;
  } else {
    const Fe<P> t = fe_mul(a, b);
    s = fe_mul(c, d);
    r = t;
  }
}
// r = a^2, s = c^2 (r, s may alias any operand)
template <class P>
__device__ __forceinline__ void fe_sqr2(Fe<P>& r, const Fe<P>& a, Fe<P>& s, const Fe<P>& c) {
  if constexpr (P::DPF && P::N == 8) {
    const Fe2<P> t = fe_sqr2_dpf_call<P>(a, c);
    r = t.a;
    s = t.b;
  } else {
    const Fe<P> t = fe_sqr(a);
    s = fe_sqr(c);
    r = t;
  }
}

// a^e for an exponent given as 32-bit words (most significant first scan)
template <class P, int EW>
__device__ __forceinline__ Fe<P> fe_pow(const Fe<P>& a, const uint32_t (&e)[EW]) {
  Fe<P> acc = fe_one<P>();
  bool started = false;
  for (int w = EW - 1; w >= 0; w--) {
    for (int bit = 31; bit >= 0; bit--) {
      if (started) acc = fe_sqr(acc);
      if ((e[w] >> bit) & 1u) { acc = started ? fe_mul(acc, a) : a; started = true; }
    }
  }
  return acc;
}

// a^-1 = a^(p-2) (Fermat); 0 maps to 0, as the reference's inversion does
// (bn128_Fr_std.c:298-301)
template <class P>
__device__ __forceinline__ Fe<P> fe_inv_fermat(const Fe<P>& a) {
  uint32_t e[P::N];   // p - 2 (BLS12-381 r has low word 1, so the borrow can propagate)
  uint32_t borrow = 2;
#pragma unroll
  for (int i = 0; i < P::N; i++) {
    const uint32_t w = P::mod(i);
    e[i] = w - borrow;
    borrow = w < borrow ? 1u : 0u;
  }
  return fe_pow<P, P::N>(a, e);
}

// a^-1 for a Montgomery element a = x R (result x^-1 R; 0 maps to 0), by the binary extended
// Euclidean algorithm on the integer a and p (each step halves u or v, or subtracts the smaller
// from the larger, so at most 2 (bits(a) + bits(p)) steps; capped at 32 N * 8). The integer
// inverse a^-1 = x^-1 R^-1 is brought back to Montgomery form by one product with R^3 =
// mont(R^2, R^2). Its dependency chain is a few thousand word operations, against ~380
// sequential products for a^(p-2): the inversion one thread runs for a whole block.
template <class P>
__device__ Fe<P> fe_inv_binary(const Fe<P>& a) {
  constexpr int N = P::N;
  if (fe_is_zero(a)) return fe_zero<P>();
  uint32_t u[N], v[N], x1[N], x2[N];
  for (int k = 0; k < N; k++) { u[k] = a.v[k]; v[k] = P::mod(k); x1[k] = 0; x2[k] = 0; }
  x1[0] = 1;
  auto is_one = [](const uint32_t* w) {
    uint32_t o = w[0] ^ 1u;
    for (int k = 1; k < N; k++) o |= w[k];
    return o == 0;
  };
  auto halve = [](uint32_t* w) {
    for (int k = 0; k < N - 1; k++) w[k] = (w[k] >> 1) | (w[k + 1] << 31);
    w[N - 1] >>= 1;
  };
  auto halve_mod = [&](uint32_t* x) {   // x / 2 mod p (x + p < 2^(32 N): p has a spare top bit)
    if (x[0] & 1u) {
      uint64_t c = 0;
      for (int k = 0; k < N; k++) {
        c += (uint64_t)x[k] + P::mod(k);
        x[k] = (uint32_t)c;
        c >>= 32;
      }
    }
    halve(x);
  };
  auto geq = [](const uint32_t* x, const uint32_t* y) {
    for (int k = N - 1; k >= 0; k--)
      if (x[k] != y[k]) return x[k] > y[k];
    return true;
  };
  auto sub = [](uint32_t* x, const uint32_t* y) {   // x -= y; returns the borrow
    uint32_t b = 0;
    for (int k = 0; k < N; k++) {
      const uint64_t d = (uint64_t)x[k] - y[k] - b;
      x[k] = (uint32_t)d;
      b = (uint32_t)(d >> 63);
    }
    return b;
  };
  auto sub_mod = [&](uint32_t* x, const uint32_t* y) {   // x = x - y mod p
    if (sub(x, y)) {
      uint64_t c = 0;
      for (int k = 0; k < N; k++) {
        c += (uint64_t)x[k] + P::mod(k);
        x[k] = (uint32_t)c;
        c >>= 32;
      }
    }
  };
  for (int it = 0; it < 32 * N * 8; it++) {
    if (is_one(u) || is_one(v)) break;
    if (!(u[0] & 1u)) { halve(u); halve_mod(x1); }
    else if (!(v[0] & 1u)) { halve(v); halve_mod(x2); }
    else if (geq(u, v)) { sub(u, v); sub_mod(x1, x2); }
    else { sub(v, u); sub_mod(x2, x1); }
  }
  Fe<P> r;
  const bool one_u = is_one(u);
  for (int k = 0; k < N; k++) r.v[k] = one_u ? x1[k] : x2[k];
  Fe<P> r2;
  for (int k = 0; k < N; k++) r2.v[k] = P::r2(k);
  return fe_mul(r, fe_mul(r2, r2));
}

// x -> x * R^-1 (Montgomery -> standard), the reference's to_std (bn128_Fr_mont.c:330)
template <class P>
__device__ __forceinline__ Fe<P> fe_from_mont(const Fe<P>& a) {
  Fe<P> one_std = fe_zero<P>();
  one_std.v[0] = 1;
  return fe_mul(a, one_std);
}
// x -> x * R (standard -> Montgomery)
template <class P>
__device__ __forceinline__ Fe<P> fe_to_mont(const Fe<P>& a) {
  Fe<P> r2;
#pragma unroll
  for (int i = 0; i < P::N; i++) r2.v[i] = P::r2(i);
  return fe_mul(a, r2);
}

// ------------------------------------------------------------------------ memory helpers
template <class P>
__device__ __forceinline__ Fe<P> fe_load(const uint32_t* __restrict__ src) {
  static_assert(P::N % 4 == 0, "vector loads need N % 4 == 0");
  Fe<P> r;
  const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
  for (int q = 0; q < P::N / 4; q++) {
    const uint4 x = s[q];
    r.v[4 * q + 0] = x.x; r.v[4 * q + 1] = x.y; r.v[4 * q + 2] = x.z; r.v[4 * q + 3] = x.w;
  }
  return r;
}
template <class P>
__device__ __forceinline__ Fe<P> fe_load_cg(const uint32_t* __restrict__ src) {   // L2 only (data written by
  Fe<P> r;                                                                         // other CTAs of a running kernel)
  const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
  for (int q = 0; q < P::N / 4; q++) {
    const uint4 x = __ldcg(s + q);
    r.v[4 * q + 0] = x.x; r.v[4 * q + 1] = x.y; r.v[4 * q + 2] = x.z; r.v[4 * q + 3] = x.w;
  }
  return r;
}
template <class P>
__device__ __forceinline__ Fe<P> fe_load_nc(const uint32_t* __restrict__ src) {
  Fe<P> r;
  const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
  for (int q = 0; q < P::N / 4; q++) {
    const uint4 x = __ldg(s + q);
    r.v[4 * q + 0] = x.x; r.v[4 * q + 1] = x.y; r.v[4 * q + 2] = x.z; r.v[4 * q + 3] = x.w;
  }
  return r;
}
template <class P>
__device__ __forceinline__ void fe_store(uint32_t* __restrict__ dst, const Fe<P>& a) {
  uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
  for (int q = 0; q < P::N / 4; q++)
    d[q] = make_uint4(a.v[4 * q + 0], a.v[4 * q + 1], a.v[4 * q + 2], a.v[4 * q + 3]);
}

}  // namespace zkb
