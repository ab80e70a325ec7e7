// Host-side field and G1 arithmetic for the serial tail of an MSM.
//
// After the GPU has reduced all buckets to a few dozen points per window, what remains is a
// chain of ~250 dependent doublings (Horner over windows) and one inversion. A single CPU core
// runs one 256-bit Montgomery product in ~30 ns versus ~1 us for one GPU thread, so this
// O(windows * c) tail runs here. It also produces the reference's exact output encodings:
//   projective (X, Y, Z) with infinity (0, 1, 0)      lib/cbits/curves/g1/proj/bn128_G1_proj.c:183-187
//   Jacobian   (X, Y, Z) with infinity (1, 1, 0)      lib/cbits/curves/g1/jac/bn128_G1_jac.c:182-187
//   affine     (x, y)    with infinity all 0xff bytes  bn128_G1_proj.c:132-137
// Finite outputs are normalised (Z = 1), so every output is canonical and deterministic.
#pragma once
#include <cstdint>
#include <cstring>

namespace zkb {
namespace host {

typedef unsigned __int128 u128;

template <int NL>
struct Field {
  uint64_t p[NL];
  uint64_t n0;     // -p^-1 mod 2^64
  uint64_t one[NL];
  uint64_t r2[NL];
};

template <int NL>
struct El {
  uint64_t v[NL];
};

template <int NL>
inline bool is_zero(const El<NL>& a) {
  uint64_t x = 0;
  for (int i = 0; i < NL; i++) x |= a.v[i];
  return x == 0;
}
template <int NL>
inline bool ge_p(const Field<NL>& F, const uint64_t* a) {
  for (int i = NL - 1; i >= 0; i--) {
    if (a[i] > F.p[i]) return true;
    if (a[i] < F.p[i]) return false;
  }
  return true;
}
template <int NL>
inline uint64_t sub_raw(const uint64_t* a, const uint64_t* b, uint64_t* o) {
  uint64_t br = 0;
  for (int i = 0; i < NL; i++) {
    u128 d = (u128)a[i] - b[i] - br;
    o[i] = (uint64_t)d;
    br = (uint64_t)(d >> 64) & 1;
  }
  return br;
}
template <int NL>
inline uint64_t add_raw(const uint64_t* a, const uint64_t* b, uint64_t* o) {
  uint64_t c = 0;
  for (int i = 0; i < NL; i++) {
    u128 s = (u128)a[i] + b[i] + c;
    o[i] = (uint64_t)s;
    c = (uint64_t)(s >> 64);
  }
  return c;
}
template <int NL>
inline El<NL> add(const Field<NL>& F, const El<NL>& a, const El<NL>& b) {
  El<NL> r;
  uint64_t c = add_raw<NL>(a.v, b.v, r.v);
  if (c || ge_p<NL>(F, r.v)) sub_raw<NL>(r.v, F.p, r.v);
  return r;
}
template <int NL>
inline El<NL> sub(const Field<NL>& F, const El<NL>& a, const El<NL>& b) {
  El<NL> r;
  if (sub_raw<NL>(a.v, b.v, r.v)) add_raw<NL>(r.v, F.p, r.v);
  return r;
}
template <int NL>
inline El<NL> mul(const Field<NL>& F, const El<NL>& a, const El<NL>& b) {
  uint64_t t[NL + 2] = {0};
  for (int i = 0; i < NL; i++) {
    u128 c = 0;
    for (int j = 0; j < NL; j++) {
      c += (u128)a.v[j] * b.v[i] + t[j];
      t[j] = (uint64_t)c;
      c >>= 64;
    }
    c += t[NL];
    t[NL] = (uint64_t)c;
    t[NL + 1] = (uint64_t)(c >> 64);
    const uint64_t m = t[0] * F.n0;
    c = (u128)m * F.p[0] + t[0];
    c >>= 64;
    for (int j = 1; j < NL; j++) {
      c += (u128)m * F.p[j] + t[j];
      t[j - 1] = (uint64_t)c;
      c >>= 64;
    }
    c += t[NL];
    t[NL - 1] = (uint64_t)c;
    t[NL] = t[NL + 1] + (uint64_t)(c >> 64);
  }
  El<NL> r;
  if (t[NL] || ge_p<NL>(F, t)) sub_raw<NL>(t, F.p, t);
  std::memcpy(r.v, t, sizeof(r.v));
  return r;
}
template <int NL>
inline El<NL> one(const Field<NL>& F) {
  El<NL> r;
  std::memcpy(r.v, F.one, sizeof(r.v));
  return r;
}
template <int NL>
inline El<NL> zero() {
  El<NL> r;
  std::memset(r.v, 0, sizeof(r.v));
  return r;
}
// a^(p-2) (0 -> 0, matching the reference's inverse of zero, bn128_Fr_std.c:298-301)
template <int NL>
inline El<NL> inv(const Field<NL>& F, const El<NL>& a) {
  if (is_zero(a)) return a;
  uint64_t e[NL];
  uint64_t two[NL] = {2};
  sub_raw<NL>(F.p, two, e);
  El<NL> acc = one(F), base = a;
  for (int i = 0; i < NL; i++)
    for (int b = 0; b < 64; b++) {
      if ((e[i] >> b) & 1) acc = mul(F, acc, base);
      base = mul(F, base, base);
    }
  return acc;
}
template <int NL>
inline El<NL> from_std(const Field<NL>& F, const El<NL>& a) {
  El<NL> r2;
  std::memcpy(r2.v, F.r2, sizeof(r2.v));
  return mul(F, a, r2);
}
template <int NL>
inline El<NL> pow_u64(const Field<NL>& F, const El<NL>& a, uint64_t e) {
  El<NL> acc = one(F), base = a;
  while (e) {
    if (e & 1) acc = mul(F, acc, base);
    base = mul(F, base, base);
    e >>= 1;
  }
  return acc;
}

// ---------------------------------------------------------------- XYZZ points (a = 0)
template <int NL>
struct Xyzz {
  El<NL> X, Y, ZZ, ZZZ;
};

template <int NL>
inline Xyzz<NL> xyzz_inf() {
  Xyzz<NL> r;
  r.X = zero<NL>(); r.Y = zero<NL>(); r.ZZ = zero<NL>(); r.ZZZ = zero<NL>();
  return r;
}

template <int NL>
inline Xyzz<NL> xyzz_dbl(const Field<NL>& F, const Xyzz<NL>& p) {
  if (is_zero(p.ZZ)) return p;
  El<NL> U = add(F, p.Y, p.Y);
  El<NL> V = mul(F, U, U);
  El<NL> W = mul(F, U, V);
  El<NL> S = mul(F, p.X, V);
  El<NL> xx = mul(F, p.X, p.X);
  El<NL> M = add(F, add(F, xx, xx), xx);
  Xyzz<NL> r;
  r.X = sub(F, mul(F, M, M), add(F, S, S));
  r.Y = sub(F, mul(F, M, sub(F, S, r.X)), mul(F, W, p.Y));
  r.ZZ = mul(F, V, p.ZZ);
  r.ZZZ = mul(F, W, p.ZZZ);
  return r;
}

template <int NL>
inline Xyzz<NL> xyzz_add(const Field<NL>& F, const Xyzz<NL>& a, const Xyzz<NL>& q) {
  if (is_zero(q.ZZ)) return a;
  if (is_zero(a.ZZ)) return q;
  El<NL> U1 = mul(F, a.X, q.ZZ), U2 = mul(F, q.X, a.ZZ);
  El<NL> S1 = mul(F, a.Y, q.ZZZ), S2 = mul(F, q.Y, a.ZZZ);
  El<NL> P = sub(F, U2, U1), R = sub(F, S2, S1);
  if (is_zero(P)) return is_zero(R) ? xyzz_dbl(F, a) : xyzz_inf<NL>();
  El<NL> PP = mul(F, P, P), PPP = mul(F, P, PP), Q = mul(F, U1, PP);
  Xyzz<NL> r;
  r.X = sub(F, sub(F, mul(F, R, R), PPP), add(F, Q, Q));
  r.Y = sub(F, mul(F, R, sub(F, Q, r.X)), mul(F, S1, PPP));
  r.ZZ = mul(F, mul(F, a.ZZ, q.ZZ), PP);
  r.ZZZ = mul(F, mul(F, a.ZZZ, q.ZZZ), PPP);
  return r;
}

// Output kinds of the drop-in entry points
enum OutKind { OUT_PROJ = 0, OUT_JAC = 1, OUT_AFFINE = 2 };

// Write the canonical encoding of p (Montgomery limbs) into out.
template <int NL>
inline void xyzz_write(const Field<NL>& F, const Xyzz<NL>& p, int kind, uint64_t* out) {
  if (is_zero(p.ZZ)) {
    if (kind == OUT_AFFINE) { std::memset(out, 0xff, 16 * NL); return; }
    El<NL> o = one(F), z = zero<NL>();
    std::memcpy(out, (kind == OUT_JAC ? o : z).v, 8 * NL);
    std::memcpy(out + NL, o.v, 8 * NL);
    std::memcpy(out + 2 * NL, z.v, 8 * NL);
    return;
  }
  // x = X / ZZ, y = Y / ZZZ with one inversion of ZZ * ZZZ
  El<NL> d = inv(F, mul(F, p.ZZ, p.ZZZ));
  El<NL> izz = mul(F, d, p.ZZZ);   // 1/ZZ
  El<NL> izzz = mul(F, d, p.ZZ);   // 1/ZZZ
  El<NL> x = mul(F, p.X, izz), y = mul(F, p.Y, izzz);
  std::memcpy(out, x.v, 8 * NL);
  std::memcpy(out + NL, y.v, 8 * NL);
  if (kind != OUT_AFFINE) std::memcpy(out + 2 * NL, one(F).v, 8 * NL);
}

// Field tables (64-bit limbs). Moduli: lib/cbits/curves/fields/mont/bn128_Fp_mont.c:20,
// bn128_Fr_mont.c:20, bls12_381_Fp_mont.c:20, bls12_381_Fr_mont.c:20.
static const Field<4> BN_FP = {{0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0x87d20782e4866389ULL, {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL}, {0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL}};
static const Field<4> BN_FR = {{0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0xc2e1f593efffffffULL, {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL}, {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL}};
static const Field<6> BLS_FP = {{0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL, 0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL}, 0x89f3fffcfffcfffdULL, {0x760900000002fffdULL, 0xebf4000bc40c0002ULL, 0x5f48985753c758baULL, 0x77ce585370525745ULL, 0x5c071a97a256ec6dULL, 0x15f65ec3fa80e493ULL}, {0xf4df1f341c341746ULL, 0x0a76e6a609d104f1ULL, 0x8de5476c4c95b6d5ULL, 0x67eb88a9939d83c0ULL, 0x9a793e85b519952dULL, 0x11988fe592cae3aaULL}};
static const Field<4> BLS_FR = {{0xffffffff00000001ULL, 0x53bda402fffe5bfeULL, 0x3339d80809a1d805ULL, 0x73eda753299d7d48ULL}, 0xfffffffeffffffffULL, {0x00000001fffffffeULL, 0x5884b7fa00034802ULL, 0x998c4fefecbc4ff5ULL, 0x1824b159acc5056fULL}, {0xc999e990f3f29c6dULL, 0x2b6cedcb87925c23ULL, 0x05d314967254398fULL, 0x0748d9d99f59ff11ULL}};

}  // namespace host
}  // namespace zkb
