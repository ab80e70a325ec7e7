/*
 * TEST ORACLE -- NOT PART OF THE PRODUCT.
 *
 * A plain-C, single-threaded restatement of the algorithms that faulhornlabs/zikkurat-algebra
 * runs on the two hot paths this repository accelerates:
 *   - Pippenger MSM on BN254 / BLS12-381 G1 (projective, unsigned windows);
 *   - radix-2 NTT (forward DIT, inverse DIF with per-stage halving) over Fr.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only
 * to check results. The product library (libzkb200.so) never links or calls it.
 *
 * Every routine is written from the reference's behaviour, not copied; each cites the
 * reference file:line it restates (paths relative to the reference project root).
 * Parity of this restatement is pinned two ways: against golden vectors generated by the
 * reference C itself (tests/golden/), and against the reference C compiled here
 * (oracle/_ref/libzkref.so) when that library is available.
 *
 * Representation (same as the reference): little-endian 64-bit limbs; Montgomery form
 * with R = 2^(64*nlimbs); affine points (x, y) with infinity encoded as (0, 0) on input
 * and as all-0xff bytes on affine output; projective (X, Y, Z) with infinity (0, 1, 0).
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <math.h>

typedef uint64_t u64;
typedef unsigned __int128 u128;

#define MAXL 6

typedef struct {
  int nl;        /* number of 64-bit limbs */
  u64 p[MAXL];   /* modulus */
  u64 n0;        /* -p^-1 mod 2^64 */
  u64 one[MAXL]; /* R mod p (Montgomery one) */
  u64 r2[MAXL];  /* R^2 mod p */
} fld_t;

/* moduli: lib/cbits/curves/fields/mont/bn128_Fp_mont.c:20 (n0 :145),
 *         lib/cbits/curves/fields/mont/bn128_Fr_mont.c:20 (n0 :145, R :130, R^2 :131),
 *         lib/cbits/curves/fields/mont/bls12_381_Fp_mont.c:20 (n0 :151),
 *         lib/cbits/curves/fields/mont/bls12_381_Fr_mont.c:20 (n0 :145) */
static const fld_t BN_FP = { 4, {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0x87d20782e4866389ULL, {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL}, {0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL} };
static const fld_t BN_FR = { 4, {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0xc2e1f593efffffffULL, {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL}, {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL} };
static const fld_t BLS_FP = { 6, {0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL, 0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL}, 0x89f3fffcfffcfffdULL, {0x760900000002fffdULL, 0xebf4000bc40c0002ULL, 0x5f48985753c758baULL, 0x77ce585370525745ULL, 0x5c071a97a256ec6dULL, 0x15f65ec3fa80e493ULL}, {0xf4df1f341c341746ULL, 0x0a76e6a609d104f1ULL, 0x8de5476c4c95b6d5ULL, 0x67eb88a9939d83c0ULL, 0x9a793e85b519952dULL, 0x11988fe592cae3aaULL} };
static const fld_t BLS_FR = { 4, {0xffffffff00000001ULL, 0x53bda402fffe5bfeULL, 0x3339d80809a1d805ULL, 0x73eda753299d7d48ULL}, 0xfffffffeffffffffULL, {0x00000001fffffffeULL, 0x5884b7fa00034802ULL, 0x998c4fefecbc4ff5ULL, 0x1824b159acc5056fULL}, {0xc999e990f3f29c6dULL, 0x2b6cedcb87925c23ULL, 0x05d314967254398fULL, 0x0748d9d99f59ff11ULL} };

typedef struct {
  const fld_t *fp, *fr;
  int b3;               /* 3*b as a small integer: BN b=3 -> 9, BLS b=4 -> 12 */
  u64 gen_std[2][MAXL]; /* G1 generator, standard (non-Montgomery) coordinates */
} curve_t;

/* generators: lib/cbits/curves/g1/affine/bn128_G1_affine.c:33, bls12_381_G1_affine.c:33
 * (stored there in Montgomery form; the standard coordinates are (1,2) for BN254) */
static const curve_t CURVES[2] = {
  { &BN_FP, &BN_FR, 9, { {1,0,0,0,0,0}, {2,0,0,0,0,0} } },
  { &BLS_FP, &BLS_FR, 12, {
      {0xfb3af00adb22c6bbULL, 0x6c55e83ff97a1aefULL, 0xa14e3a3f171bac58ULL, 0xc3688c4f9774b905ULL, 0x2695638c4fa9ac0fULL, 0x17f1d3a73197d794ULL},
      {0x0caa232946c5e7e1ULL, 0xd03cc744a2888ae4ULL, 0x00db18cb2c04b3edULL, 0xfcf5e095d5d00af6ULL, 0xa09e30ed741d8ae4ULL, 0x08b3f481e3aaa0f1ULL} } },
};

/* ---------------------------------------------------------------- field arithmetic ---- */

static int f_is_zero(const fld_t *F, const u64 *a) {
  for (int i = 0; i < F->nl; i++) if (a[i]) return 0;
  return 1;
}
static int f_eq(const fld_t *F, const u64 *a, const u64 *b) {
  for (int i = 0; i < F->nl; i++) if (a[i] != b[i]) return 0;
  return 1;
}
static void f_copy(const fld_t *F, const u64 *a, u64 *o) { memmove(o, a, 8 * F->nl); }
static void f_zero(const fld_t *F, u64 *o) { memset(o, 0, 8 * F->nl); }
static void f_one(const fld_t *F, u64 *o) { f_copy(F, F->one, o); }

/* returns borrow of o = a - b over nl limbs */
static u64 raw_sub(int nl, const u64 *a, const u64 *b, u64 *o) {
  u64 br = 0;
  for (int i = 0; i < nl; i++) {
    u128 d = (u128)a[i] - b[i] - br;
    o[i] = (u64)d;
    br = (u64)(d >> 64) & 1;
  }
  return br;
}
static u64 raw_add(int nl, const u64 *a, const u64 *b, u64 *o) {
  u64 c = 0;
  for (int i = 0; i < nl; i++) {
    u128 s = (u128)a[i] + b[i] + c;
    o[i] = (u64)s;
    c = (u64)(s >> 64);
  }
  return c;
}
/* is a >= p ? */
static int ge_p(const fld_t *F, const u64 *a) {
  for (int i = F->nl - 1; i >= 0; i--) {
    if (a[i] > F->p[i]) return 1;
    if (a[i] < F->p[i]) return 0;
  }
  return 1;
}

/* add: bigint add then one conditional subtraction (bn128_Fr_mont.c:86-90, :72-81) */
static void f_add(const fld_t *F, const u64 *a, const u64 *b, u64 *o) {
  u64 t[MAXL];
  raw_add(F->nl, a, b, t);
  if (ge_p(F, t)) raw_sub(F->nl, t, F->p, t);
  f_copy(F, t, o);
}
/* sub: bigint sub, add p back on borrow (bn128_Fr_mont.c:99-103) */
static void f_sub(const fld_t *F, const u64 *a, const u64 *b, u64 *o) {
  u64 t[MAXL];
  if (raw_sub(F->nl, a, b, t)) raw_add(F->nl, t, F->p, t);
  f_copy(F, t, o);
}
/* neg: 0 -> 0, else p - a (bn128_Fr_mont.c:41-55) */
static void f_neg(const fld_t *F, const u64 *a, u64 *o) {
  if (f_is_zero(F, a)) { f_zero(F, o); return; }
  raw_sub(F->nl, F->p, a, o);
}
/* Montgomery product a*b*R^-1 mod p, fully reduced (bn128_Fr_mont.c:189 = bigint mul
 * bigint256.c:267 followed by REDC bn128_Fr_mont.c:140-169). Restated as word-serial CIOS;
 * the reduced result is unique, so it equals the reference's for inputs below p. */
static void f_mul(const fld_t *F, const u64 *a, const u64 *b, u64 *o) {
  const int n = F->nl;
  u64 t[MAXL + 2] = {0};
  for (int i = 0; i < n; i++) {
    u128 c = 0;
    for (int j = 0; j < n; j++) {
      c += (u128)a[j] * b[i] + t[j];
      t[j] = (u64)c;
      c >>= 64;
    }
    c += t[n];
    t[n] = (u64)c;
    t[n + 1] = (u64)(c >> 64);
    u64 m = t[0] * F->n0;
    c = (u128)m * F->p[0] + t[0];
    c >>= 64;
    for (int j = 1; j < n; j++) {
      c += (u128)m * F->p[j] + t[j];
      t[j - 1] = (u64)c;
      c >>= 64;
    }
    c += t[n];
    t[n - 1] = (u64)c;
    t[n] = t[n + 1] + (u64)(c >> 64);
  }
  if (t[n] || ge_p(F, t)) raw_sub(n, t, F->p, t);
  f_copy(F, t, o);
}
static void f_sqr(const fld_t *F, const u64 *a, u64 *o) { f_mul(F, a, a, o); }

/* x -> x*R^-1 (REDC of x with zero upper half; bn128_Fr_mont.c:330) */
static void f_to_std(const fld_t *F, const u64 *a, u64 *o) {
  u64 one[MAXL] = {1, 0, 0, 0, 0, 0};
  f_mul(F, a, one, o);
}
/* x -> x*R (bn128_Fr_mont.c:325: multiply by R^2) */
static void f_from_std(const fld_t *F, const u64 *a, u64 *o) { f_mul(F, a, F->r2, o); }

/* inverse by Fermat a^(p-2); 0 maps to 0 like the reference's Euclid
 * (bn128_Fr_std.c:298-301 returns 0 for 0; bn128_Fr_mont.c:201 then scales by R^3) */
static void f_inv(const fld_t *F, const u64 *a, u64 *o) {
  if (f_is_zero(F, a)) { f_zero(F, o); return; }
  u64 e[MAXL], two[MAXL] = {2, 0, 0, 0, 0, 0};
  raw_sub(F->nl, F->p, two, e);
  u64 acc[MAXL], base[MAXL];
  f_one(F, acc);
  f_copy(F, a, base);
  for (int i = 0; i < F->nl; i++)
    for (int bit = 0; bit < 64; bit++) {
      if ((e[i] >> bit) & 1) f_mul(F, acc, base, acc);
      f_sqr(F, base, base);
    }
  f_copy(F, acc, o);
}
/* x/2 on the representation (bn128_Fr_std.c:241-244) */
static void f_div2(const fld_t *F, const u64 *a, u64 *o) {
  u64 t[MAXL + 1];
  f_copy(F, a, t);
  u64 hi = 0;
  if (t[0] & 1) hi = raw_add(F->nl, t, F->p, t);
  for (int i = 0; i < F->nl; i++) {
    u64 nxt = (i + 1 < F->nl) ? t[i + 1] : hi;
    t[i] = (t[i] >> 1) | (nxt << 63);
  }
  f_copy(F, t, o);
}
static void f_small_mul(const fld_t *F, const u64 *a, int k, u64 *o) {
  u64 acc[MAXL];
  f_zero(F, acc);
  for (int i = 0; i < k; i++) f_add(F, acc, a, acc);
  f_copy(F, acc, o);
}

/* ------------------------------------------------------------ projective G1 (a = 0) ---- */
/* point layout: X | Y | Z, each nl limbs */
#define PX(P) (P)
#define PY(P) ((P) + F->nl)
#define PZ(P) ((P) + 2 * F->nl)

static void p_set_inf(const fld_t *F, u64 *P) {   /* bn128_G1_proj.c:183-187 */
  f_zero(F, PX(P)); f_one(F, PY(P)); f_zero(F, PZ(P));
}
static int p_is_inf(const fld_t *F, const u64 *P) { /* bn128_G1_proj.c:177-181 */
  return f_is_zero(F, PZ(P)) && !f_is_zero(F, PY(P)) && f_is_zero(F, PX(P));
}
static int a_is_inf(const fld_t *F, const u64 *A) { /* bn128_G1_affine.c:57-60 */
  return f_is_zero(F, A) && f_is_zero(F, A + F->nl);
}
static void p_from_affine(const fld_t *F, const u64 *A, u64 *P) { /* bn128_G1_proj.c:120-128 */
  if (a_is_inf(F, A)) { p_set_inf(F, P); return; }
  f_copy(F, A, PX(P)); f_copy(F, A + F->nl, PY(P)); f_one(F, PZ(P));
}
/* Z == 0 -> all 0xff bytes; else (X/Z, Y/Z) (bn128_G1_proj.c:132-144) */
static void p_to_affine(const fld_t *F, const u64 *P, u64 *A) {
  if (f_is_zero(F, PZ(P))) { memset(A, 0xff, 16 * F->nl); return; }
  u64 zi[MAXL];
  f_inv(F, PZ(P), zi);
  f_mul(F, PX(P), zi, A);
  f_mul(F, PY(P), zi, A + F->nl);
}

/* dbl-2007-bl (bn128_G1_proj.c:230-263) */
static void p_dbl(const fld_t *F, const u64 *P, u64 *O) {
  u64 XX[MAXL], ZZ[MAXL], w[MAXL], s[MAXL], ss[MAXL], R[MAXL], RR[MAXL], B[MAXL], h[MAXL], t[MAXL];
  f_sqr(F, PX(P), XX);
  f_sqr(F, PZ(P), ZZ);
  f_add(F, XX, XX, w); f_add(F, w, XX, w);            /* w = 3 XX (a = 0) */
  f_mul(F, PY(P), PZ(P), s); f_add(F, s, s, s);       /* s = 2 Y Z */
  f_sqr(F, s, ss);
  f_mul(F, PY(P), s, R);
  f_sqr(F, R, RR);
  f_add(F, PX(P), R, B); f_sqr(F, B, B); f_sub(F, B, XX, B); f_sub(F, B, RR, B);
  f_sqr(F, w, h); f_sub(F, h, B, h); f_sub(F, h, B, h);
  u64 X3[MAXL], Y3[MAXL], Z3[MAXL];
  f_mul(F, s, ss, Z3);
  f_mul(F, h, s, X3);
  f_sub(F, B, h, t); f_mul(F, t, w, Y3); f_sub(F, Y3, RR, Y3); f_sub(F, Y3, RR, Y3);
  f_copy(F, X3, PX(O)); f_copy(F, Y3, PY(O)); f_copy(F, Z3, PZ(O));
}

/* complete addition add-2015-rcb for a = 0 (bn128_G1_proj.c:272-313) */
static void p_add(const fld_t *F, int b3, const u64 *P, const u64 *Q, u64 *O) {
  u64 t0[MAXL], t1[MAXL], t2[MAXL], t3[MAXL], t4[MAXL], t5[MAXL], X3[MAXL], Y3[MAXL], Z3[MAXL];
  f_mul(F, PX(P), PX(Q), t0);
  f_mul(F, PY(P), PY(Q), t1);
  f_mul(F, PZ(P), PZ(Q), t2);
  f_add(F, PX(P), PY(P), t3); f_add(F, PX(Q), PY(Q), t4); f_mul(F, t3, t4, t3);
  f_add(F, t0, t1, t4); f_sub(F, t3, t4, t3);
  f_add(F, PX(P), PZ(P), t4); f_add(F, PX(Q), PZ(Q), t5); f_mul(F, t4, t5, t4);
  f_add(F, t0, t2, t5); f_sub(F, t4, t5, t4);
  f_add(F, PY(P), PZ(P), t5); f_add(F, PY(Q), PZ(Q), X3); f_mul(F, t5, X3, t5);
  f_add(F, t1, t2, X3); f_sub(F, t5, X3, t5);
  f_small_mul(F, t2, b3, X3);
  f_copy(F, X3, Z3);
  f_sub(F, t1, Z3, X3);
  f_add(F, Z3, t1, Z3);
  f_mul(F, X3, Z3, Y3);
  f_add(F, t0, t0, t1); f_add(F, t1, t0, t1);
  f_small_mul(F, t4, b3, t4);
  f_mul(F, t1, t4, t0); f_add(F, Y3, t0, Y3);
  f_mul(F, t4, t5, t0);
  f_mul(F, X3, t3, X3); f_sub(F, X3, t0, X3);
  f_mul(F, t1, t3, t0);
  f_mul(F, Z3, t5, Z3); f_add(F, Z3, t0, Z3);
  f_copy(F, X3, PX(O)); f_copy(F, Y3, PY(O)); f_copy(F, Z3, PZ(O));
}

/* mixed addition madd-1998-cmo with the reference's special cases (bn128_G1_proj.c:333-373):
 * P = infinity -> from_affine(A); A = (0,0) -> P; u = v = 0 -> dbl(P) */
static void p_madd(const fld_t *F, const u64 *P, const u64 *A, u64 *O) {
  if (p_is_inf(F, P)) { p_from_affine(F, A, O); return; }
  if (a_is_inf(F, A)) { memmove(O, P, 24 * F->nl); return; }
  const u64 *X2 = A, *Y2 = A + F->nl;
  u64 u[MAXL], uu[MAXL], v[MAXL], vv[MAXL], vvv[MAXL], R[MAXL], Av[MAXL];
  f_mul(F, Y2, PZ(P), u); f_sub(F, u, PY(P), u);
  f_mul(F, X2, PZ(P), v); f_sub(F, v, PX(P), v);
  if (f_is_zero(F, u) && f_is_zero(F, v)) { p_dbl(F, P, O); return; }
  f_sqr(F, u, uu);
  f_sqr(F, v, vv);
  f_mul(F, v, vv, vvv);
  f_mul(F, vv, PX(P), R);
  f_mul(F, uu, PZ(P), Av); f_sub(F, Av, vvv, Av); f_sub(F, Av, R, Av); f_sub(F, Av, R, Av);
  u64 X3[MAXL], Y3[MAXL], Z3[MAXL];
  f_mul(F, v, Av, X3);
  f_mul(F, PZ(P), vvv, Z3);
  f_sub(F, R, Av, R);
  f_mul(F, vvv, PY(P), vvv);
  f_mul(F, u, R, Y3); f_sub(F, Y3, vvv, Y3);
  f_copy(F, X3, PX(O)); f_copy(F, Y3, PY(O)); f_copy(F, Z3, PZ(O));
}

/* scalar multiplication k*P with a plain double-and-add over all bits of k
 * (same group result as bn128_G1_proj.c:379-400 scl_naive) */
static void p_scl(const fld_t *F, int b3, const u64 *k, int klimbs, const u64 *P, u64 *O) {
  u64 acc[3 * MAXL], dbl[3 * MAXL];
  p_set_inf(F, acc);
  memcpy(dbl, P, 24 * F->nl);
  for (int i = 0; i < klimbs; i++)
    for (int bit = 0; bit < 64; bit++) {
      if ((k[i] >> bit) & 1) p_add(F, b3, acc, dbl, acc);
      p_add(F, b3, dbl, dbl, dbl);
    }
  memcpy(O, acc, 24 * F->nl);
}

/* ----------------------------------------------------------------------------- MSM ---- */

/* Pippenger with unsigned c-bit windows over all 64*nlimbs scalar bits, buckets madd'ed,
 * running-sum reduce, c doublings per window (bn128_G1_proj.c:506-586). */
static void msm_std_variable(const curve_t *C, int n, const u64 *expos, const u64 *grps,
                             u64 *tgt, int nlimbs, int c) {
  const fld_t *F = C->fp;
  const int nl = F->nl;
  const int nbits = 64 * nlimbs;
  const int nwin = (nbits + c - 1) / c;
  const long nb = 1L << c;
  u64 *S = (u64 *)malloc(sizeof(u64) * 3 * nl * (size_t)(nb - 1));
  p_set_inf(F, tgt);
  for (int K = nwin - 1; K >= 0; K--) {
    int A = K * c, B = A + c;
    if (B > nbits) B = nbits;
    for (long b = 0; b < nb - 1; b++) p_set_inf(F, S + 3 * nl * b);
    for (int j = 0; j < n; j++) {
      const u64 *e = expos + (size_t)nlimbs * j;
      u64 d = 0;
      for (int bit = A; bit < B; bit++) d |= ((e[bit >> 6] >> (bit & 63)) & 1ULL) << (bit - A);
      if (d) {
        u64 *Sb = S + 3 * nl * (d - 1);
        p_madd(F, Sb, grps + (size_t)2 * nl * j, Sb);
      }
    }
    u64 T[3 * MAXL], R[3 * MAXL];
    p_set_inf(F, T);
    p_set_inf(F, R);
    for (long b = nb - 1; b > 0; b--) {
      p_add(F, C->b3, T, S + 3 * nl * (b - 1), T);
      p_add(F, C->b3, R, T, R);
    }
    if (!p_is_inf(F, tgt))
      for (int i = 0; i < c; i++) p_dbl(F, tgt, tgt);
    p_add(F, C->b3, tgt, R, tgt);
  }
  free(S);
}

/* window choice c = round(log2 n - 3.5) clamped to [1, 64] (bn128_G1_proj.c:597-605) */
int oracle_msm_window(int n) {
  double c = round(log2((double)n) - 3.5);
  if (!(c >= 1)) c = 1;   /* also catches n = 0 (log2 -> -inf) */
  if (c > 64) c = 64;
  return (int)c;
}

/* curve: 0 = BN254, 1 = BLS12-381. mont != 0: scalars are Montgomery Fr (4 limbs each),
 * converted with to_std first (bn128_G1_proj.c:631-645). window <= 0 uses the reference rule.
 * Output: projective point (3*nl limbs). Returns 0, or -1 on unsupported arguments. */
int oracle_msm_proj(int curve, int n, const u64 *expos, int nlimbs, int mont,
                    const u64 *grps, u64 *tgt, int window) {
  const curve_t *C = &CURVES[curve];
  if (n < 0 || nlimbs < 1 || (mont && nlimbs != 4)) return -1;
  int c = window > 0 ? window : oracle_msm_window(n);
  if (c > 30) return -1;
  const u64 *use = expos;
  u64 *conv = NULL;
  if (mont) {
    conv = (u64 *)malloc(sizeof(u64) * 4 * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) f_to_std(C->fr, expos + 4 * (size_t)i, conv + 4 * (size_t)i);
    use = conv;
  }
  msm_std_variable(C, n, use, grps, tgt, nlimbs, c);
  free(conv);
  return 0;
}

void oracle_proj_to_affine(int curve, const u64 *P, u64 *A) { p_to_affine(CURVES[curve].fp, P, A); }

/* complete projective addition (bn128_G1_proj.c:272-313) */
void oracle_proj_add(int curve, const u64 *P, const u64 *Q, u64 *O) {
  p_add(CURVES[curve].fp, CURVES[curve].b3, P, Q, O);
}

/* Jacobian coordinates of the same point (reference jac infinity is [1:1:0],
 * lib/cbits/curves/g1/jac/bn128_G1_jac.c:182-187). From projective (X:Y:Z), x = X/Z, y = Y/Z:
 * Jacobian (X Z : Y Z^2 : Z). */
void oracle_proj_to_jac(int curve, const u64 *P, u64 *J) {
  const fld_t *F = CURVES[curve].fp;
  if (f_is_zero(F, PZ(P))) { f_one(F, J); f_one(F, J + F->nl); f_zero(F, J + 2 * F->nl); return; }
  u64 zz[MAXL];
  f_sqr(F, PZ(P), zz);
  f_mul(F, PX(P), PZ(P), J);
  f_mul(F, PY(P), zz, J + F->nl);
  f_copy(F, PZ(P), J + 2 * F->nl);
}

/* Jacobian -> affine with the 0xff rule (bn128_G1_jac.c:120-135) */
void oracle_jac_to_affine(int curve, const u64 *J, u64 *A) {
  const fld_t *F = CURVES[curve].fp;
  if (f_is_zero(F, J + 2 * F->nl)) { memset(A, 0xff, 16 * F->nl); return; }
  u64 zi[MAXL], zi2[MAXL], zi3[MAXL];
  f_inv(F, J + 2 * F->nl, zi);
  f_sqr(F, zi, zi2);
  f_mul(F, zi, zi2, zi3);
  f_mul(F, J, zi2, A);
  f_mul(F, J + F->nl, zi3, A + F->nl);
}

/* k_i * G for standard-form scalars k_i (4 limbs each), affine Montgomery output, infinity
 * written as (0,0) (the base generator of the reference's tests: rndG1 = k*G,
 * lib/src/ZK/Algebra/Curves/BN128/G1/Affine.hs). Fixed-base comb over 8-bit digits:
 * T[j][v] = v * 256^j * G, 32 complete additions per point, then one batched inversion
 * (Montgomery's trick) for the affine conversion. Any correct scalar multiplication gives the
 * same affine point; the tests pin this one against the reference's scl_Fr_std. */
void oracle_gen_bases(int curve, int n, const u64 *ks, u64 *out) {
  const curve_t *C = &CURVES[curve];
  const fld_t *F = C->fp;
  const int nl = F->nl, pw = 3 * nl;
  u64 *T = (u64 *)malloc(sizeof(u64) * pw * 32 * 256);
  u64 base[3 * MAXL];
  f_from_std(F, C->gen_std[0], PX(base));
  f_from_std(F, C->gen_std[1], PY(base));
  f_one(F, PZ(base));
  for (int j = 0; j < 32; j++) {
    p_set_inf(F, T + (size_t)(j * 256) * pw);
    for (int v = 1; v < 256; v++)
      p_add(F, C->b3, T + (size_t)(j * 256 + v - 1) * pw, base, T + (size_t)(j * 256 + v) * pw);
    for (int d = 0; d < 8; d++) p_add(F, C->b3, base, base, base);
  }
  u64 *P = (u64 *)malloc(sizeof(u64) * pw * (size_t)(n > 0 ? n : 1));
  u64 *pref = (u64 *)malloc(sizeof(u64) * nl * (size_t)(n > 0 ? n : 1));
  u64 acc[MAXL];
  f_one(F, acc);
  for (int i = 0; i < n; i++) {
    u64 *Pi = P + (size_t)i * pw;
    p_set_inf(F, Pi);
    const u64 *k = ks + 4 * (size_t)i;
    for (int j = 0; j < 32; j++) {
      const unsigned d = (unsigned)((k[j >> 3] >> (8 * (j & 7))) & 0xff);
      if (d) p_add(F, C->b3, Pi, T + (size_t)(j * 256 + d) * pw, Pi);
    }
    /* prefix products of the non-zero Z coordinates */
    if (!f_is_zero(F, PZ(Pi))) f_mul(F, acc, PZ(Pi), acc);
    f_copy(F, acc, pref + (size_t)i * nl);
  }
  u64 inv[MAXL];
  f_inv(F, acc, inv);   /* 1 / prod of all non-zero Z */
  for (int i = n - 1; i >= 0; i--) {
    u64 *Pi = P + (size_t)i * pw;
    u64 *o = out + 2 * (size_t)nl * i;
    if (f_is_zero(F, PZ(Pi))) { memset(o, 0, 16 * nl); continue; }
    u64 zi[MAXL], prev[MAXL];
    if (i > 0) f_copy(F, pref + (size_t)(i - 1) * nl, prev); else f_one(F, prev);
    f_mul(F, inv, prev, zi);           /* 1/Z_i */
    f_mul(F, inv, PZ(Pi), inv);        /* drop Z_i from the running inverse */
    f_mul(F, PX(Pi), zi, o);
    f_mul(F, PY(Pi), zi, o + nl);
  }
  free(pref);
  free(P);
  free(T);
}

/* sum_i a_i * b_i mod r for standard-form Fr values (4 limbs each); standard-form result */
void oracle_fr_dot_std(int curve, int n, const u64 *a, const u64 *b, u64 *out) {
  const fld_t *F = CURVES[curve].fr;
  u64 acc[MAXL], x[MAXL], t[MAXL];
  f_zero(F, acc);
  for (int i = 0; i < n; i++) {
    f_from_std(F, a + 4 * (size_t)i, x);
    f_mul(F, x, b + 4 * (size_t)i, t);   /* (a R) * b / R = a b */
    f_add(F, acc, t, acc);
  }
  f_copy(F, acc, out);
}

/* ----------------------------------------------------------------------------- NTT ---- */

/* forward DIT recursion (bn128_poly_mont.c:418-447) */
static void ntt_fwd_rec(const fld_t *F, int m, int stride, const u64 *gp, const u64 *src, u64 *buf, u64 *tgt) {
  const int nl = F->nl;
  if (m == 0) { f_copy(F, src, tgt); return; }
  if (m == 1) {
    f_add(F, src, src + (size_t)stride * nl, tgt);
    f_sub(F, src, src + (size_t)stride * nl, tgt + nl);
    return;
  }
  const size_t N = (size_t)1 << m, half = N >> 1;
  ntt_fwd_rec(F, m - 1, stride << 1, gp, src, buf + N * nl, buf);
  ntt_fwd_rec(F, m - 1, stride << 1, gp, src + (size_t)stride * nl, buf + N * nl, buf + half * nl);
  for (size_t j = 0; j < half; j++) {
    u64 t[MAXL];
    f_mul(F, buf + (j + half) * nl, gp + j * stride * nl, t);
    f_add(F, buf + j * nl, t, tgt + j * nl);
    f_sub(F, buf + j * nl, t, tgt + (j + half) * nl);
  }
}

/* inverse DIF recursion with halving per stage (bn128_poly_mont.c:565-596) */
static void ntt_inv_rec(const fld_t *F, int m, int stride, const u64 *gp, const u64 *src, u64 *buf, u64 *tgt) {
  const int nl = F->nl;
  if (m == 0) { f_copy(F, src, tgt); return; }
  if (m == 1) {
    u64 a[MAXL], b[MAXL];
    f_add(F, src, src + nl, a);
    f_sub(F, src, src + nl, b);
    f_div2(F, a, tgt);
    f_div2(F, b, tgt + (size_t)stride * nl);
    return;
  }
  const size_t N = (size_t)1 << m, half = N >> 1;
  for (size_t j = 0; j < half; j++) {
    u64 a[MAXL], b[MAXL];
    f_add(F, src + j * nl, src + (j + half) * nl, a);
    f_sub(F, src + j * nl, src + (j + half) * nl, b);
    f_div2(F, a, buf + j * nl);
    f_mul(F, b, gp + j * stride * nl, buf + (j + half) * nl);
  }
  ntt_inv_rec(F, m - 1, stride << 1, gp, buf, buf + N * nl, tgt);
  ntt_inv_rec(F, m - 1, stride << 1, gp, buf + half * nl, buf + N * nl, tgt + (size_t)stride * nl);
}

/* forward: gpows[i] = g^i (bn128_poly_mont.c:452-473); inverse: gpows[i] = g^-i / 2
 * (bn128_poly_mont.c:601-622). Twiddle tables sized max(N/2, 1) (the reference writes
 * two entries even for N <= 2). curve selects Fr of BN254 (0) or BLS12-381 (1). */
int oracle_ntt(int curve, int m, const u64 *gen, const u64 *src, u64 *tgt, int inverse) {
  const fld_t *F = CURVES[curve].fr;
  const int nl = F->nl;
  if (m < 0 || m > 30) return -1;
  const size_t N = (size_t)1 << m, half = N > 1 ? N / 2 : 1;
  u64 *gp = (u64 *)malloc(sizeof(u64) * nl * (half + 1));
  u64 *buf = (u64 *)malloc(sizeof(u64) * nl * 2 * N);
  if (!gp || !buf) { free(gp); free(buf); return -2; }
  u64 x[MAXL], step[MAXL];
  if (!inverse) {
    f_one(F, x);
    f_copy(F, gen, step);
  } else {
    u64 two[MAXL] = {2, 0, 0, 0, 0, 0}, twom[MAXL];
    f_from_std(F, two, twom);
    f_inv(F, twom, x);          /* 1/2 (bn128_poly_mont.c:563) */
    f_inv(F, gen, step);
  }
  for (size_t i = 0; i < half; i++) {
    f_copy(F, x, gp + i * nl);
    f_mul(F, x, step, x);
  }
  if (!inverse) ntt_fwd_rec(F, m, 1, gp, src, buf, tgt);
  else ntt_inv_rec(F, m, 1, gp, src, buf, tgt);
  free(gp);
  free(buf);
  return 0;
}

/* f(eta x) evaluations: pre-multiply src[i] by eta^i, then the forward NTT
 * (bn128_poly_mont.c:477-488 ntt_forward_shifted); inverse: the inverse NTT, then multiply output
 * i by eta^i (bn128_poly_mont.c:626-641 ntt_inverse_shifted). Powers by repeated products. */
int oracle_ntt_shifted(int curve, int m, const u64 *eta, const u64 *gen, const u64 *src, u64 *tgt, int inverse) {
  const fld_t *F = CURVES[curve].fr;
  const int nl = F->nl;
  if (m < 0 || m > 30) return -1;
  const size_t N = (size_t)1 << m;
  u64 *tmp = (u64 *)malloc(sizeof(u64) * nl * N);
  u64 x[MAXL];
  if (!inverse) {
    f_one(F, x);
    for (size_t i = 0; i < N; i++) {
      f_mul(F, src + i * nl, x, tmp + i * nl);
      f_mul(F, x, eta, x);
    }
    int rc = oracle_ntt(curve, m, gen, tmp, tgt, 0);
    free(tmp);
    return rc;
  }
  int rc = oracle_ntt(curve, m, gen, src, tmp, 1);
  f_one(F, x);
  for (size_t i = 0; i < N; i++) {
    f_mul(F, tmp + i * nl, x, tgt + i * nl);
    f_mul(F, x, eta, x);
  }
  free(tmp);
  return rc;
}

/* evaluation of a size-2^m_src polynomial on the size-2^m_tgt subgroup: for k < K = 2^(m_tgt-m_src)
 * the NTT (generator gen_src) of src[i] * gen_tgt^(k i), written to tgt[i K + k]
 * (bn128_poly_mont.c:492-555 ntt_forward_asymmetric; k = 0 uses src unscaled) */
int oracle_ntt_asymmetric(int curve, int m_src, int m_tgt, const u64 *gen_src, const u64 *gen_tgt, const u64 *src,
                          u64 *tgt) {
  const fld_t *F = CURVES[curve].fr;
  const int nl = F->nl;
  if (m_src < 0 || m_tgt < m_src || m_tgt > 30) return -1;
  const size_t Ns = (size_t)1 << m_src, K = (size_t)1 << (m_tgt - m_src);
  u64 *out = (u64 *)malloc(sizeof(u64) * nl * Ns);
  u64 eta[MAXL];
  f_one(F, eta);
  for (size_t k = 0; k < K; k++) {
    if (k) f_mul(F, eta, gen_tgt, eta);
    if (oracle_ntt_shifted(curve, m_src, eta, gen_src, src, out, 0)) { free(out); return -1; }
    for (size_t i = 0; i < Ns; i++) f_copy(F, out + i * nl, tgt + (i * K + k) * nl);
  }
  free(out);
  return 0;
}

/* polynomial evaluation at a point by Horner (bn128_poly_mont.c:225 eval_at) */
void oracle_eval_at(int curve, int n, const u64 *coeffs, const u64 *x, u64 *out) {
  const fld_t *F = CURVES[curve].fr;
  u64 acc[MAXL];
  f_zero(F, acc);
  for (int i = n - 1; i >= 0; i--) {
    f_mul(F, acc, x, acc);
    f_add(F, acc, coeffs + (size_t)i * F->nl, acc);
  }
  f_copy(F, acc, out);
}

/* -------------------------------------------------------------------- binary MSMs ---- */

/* sum of the bases whose byte coefficient is non-zero, by mixed additions into a projective
 * accumulator (bn128_G1_proj.c:684-692). Output: projective point. */
void oracle_msm_binary(int curve, int n, const uint8_t *expos, const u64 *grps, u64 *tgt) {
  const fld_t *F = CURVES[curve].fp;
  p_set_inf(F, tgt);
  for (int i = 0; i < n; i++)
    if (expos[i]) p_madd(F, tgt, grps + (size_t)2 * F->nl * i, tgt);
}

/* rows of an nrows x npoints byte matrix (row-major here; the reference takes row pointers),
 * each summed over the same bases with the reference's windowed subset-sum tables
 * (bn128_G1_proj.c:718-770): c = round(1.22 ln(nrows) - 0.5) clamped to [1, 15]; per window of
 * c points, PRECALC[i + 2^j] = PRECALC[i] + P_j; each row adds PRECALC[idx]. Output: nrows
 * projective points. */
int oracle_multi_msm_binary(int curve, int nrows, int npoints, const uint8_t *coeffs, const u64 *grps, u64 *tgt) {
  const curve_t *C = &CURVES[curve];
  const fld_t *F = C->fp;
  const int nl = F->nl, pw = 3 * nl;
  if (nrows <= 0) return 0;
  int c = (int)round(1.22 * log((double)nrows) - 0.5);
  if (c < 1) c = 1;
  if (c > 15) c = 15;
  for (int i = 0; i < nrows; i++) p_set_inf(F, tgt + (size_t)i * pw);
  u64 *pre = (u64 *)malloc(sizeof(u64) * pw * ((size_t)1 << c));
  if (!pre) return -2;
  p_set_inf(F, pre);
  const int nwin = (npoints + c - 1) / c;
  for (int k = 0; k < nwin; k++) {
    const int A = k * c, B = (A + c < npoints) ? A + c : npoints, W = B - A;
    for (int j = 0; j < W; j++) {
      const u64 *g = grps + (size_t)2 * nl * (A + j);
      if (j == 0) { p_from_affine(F, g, pre + pw); continue; }
      const size_t m = (size_t)1 << j;
      for (size_t i = 0; i < m; i++) p_madd(F, pre + i * pw, g, pre + (i + m) * pw);
    }
    for (int r = 0; r < nrows; r++) {
      size_t idx = 0;
      for (int j = 0; j < W; j++)
        if (coeffs[(size_t)r * npoints + A + j]) idx |= (size_t)1 << j;
      if (idx) p_add(F, C->b3, tgt + (size_t)r * pw, pre + idx * pw, tgt + (size_t)r * pw);
    }
  }
  free(pre);
  return 0;
}

/* ------------------------------------------------------------------- G1 group FFT ---- */

/* [k]P for a Montgomery Fr element k: to_std, then double-and-add
 * (bn128_G1_proj.c:478-482 scl_Fr_mont; any correct scalar multiplication gives the same point) */
static void p_scl_fr_mont(const curve_t *C, const u64 *k_mont, const u64 *P, u64 *O) {
  u64 k[MAXL];
  f_to_std(C->fr, k_mont, k);
  p_scl(C->fp, C->b3, k, 4, P, O);
}
static void p_sub(const curve_t *C, const u64 *P, const u64 *Q, u64 *O) {
  const fld_t *F = C->fp;
  u64 nq[3 * MAXL];
  memcpy(nq, Q, 24 * F->nl);
  f_neg(F, PY(nq), PY(nq));
  p_add(F, C->b3, P, nq, O);
}

/* forward DIT recursion over points (bn128_G1_proj.c:791-824) */
static void g1fft_fwd_rec(const curve_t *C, int m, int stride, const u64 *gen, const u64 *src, u64 *buf, u64 *tgt) {
  const fld_t *F = C->fp;
  const int pw = 3 * F->nl;
  if (m == 0) { memcpy(tgt, src, 8 * pw); return; }
  if (m == 1) {
    p_add(F, C->b3, src, src + (size_t)stride * pw, tgt);
    p_sub(C, src, src + (size_t)stride * pw, tgt + pw);
    return;
  }
  const size_t N = (size_t)1 << m, half = N >> 1;
  u64 g2[MAXL], gp[MAXL];
  f_sqr(C->fr, gen, g2);
  g1fft_fwd_rec(C, m - 1, stride << 1, g2, src, buf + N * pw, buf);
  g1fft_fwd_rec(C, m - 1, stride << 1, g2, src + (size_t)stride * pw, buf + N * pw, buf + half * pw);
  f_one(C->fr, gp);
  for (size_t j = 0; j < half; j++) {
    u64 t[3 * MAXL], u[3 * MAXL];
    p_scl_fr_mont(C, gp, buf + (j + half) * pw, t);
    memcpy(u, buf + j * pw, 8 * pw);
    p_add(F, C->b3, u, t, tgt + j * pw);
    p_sub(C, u, t, tgt + (j + half) * pw);
    f_mul(C->fr, gp, gen, gp);
  }
}

/* inverse DIF recursion over points, halving at every level (bn128_G1_proj.c:853-890) */
static void g1fft_inv_rec(const curve_t *C, int m, int tstride, const u64 *gen, const u64 *src, u64 *buf, u64 *tgt) {
  const fld_t *F = C->fp;
  const int pw = 3 * F->nl;
  u64 half_m[MAXL], two[MAXL] = {2, 0, 0, 0, 0, 0}, twom[MAXL];
  f_from_std(C->fr, two, twom);
  f_inv(C->fr, twom, half_m);               /* 1/2 in Montgomery form (bn128_G1_proj.c:851) */
  if (m == 0) { memcpy(tgt, src, 8 * pw); return; }
  if (m == 1) {
    u64 a[3 * MAXL], b[3 * MAXL];
    p_add(F, C->b3, src, src + pw, a);
    p_sub(C, src, src + pw, b);
    p_scl_fr_mont(C, half_m, a, tgt);
    p_scl_fr_mont(C, half_m, b, tgt + (size_t)tstride * pw);
    return;
  }
  const size_t N = (size_t)1 << m, half = N >> 1;
  u64 ginv[MAXL], gp[MAXL], g2[MAXL];
  f_inv(C->fr, gen, ginv);
  f_copy(C->fr, half_m, gp);
  for (size_t j = 0; j < half; j++) {
    u64 a[3 * MAXL], b[3 * MAXL];
    p_add(F, C->b3, src + j * pw, src + (j + half) * pw, a);
    p_sub(C, src + j * pw, src + (j + half) * pw, b);
    p_scl_fr_mont(C, half_m, a, buf + j * pw);
    p_scl_fr_mont(C, gp, b, buf + (j + half) * pw);
    f_mul(C->fr, gp, ginv, gp);
  }
  f_sqr(C->fr, gen, g2);
  g1fft_inv_rec(C, m - 1, tstride << 1, g2, buf, buf + N * pw, tgt);
  g1fft_inv_rec(C, m - 1, tstride << 1, g2, buf + half * pw, buf + N * pw, tgt + (size_t)tstride * pw);
}

/* normalisation (bn128_G1_proj.c:78-97): Z = 0 -> (0, 1, 0); else (X/Z, Y/Z, 1) */
static void p_normalize(const fld_t *F, const u64 *P, u64 *O) {
  if (f_is_zero(F, PZ(P))) { p_set_inf(F, O); return; }
  u64 zi[MAXL], x[MAXL], y[MAXL];
  f_inv(F, PZ(P), zi);
  f_mul(F, PX(P), zi, x);
  f_mul(F, PY(P), zi, y);
  f_copy(F, x, PX(O)); f_copy(F, y, PY(O)); f_one(F, PZ(O));
}

/* *_G1_{proj,jac}_fft_{forward,inverse} (bn128_G1_proj.c:831-842, 893-902; Jacobian twins
 * bn128_G1_jac.c:880-950): jac != 0 reads Jacobian inputs (x = X/Z^2, y = Y/Z^3), converted to
 * projective (X Z : Y : Z^3) first. Outputs normalised, (x, y, 1) or (0, 1, 0), which is also
 * the Jacobian normal form (bn128_G1_jac.c:62-85). */
int oracle_g1_fft(int curve, int jac, int m, const u64 *gen, const u64 *src, u64 *tgt, int inverse) {
  const curve_t *C = &CURVES[curve];
  const fld_t *F = C->fp;
  const int pw = 3 * F->nl;
  if (m < 0 || m > 20) return -1;
  const size_t N = (size_t)1 << m;
  u64 *in = (u64 *)malloc(sizeof(u64) * pw * N);
  u64 *buf = (u64 *)malloc(sizeof(u64) * pw * 2 * N);
  u64 *out = (u64 *)malloc(sizeof(u64) * pw * N);
  if (!in || !buf || !out) { free(in); free(buf); free(out); return -2; }
  for (size_t i = 0; i < N; i++) {
    const u64 *s = src + i * pw;
    u64 *d = in + i * pw;
    if (!jac) { memcpy(d, s, 8 * pw); continue; }
    if (f_is_zero(F, PZ(s))) { p_set_inf(F, d); continue; }
    u64 zz[MAXL];
    f_sqr(F, PZ(s), zz);
    f_mul(F, PX(s), PZ(s), PX(d));
    f_copy(F, PY(s), PY(d));
    f_mul(F, zz, PZ(s), PZ(d));
  }
  if (!inverse) g1fft_fwd_rec(C, m, 1, gen, in, buf, out);
  else g1fft_inv_rec(C, m, 1, gen, in, buf, out);
  for (size_t i = 0; i < N; i++) p_normalize(F, out + i * pw, tgt + i * pw);
  free(in); free(buf); free(out);
  return 0;
}

/* ------------------------------------------------------------- Fr vector operations ---- */

/* batch inversion by partial products (bn128_Fr_mont.c:258-285): one inversion of the full
 * product, so a zero anywhere gives all-zero outputs; n >= 1 */
static void fr_batch_inv(const fld_t *F, int n, const u64 *src, u64 *tgt) {
  const int nl = F->nl;
  u64 *prods = (u64 *)malloc(sizeof(u64) * nl * (size_t)n);
  u64 *recips = (u64 *)malloc(sizeof(u64) * nl * (size_t)n);
  f_copy(F, src, prods);
  for (int i = 1; i < n; i++) f_mul(F, prods + (size_t)(i - 1) * nl, src + (size_t)i * nl, prods + (size_t)i * nl);
  f_inv(F, prods + (size_t)(n - 1) * nl, recips + (size_t)(n - 1) * nl);
  for (int i = n - 2; i >= 0; i--)
    f_mul(F, recips + (size_t)(i + 1) * nl, src + (size_t)(i + 1) * nl, recips + (size_t)i * nl);
  u64 first[MAXL];
  f_copy(F, recips, first);
  for (int i = n - 1; i >= 1; i--) f_mul(F, recips + (size_t)i * nl, prods + (size_t)(i - 1) * nl, tgt + (size_t)i * nl);
  f_copy(F, first, tgt);
  free(prods);
  free(recips);
}

/* element-wise operations of the *_arr_mont_* module (bn128_arr_mont.c:94-278); op codes as
 * ZKG_FR_* of the product header: 0 from_std, 1 to_std, 2 neg, 3 add, 4 sub, 5 sqr, 6 mul, 7 inv,
 * 8 div, 9 mul_add, 10 mul_sub, 11 scale, 12 Ax+y, 13 Ax+By, 14 powers, 15 mul_by_powers (tgt[0]
 * untouched, tgt[i] = src[i] A B^(i-1), bn128_arr_mont.c:208-216). Returns -1 on a bad op. */
int oracle_fr_op(int curve, int op, int n, const u64 *a, const u64 *b, const u64 *c, const u64 *ka, const u64 *kb,
                 u64 *out) {
  const fld_t *F = CURVES[curve].fr;
  const int nl = F->nl;
  if (n <= 0) return 0;
  if (op == 7 || op == 8) {
    u64 *tmp = (u64 *)malloc(sizeof(u64) * nl * (size_t)n);
    fr_batch_inv(F, n, op == 7 ? a : b, tmp);
    for (int i = 0; i < n; i++) {
      if (op == 7) f_copy(F, tmp + (size_t)i * nl, out + (size_t)i * nl);
      else f_mul(F, a + (size_t)i * nl, tmp + (size_t)i * nl, out + (size_t)i * nl);
    }
    free(tmp);
    return 0;
  }
  if (op == 14) {   /* bn128_arr_mont.c:199-205 */
    f_copy(F, ka, out);
    for (int i = 1; i < n; i++) f_mul(F, out + (size_t)(i - 1) * nl, kb, out + (size_t)i * nl);
    return 0;
  }
  if (op == 15) {
    u64 x[MAXL];
    f_copy(F, ka, x);
    for (int i = 1; i < n; i++) {
      f_mul(F, a + (size_t)i * nl, x, out + (size_t)i * nl);
      f_mul(F, x, kb, x);
    }
    return 0;
  }
  for (int i = 0; i < n; i++) {
    const u64 *ai = a + (size_t)i * nl, *bi = b ? b + (size_t)i * nl : NULL, *ci = c ? c + (size_t)i * nl : NULL;
    u64 r[MAXL], t[MAXL];
    switch (op) {
      case 0: f_from_std(F, ai, r); break;
      case 1: f_to_std(F, ai, r); break;
      case 2: f_neg(F, ai, r); break;
      case 3: f_add(F, ai, bi, r); break;
      case 4: f_sub(F, ai, bi, r); break;
      case 5: f_sqr(F, ai, r); break;
      case 6: f_mul(F, ai, bi, r); break;
      case 9: f_mul(F, ai, bi, r); f_add(F, r, ci, r); break;
      case 10: f_mul(F, ai, bi, r); f_sub(F, r, ci, r); break;
      case 11: f_mul(F, ka, ai, r); break;
      case 12: f_mul(F, ka, ai, r); f_add(F, r, bi, r); break;
      case 13: f_mul(F, ka, ai, r); f_mul(F, kb, bi, t); f_add(F, r, t, r); break;
      default: return -1;
    }
    f_copy(F, r, out + (size_t)i * nl);
  }
  return 0;
}

/* sum of a[i] b[i] (bn128_arr_mont.c:187-196) */
void oracle_fr_dot(int curve, int n, const u64 *a, const u64 *b, u64 *out) {
  const fld_t *F = CURVES[curve].fr;
  u64 acc[MAXL], t[MAXL];
  f_zero(F, acc);
  for (int i = 0; i < n; i++) {
    f_mul(F, a + (size_t)i * F->nl, b + (size_t)i * F->nl, t);
    f_add(F, acc, t, acc);
  }
  f_copy(F, acc, out);
}

/* tgt = A src for a matrix given by K (row, col, coeff) triples (bn128_arr_mont.c:226-237) */
void oracle_fr_sparse(int curve, int N, int K, const u64 *rows, const u64 *cols, const u64 *coeffs, const u64 *src,
                      u64 *tgt) {
  const fld_t *F = CURVES[curve].fr;
  const int nl = F->nl;
  memset(tgt, 0, sizeof(u64) * nl * (size_t)N);
  for (int k = 0; k < K; k++) {
    u64 t[MAXL];
    f_mul(F, coeffs + (size_t)k * nl, src + (size_t)(int)cols[k] * nl, t);
    f_add(F, tgt + (size_t)(int)rows[k] * nl, t, tgt + (size_t)(int)rows[k] * nl);
  }
}

/* ----------------------------------------------------- element-wise helpers for tests ---- */
/* which: 0 = Fp, 1 = Fr; op: 0 to_std, 1 from_std, 2 mul, 3 add, 4 sub, 5 neg, 6 inv, 7 div2 */
void oracle_field_op(int curve, int which, int op, int n, const u64 *a, const u64 *b, u64 *o) {
  const fld_t *F = which ? CURVES[curve].fr : CURVES[curve].fp;
  const int nl = F->nl;
  for (int i = 0; i < n; i++) {
    const u64 *ai = a + (size_t)i * nl, *bi = b ? b + (size_t)i * nl : NULL;
    u64 *oi = o + (size_t)i * nl;
    switch (op) {
      case 0: f_to_std(F, ai, oi); break;
      case 1: f_from_std(F, ai, oi); break;
      case 2: f_mul(F, ai, bi, oi); break;
      case 3: f_add(F, ai, bi, oi); break;
      case 4: f_sub(F, ai, bi, oi); break;
      case 5: f_neg(F, ai, oi); break;
      case 6: f_inv(F, ai, oi); break;
      case 7: f_div2(F, ai, oi); break;
    }
  }
}
