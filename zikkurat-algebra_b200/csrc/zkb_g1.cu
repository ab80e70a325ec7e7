// G1 group FFT and binary MSMs on the device.
//
// Group FFT: the reference's *_G1_{proj,jac}_fft_forward / _fft_inverse
// (lib/cbits/curves/g1/proj/bn128_G1_proj.c:791-902, jac/bn128_G1_jac.c:840-950) are the NTT
// networks of poly_mont with points in place of field elements: a forward DIT whose butterfly
// is (u + [w]v, u - [w]v) and an inverse DIF with (u + v)/2, [w^-1](u - v)/2, where [w]P is a
// scalar multiplication by the standard integer of a Montgomery Fr element. The map from input
// points to output points is Fr-linear, so any evaluation order of the same network gives the
// same group elements. Here:
//   - points live in XYZZ coordinates in one device buffer; the input is written in
//     bit-reversed order for the DIT (natural for the DIF) and stages run in place, one launch
//     per stage, one thread per butterfly;
//   - stage s (block size 2^s) uses the twiddle gen^(j 2^(m-s)) for j < 2^(s-1) (the reference
//     squares the generator per recursion level and multiplies up the powers), read from one
//     table of gen^e, e < N/2, in standard form; j = 0 needs no multiplication;
//   - the inverse's per-level halving, (1/2)^m per output, is folded into the first DIF stage:
//     its sum takes [2^-m] and its difference [2^-m ginv^j];
//   - scalar multiplication uses signed 4-bit windows (digits -7..8, table 1P..8P, 4 doublings
//     per window); the results are converted to the reference's normalised form
//     (bn128_G1_proj.c:78-97; the Jacobian normalisation bn128_G1_jac.c:62-85 writes the same
//     bytes: (x, y, 1), infinity (0, 1, 0)).
//
// Binary MSMs: *_MSM_binary_coeff_* (bn128_G1_proj.c:684-698) sums the bases whose byte
// coefficient is non-zero; *_multi_MSM_binary_coeff_* (bn128_G1_proj.c:718-782) does that for
// each row of an nrows x npoints byte matrix, with the bases split into windows of c columns and
// all 2^c subset sums of a window precomputed, so a row adds one table entry per window. Both
// run here as one pipeline:
//   - "direct" (few rows): thread (row, g) madds the selected affine bases of columns
//     g, g + G, ...;
//   - "windowed" (many rows): per window of c columns the subset-sum table T[k][0..2^c) is built
//     in c level launches (T[k][2^l + i] = T[k][i] + P[kc + l]); thread (row, g) then adds
//     T[k][idx] for windows k = g, g + G, ...;
//   - columns are processed in chunks (host coefficient rows and bases are gathered into pinned
//     staging and copied while the previous chunk computes); per-(row, g) partial sums carry
//     across chunks and are reduced per row at the end.
// The choice between direct and windowed, c and G only changes the order of additions; every
// result is the same group element, written in the drop-in's output encoding.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "zkb_curve.cuh"
#include "zkb_dpf.cuh"
#include "zkb_host_ec.h"
#include "zkb_runtime.h"

namespace zkb {

// ------------------------------------------------------------------------ device helpers
template <class F>
__device__ __noinline__ Xyzz<F> xyzz_sum(Xyzz<F> a, const Xyzz<F> b) {
  xyzz_add(a, b);
  return a;
}

template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_negate(Xyzz<F> p) {
  p.Y = fe_neg(p.Y);
  return p;
}

// Output encodings of the drop-in entry points (the host twin is host::xyzz_write). With CONV, p
// is in the FP64 radix R' (zkb_dpf.cuh) and the coordinates go back to the reference's radix R
// with kout = R mod p, which is also the radix-R form of 1.
template <class F, bool CONV>
__device__ void xyzz_write_out(const Xyzz<F>& p, int kind, uint32_t* __restrict__ out, const Fe<F>& kout) {
  const Fe<F> one = CONV ? kout : fe_one<F>();
  if (xyzz_is_inf(p)) {
    if (kind == ZKG_OUT_AFFINE) {
      for (int i = 0; i < 2 * F::N; i++) out[i] = 0xffffffffu;
      return;
    }
    fe_store<F>(out, kind == ZKG_OUT_JAC ? one : fe_zero<F>());
    fe_store<F>(out + F::N, one);
    fe_store<F>(out + 2 * F::N, fe_zero<F>());
    return;
  }
  const Fe<F> d = fe_inv_fermat(fe_mul(p.ZZ, p.ZZZ));
  Fe<F> x = fe_mul(p.X, fe_mul(d, p.ZZZ)), y = fe_mul(p.Y, fe_mul(d, p.ZZ));
  if (CONV) {
    x = fe_mul(x, kout);
    y = fe_mul(y, kout);
  }
  fe_store<F>(out, x);
  fe_store<F>(out + F::N, y);
  if (kind != ZKG_OUT_AFFINE) fe_store<F>(out + 2 * F::N, one);
}
template <class F>
__device__ void xyzz_write_dev(const Xyzz<F>& p, int kind, uint32_t* __restrict__ out) {
  xyzz_write_out<F, false>(p, kind, out, fe_zero<F>());
}

// [k]P by the GLV endomorphism phi(x, y) = (beta x, y) = [lambda](x, y): k = k1 + k2 lambda
// mod r with |k1|, |k2| < 2^136, split on the host (glv_split). Record g: words 0-4 |k1|,
// words 5-9 |k2| (little-endian), word 10 bit 0 = (k1 < 0), bit 1 = (k2 < 0).
// Both halves use signed 4-bit windows (35 digits in -7..8, the top one the final carry) over
// one table 1P..8P; phi of an entry costs one product (beta X). 4 doublings per window.
__device__ __forceinline__ void glv_digits(const uint32_t* k, uint32_t (&dg)[5]) {   // 35 nibbles, d + 7
#pragma unroll
  for (int i = 0; i < 5; i++) dg[i] = 0;
  uint32_t carry = 0;
#pragma unroll
  for (int w = 0; w < 34; w++) {
    const uint32_t v = ((k[w >> 3] >> (4 * (w & 7))) & 15u) + carry;
    const int d = v > 8 ? (int)v - 16 : (int)v;
    carry = v > 8 ? 1u : 0u;
    dg[w >> 3] |= (uint32_t)(d + 7) << (4 * (w & 7));
  }
  dg[4] |= (carry + 7) << 8;   // window 34
}

template <class F>
__device__ Xyzz<F> xyzz_mul_glv(const uint32_t (&g)[12], const Xyzz<F>& P, const Fe<F>& beta) {
  uint32_t d1[5], d2[5];
  glv_digits(g, d1);
  glv_digits(g + 5, d2);
  const uint32_t s1 = g[10] & 1u, s2 = (g[10] >> 1) & 1u;
  Xyzz<F> T[8];
  T[0] = P;
  T[1] = xyzz_dbl(P);
  T[2] = xyzz_sum(T[1], T[0]);
  T[3] = xyzz_dbl(T[1]);
  T[4] = xyzz_sum(T[3], T[0]);
  T[5] = xyzz_dbl(T[2]);
  T[6] = xyzz_sum(T[5], T[0]);
  T[7] = xyzz_dbl(T[3]);
  Xyzz<F> acc = xyzz_inf<F>();
  bool started = false;
  for (int w = 34; w >= 0; w--) {
    if (started) {
      acc = xyzz_dbl(acc);
      acc = xyzz_dbl(acc);
      acc = xyzz_dbl(acc);
      acc = xyzz_dbl(acc);
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const uint32_t* dg = h ? d2 : d1;
      const int d = (int)((dg[w >> 3] >> (4 * (w & 7))) & 15u) - 7;
      if (d != 0) {
        Xyzz<F> q = T[(d < 0 ? -d : d) - 1];
        if (h) q.X = fe_mul(q.X, beta);
        if ((d < 0) != ((h ? s2 : s1) != 0)) q.Y = fe_neg(q.Y);
        if (started) acc = xyzz_sum(acc, q);
        else { acc = q; started = true; }
      }
    }
  }
  return acc;
}

__device__ __forceinline__ void load_glv(const uint32_t* __restrict__ p, uint32_t (&g)[12]) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const uint4 x = __ldg(q + i);
    g[4 * i] = x.x; g[4 * i + 1] = x.y; g[4 * i + 2] = x.z; g[4 * i + 3] = x.w;
  }
}

__device__ __forceinline__ uint32_t bitrev_m(uint32_t i, int m) { return m == 0 ? 0u : (__brev(i) >> (32 - m)); }

// ------------------------------------------------------------------------ group FFT kernels
// Input point i (projective x = X/Z, y = Y/Z, or Jacobian x = X/Z^2, y = Y/Z^3; Z = 0 is the
// identity) to XYZZ at position bitrev(i) or i.
// (FP64 curve types: the coordinates are first brought into radix R' with kin = R'^2 / R.)
template <class C>
__global__ void k_g1fft_load(int m, int jac, int bitrev, const uint32_t* __restrict__ src, const Fe<typename C::Fp> kin,
                             uint32_t* __restrict__ a) {
  using F = typename C::Fp;
  const uint32_t n = 1u << m;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* p = src + (size_t)i * 3 * F::N;
  Fe<F> X = fe_load<F>(p), Y = fe_load<F>(p + F::N), Z = fe_load<F>(p + 2 * F::N);
  if constexpr (F::DPF) {
    X = fe_mul(X, kin);
    Y = fe_mul(Y, kin);
    Z = fe_mul(Z, kin);
  }
  Xyzz<F> r;
  if (fe_is_zero(Z)) {
    r = xyzz_inf<F>();
  } else {
    const Fe<F> zz = fe_sqr(Z);
    r.ZZ = zz;
    r.ZZZ = fe_mul(zz, Z);
    if (jac) { r.X = X; r.Y = Y; }
    else { r.X = fe_mul(X, Z); r.Y = fe_mul(Y, zz); }
  }
  const uint32_t pos = bitrev ? bitrev_m(i, m) : i;
  xyzz_store<F>(a + (size_t)pos * 4 * F::N, r);
}

// One radix-2 stage over all N/2 butterflies. Forward (DIT): (u + [w]v, u - [w]v) with
// w = tw[j << (m - s)]. Inverse (DIF): (u + v, [w](u - v)) with w = tw[j << (m - s)]; at s = m
// with a scale table, (u + v) takes [scale] and (u - v) takes [top[j]]. Twiddles are GLV records
// (GLV_WORDS words each, see xyzz_mul_glv).
static constexpr int GLV_WORDS = 12;
template <class C, bool INV>
__global__ void k_g1fft_stage(int m, int s, const uint32_t* __restrict__ tw, const uint32_t* __restrict__ top,
                              const Fe<typename C::Fp> beta, uint32_t* __restrict__ a) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const uint32_t nbf = 1u << (m - 1);
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbf) return;
  const uint32_t h = 1u << (s - 1);
  const uint32_t j = t & (h - 1);
  const uint32_t i0 = ((t >> (s - 1)) << s) + j, i1 = i0 + h;
  const Xyzz<F> u = xyzz_load<F>(a + (size_t)i0 * XW);
  Xyzz<F> v = xyzz_load<F>(a + (size_t)i1 * XW);
  uint32_t k[GLV_WORDS];
  Xyzz<F> o0, o1;
  if (!INV) {
    if (j != 0) {
      load_glv(tw + (size_t)GLV_WORDS * (j << (m - s)), k);
      v = xyzz_mul_glv(k, v, beta);
    }
    o0 = xyzz_sum(u, v);
    o1 = xyzz_sum(u, xyzz_negate(v));
  } else {
    o0 = xyzz_sum(u, v);
    o1 = xyzz_sum(u, xyzz_negate(v));
    if (top != nullptr) {
      load_glv(top, k);                     // top[0] = 2^-m
      o0 = xyzz_mul_glv(k, o0, beta);
      load_glv(top + (size_t)GLV_WORDS * j, k);
      o1 = xyzz_mul_glv(k, o1, beta);
    } else if (j != 0) {
      load_glv(tw + (size_t)GLV_WORDS * (j << (m - s)), k);
      o1 = xyzz_mul_glv(k, o1, beta);
    }
  }
  xyzz_store<F>(a + (size_t)i0 * XW, o0);
  xyzz_store<F>(a + (size_t)i1 * XW, o1);
}

// out[i] = normalised a[bitrev(i)] (or a[i])
template <class C>
__global__ void k_g1fft_store(int m, int bitrev, const uint32_t* __restrict__ a, const Fe<typename C::Fp> kout,
                              uint32_t* __restrict__ out) {
  using F = typename C::Fp;
  const uint32_t n = 1u << m;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t pos = bitrev ? bitrev_m(i, m) : i;
  xyzz_write_out<F, F::DPF>(xyzz_load<F>(a + (size_t)pos * 4 * F::N), ZKG_OUT_PROJ, out + (size_t)i * 3 * F::N, kout);
}

// ------------------------------------------------------------------------ binary MSM kernels
// Direct: thread (row, g) madds bases of the chunk's columns g, g + G, ... whose coefficient
// byte is non-zero. Affine (0, 0) bases are the identity and are skipped.
template <class C>
__global__ void k_bin_direct(int nrows, int cw, const uint8_t* __restrict__ coeffs, size_t ld,
                             const uint32_t* __restrict__ bases, int G, uint32_t* __restrict__ partial, int first) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)nrows * G) return;
  const int row = (int)(tid / G), g = (int)(tid % G);
  Xyzz<F> acc = first ? xyzz_inf<F>() : xyzz_load<F>(partial + tid * XW);
  const uint8_t* r = coeffs + (size_t)row * ld;
  for (int col = g; col < cw; col += G) {
    if (!r[col]) continue;
    const Affine<F> b = affine_load<F>(bases + (size_t)col * 2 * F::N);
    if (fe_is_zero(b.x) && fe_is_zero(b.y)) continue;
    xyzz_madd(acc, b);
  }
  xyzz_store<F>(partial + tid * XW, acc);
}

// Subset-sum tables, level l: T[k][2^l + i] = T[k][i] + P[kc + l] for i < 2^l (level 0 writes
// T[k][0] = identity and T[k][1] = P[kc]). Columns past the chunk width are the identity.
template <class C>
__global__ void k_bin_table(int nwin, int c, int l, int cw, const uint32_t* __restrict__ bases,
                            uint32_t* __restrict__ table) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t per = (size_t)1 << l;
  if (tid >= (size_t)nwin * per) return;
  const size_t k = tid >> l, i = tid & (per - 1);
  uint32_t* T = table + (k << c) * XW;
  const int col = (int)k * c + l;
  bool has = col < cw;
  Affine<F> b;
  if (has) {
    b = affine_load<F>(bases + (size_t)col * 2 * F::N);
    has = !(fe_is_zero(b.x) && fe_is_zero(b.y));
  }
  if (l == 0) {
    xyzz_store<F>(T, xyzz_inf<F>());
    xyzz_store<F>(T + XW, has ? xyzz_from_affine(b) : xyzz_inf<F>());
    return;
  }
  Xyzz<F> e = xyzz_load<F>(T + i * XW);
  if (has) xyzz_madd(e, b);
  xyzz_store<F>(T + (per + i) * XW, e);
}

// Windowed: thread (row, g) adds T[k][idx(row, k)] for windows k = g, g + G, ...
template <class C>
__global__ void k_bin_rows(int nrows, int nwin, int c, int cw, const uint8_t* __restrict__ coeffs, size_t ld,
                           const uint32_t* __restrict__ table, int G, uint32_t* __restrict__ partial, int first) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (size_t)nrows * G) return;
  const int row = (int)(tid / G), g = (int)(tid % G);
  Xyzz<F> acc = first ? xyzz_inf<F>() : xyzz_load<F>(partial + tid * XW);
  const uint8_t* r = coeffs + (size_t)row * ld;
  for (int k = g; k < nwin; k += G) {
    uint32_t idx = 0;
    const int c0 = k * c;
    for (int j = 0; j < c; j++) {
      const int col = c0 + j;
      if (col < cw && r[col]) idx |= 1u << j;
    }
    if (idx) acc = xyzz_sum(acc, xyzz_load<F>(table + (((size_t)k << c) + idx) * XW));
  }
  xyzz_store<F>(partial + tid * XW, acc);
}

// Sums of segments: block (seg b of row r) reduces in[r][b*256 .. min(L, b*256+256)) into
// out[r][b]; 128 threads, shared-memory tree.
template <class C>
__global__ void __launch_bounds__(128) k_xyzz_reduce(int L, int B, const uint32_t* __restrict__ in,
                                                     uint32_t* __restrict__ out) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  __shared__ __align__(16) uint32_t sh[128 * XW];
  const int r = blockIdx.y, b = blockIdx.x, t = threadIdx.x;
  const int lo = b * 256;
  Xyzz<F> acc = xyzz_inf<F>();
  for (int e = lo + t; e < L && e < lo + 256; e += 128) acc = xyzz_sum(acc, xyzz_load<F>(in + ((size_t)r * L + e) * XW));
  xyzz_store<F>(sh + t * XW, acc);
  __syncthreads();
  for (int w = 64; w >= 1; w >>= 1) {
    if (t < w) {
      Xyzz<F> x = xyzz_load<F>(sh + t * XW);
      x = xyzz_sum(x, xyzz_load<F>(sh + (t + w) * XW));
      xyzz_store<F>(sh + t * XW, x);
    }
    __syncthreads();
  }
  if (t == 0) xyzz_store<F>(out + ((size_t)r * B + b) * XW, xyzz_load<F>(sh));
}

template <class C>
__global__ void k_xyzz_write(int n, int kind, const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
  using F = typename C::Fp;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ow = (kind == ZKG_OUT_AFFINE ? 2 : 3) * F::N;
  xyzz_write_dev<F>(xyzz_load<F>(in + (size_t)i * 4 * F::N), kind, out + (size_t)i * ow);
}

// ------------------------------------------------------------------------ group FFT host side
template <class F>
static Fe<F> fe_zero_host() {
  Fe<F> r;
  for (int i = 0; i < F::N; i++) r.v[i] = 0;
  return r;
}
static inline size_t rup256(size_t x) { return (x + 255) & ~size_t(255); }

// GLV decomposition for phi(x, y) = (beta x, y) = [lambda](x, y) on G1. Lattice basis
// v1 = (a1, b1), v2 = (a2, b2) with a + b lambda = 0 mod r (extended Euclid on (r, lambda),
// det = r), b1 < 0 stored as mb1 = -b1. For k < r: c1 = floor(k G1 / 2^384), c2 = floor(k G2 / 2^384)
// with G1 = round(2^384 b2 / r), G2 = round(2^384 (-b1) / r) approximate the rounded lattice
// coordinates; k1 = k - c1 a1 - c2 a2, k2 = c1 mb1 - c2 b2 satisfy k1 + k2 lambda = k (mod r)
// for any c1, c2, and with these c1, c2 |k1|, |k2| < 2^130. beta is the cube root of unity in
// Fp paired with lambda (checked against the generator when the constants were derived).
struct GlvConst {
  uint64_t a1[2], mb1[2], a2[2], b2[2], G1[5], G2[5];
  uint64_t beta_std[6];
};
static const GlvConst GLV_BN254 = {
    {0x8211bbeb7d4f1128ULL, 0x6f4d8248eeb859fcULL}, {0x89d3256894d213e3ULL, 0},
    {0x89d3256894d213e3ULL, 0}, {0x0be4e1541221250bULL, 0x6f4d8248eeb859fdULL},
    {0x163b4843cb4b9a5fULL, 0x149d540fd5e495ccULL, 0x5398fd0300ff6565ULL, 0x4ccef014a773d2d2ULL, 0x2ULL},
    {0x8fa7d32d2fafba64ULL, 0x6eb9c714773a6ef2ULL, 0xd91d232ec7e0b3d7ULL, 0x2ULL, 0},
    {0xe4bd44e5607cfd48ULL, 0xc28f069fbb966e3dULL, 0x5e6dd9e7e0acccb0ULL, 0x30644e72e131a029ULL, 0, 0}};
static const GlvConst GLV_BLS12_381 = {
    {0x1ULL, 0}, {0x00000000ffffffffULL, 0xac45a4010001a402ULL},
    {0x0000000100000000ULL, 0xac45a4010001a402ULL}, {0x1ULL, 0},
    {0x38b5dcb707e08ed3ULL, 0x355094edfede377cULL, 0x2ULL, 0, 0},
    {0xa1a872d6818be407ULL, 0x034eb4b927adc027ULL, 0x63f6e522f6cfee2eULL, 0x7c6becf1e01faaddULL, 0x1ULL},
    {0x2e01fffffffefffeULL, 0xde17d813620a0002ULL, 0xddb3a93be6f89688ULL, 0xba69c6076a0f77eaULL,
     0x5f19672fdf76ce51ULL, 0}};

// floor(k * G / 2^384) for k < 2^256 (4 limbs), G 5 limbs; the result has at most 2 limbs here
static void glv_coord(const uint64_t k[4], const uint64_t G[5], uint64_t c[2]) {
  uint64_t prod[9] = {0};
  for (int i = 0; i < 4; i++) {
    unsigned __int128 carry = 0;
    for (int j = 0; j < 5; j++) {
      const unsigned __int128 t = (unsigned __int128)k[i] * G[j] + prod[i + j] + carry;
      prod[i + j] = (uint64_t)t;
      carry = t >> 64;
    }
    prod[i + 5] = (uint64_t)carry;
  }
  c[0] = prod[6];
  c[1] = prod[7];
}
// (x * y) mod 2^192 for 2-limb x, y
static void mul_mod192(const uint64_t x[2], const uint64_t y[2], uint64_t r[3]) {
  const unsigned __int128 p00 = (unsigned __int128)x[0] * y[0];
  const unsigned __int128 p01 = (unsigned __int128)x[0] * y[1];
  const unsigned __int128 p10 = (unsigned __int128)x[1] * y[0];
  const unsigned __int128 p11 = (unsigned __int128)x[1] * y[1];
  r[0] = (uint64_t)p00;
  const unsigned __int128 mid = (p00 >> 64) + (uint64_t)p01 + (uint64_t)p10;
  r[1] = (uint64_t)mid;
  r[2] = (uint64_t)(mid >> 64) + (uint64_t)(p01 >> 64) + (uint64_t)(p10 >> 64) + (uint64_t)p11;
}
static void sub192(uint64_t a[3], const uint64_t b[3]) {
  unsigned __int128 borrow = 0;
  for (int i = 0; i < 3; i++) {
    const unsigned __int128 t = (unsigned __int128)a[i] - b[i] - borrow;
    a[i] = (uint64_t)t;
    borrow = (t >> 64) ? 1 : 0;
  }
}
// signed 192-bit value -> sign and magnitude; false if the magnitude needs more than 136 bits
static bool sign_mag(uint64_t v[3], uint32_t& neg) {
  neg = (uint32_t)(v[2] >> 63);
  if (neg) {
    uint64_t z[3] = {0, 0, 0};
    sub192(z, v);
    v[0] = z[0]; v[1] = z[1]; v[2] = z[2];
  }
  return v[2] < (1ULL << 8);
}
// k (standard integer < r, 4 limbs) -> GLV record (GLV_WORDS 32-bit words, see xyzz_mul_glv)
static bool glv_split(const GlvConst& G, const uint64_t k[4], uint32_t out[12]) {
  uint64_t c1[2], c2[2], t[3];
  glv_coord(k, G.G1, c1);
  glv_coord(k, G.G2, c2);
  uint64_t k1[3] = {k[0], k[1], k[2]};
  mul_mod192(c1, G.a1, t);
  sub192(k1, t);
  mul_mod192(c2, G.a2, t);
  sub192(k1, t);
  uint64_t k2[3];
  mul_mod192(c1, G.mb1, k2);
  mul_mod192(c2, G.b2, t);
  sub192(k2, t);
  uint32_t n1 = 0, n2 = 0;
  if (!sign_mag(k1, n1) || !sign_mag(k2, n2)) return false;
  for (int i = 0; i < 5; i++) {
    out[i] = (uint32_t)(k1[i >> 1] >> (32 * (i & 1)));
    out[5 + i] = (uint32_t)(k2[i >> 1] >> (32 * (i & 1)));
  }
  out[10] = n1 | (n2 << 1);
  out[11] = 0;
  return true;
}

// CP: the curve type the point arithmetic runs on (C, or its FP64-product twin, zkb_dpf.cuh)
template <class CP, class C, int NL>
static zkg_status g1_fft_run(Context& cx, int jac, int m, const uint64_t* gen, const uint32_t* d_src,
                             uint32_t* d_out, int inverse, cudaStream_t st) {
  const host::Field<4>& Fr = (C::ID == 0) ? host::BN_FR : host::BLS_FR;
  const size_t n = (size_t)1 << m, half = n >> 1;
  const size_t xb = 4 * NL * 8;
  // twiddles (standard form): tw[e] = g^e for e < N/2, g = gen (forward) or gen^-1 (inverse);
  // top[j] = 2^-m gen^-j (inverse only)
  using host::El;
  El<4> g, one_std = host::zero<4>();
  one_std.v[0] = 1;
  std::memcpy(g.v, gen, 32);
  if (inverse) g = host::inv(Fr, g);
  El<4> two_std = host::zero<4>();
  two_std.v[0] = 2;
  El<4> sc = host::one(Fr);
  if (inverse) {
    const El<4> ihalf = host::inv(Fr, host::from_std(Fr, two_std));
    for (int i = 0; i < m; i++) sc = host::mul(Fr, sc, ihalf);
  }
  const size_t ntw = std::max<size_t>(half, 1);
  const GlvConst& GC = (C::ID == 0) ? GLV_BN254 : GLV_BLS12_381;
  std::vector<uint32_t> tw((size_t)GLV_WORDS * ntw * (inverse ? 2 : 1), 0);
  El<4> pw = host::one(Fr);
  for (size_t e = 0; e < half; e++) {
    const El<4> s0 = host::mul(Fr, pw, one_std);
    if (!glv_split(GC, s0.v, &tw[(size_t)GLV_WORDS * e])) return set_status(ZKG_ERR_ARG, "g1_fft", "GLV split");
    if (inverse) {
      const El<4> s1 = host::mul(Fr, host::mul(Fr, pw, sc), one_std);
      if (!glv_split(GC, s1.v, &tw[(size_t)GLV_WORDS * (ntw + e)])) return set_status(ZKG_ERR_ARG, "g1_fft", "GLV split");
    }
    pw = host::mul(Fr, pw, g);
  }
  // beta in the Montgomery radix of the point arithmetic (R, or R' for the FP64 types:
  // beta R' = mont(beta R, R' mod p))
  using F = typename CP::Fp;
  Fe<F> beta, kin = fe_zero_host<F>(), kout = fe_zero_host<F>();
  {
    const host::Field<NL>* fp;
    if constexpr (NL == 4) fp = &host::BN_FP;
    else fp = &host::BLS_FP;
    const host::Field<NL>& Fp = *fp;
    El<NL> b;
    std::memcpy(b.v, GC.beta_std, 8 * NL);
    El<NL> bm = host::from_std(Fp, b);
    if constexpr (F::DPF) {
      El<NL> rp = host::zero<NL>();
      for (int w = 0; w < F::N; w++) rp.v[w >> 1] |= (uint64_t)F::one(w) << (32 * (w & 1));
      bm = host::mul(Fp, bm, rp);
      dpf_consts_for<CP>(kin, kout);
    }
    for (int w = 0; w < F::N; w++) beta.v[w] = (uint32_t)(bm.v[w >> 1] >> (32 * (w & 1)));
  }
  const size_t bytes = rup256(n * xb) + rup256(tw.size() * 4);
  ZKB_TRY(cx.arena.reserve(bytes));
  cx.arena.reset();
  uint32_t* a = static_cast<uint32_t*>(cx.arena.take(n * xb));
  uint32_t* d_tw = static_cast<uint32_t*>(cx.arena.take(tw.size() * 4));
  if (!a || !d_tw) return set_status(ZKG_ERR_NOMEM, "g1_fft", "arena");
  ZKB_CUDA(cudaMemcpyAsync(d_tw, tw.data(), tw.size() * 4, cudaMemcpyHostToDevice, st));
  const dim3 blk(128);
  const dim3 grid_n((unsigned)((n + 127) / 128));
  ZKB_TRY(launch("g1fft_load", k_g1fft_load<CP>, grid_n, blk, 0, st, m, jac, inverse ? 0 : 1, d_src, kin, a));
  const dim3 grid_h((unsigned)((half + 127) / 128));
  if (!inverse) {
    for (int s = 1; s <= m; s++)
      ZKB_TRY(launch("g1fft_stage", k_g1fft_stage<CP, false>, grid_h, blk, 0, st, m, s, (const uint32_t*)d_tw,
                     (const uint32_t*)nullptr, beta, a));
  } else {
    for (int s = m; s >= 1; s--)
      ZKB_TRY(launch("g1fft_stage", k_g1fft_stage<CP, true>, grid_h, blk, 0, st, m, s, (const uint32_t*)d_tw,
                     s == m ? (const uint32_t*)(d_tw + (size_t)GLV_WORDS * ntw) : (const uint32_t*)nullptr, beta, a));
  }
  ZKB_TRY(launch("g1fft_store", k_g1fft_store<CP>, grid_n, blk, 0, st, m, inverse ? 1 : 0, (const uint32_t*)a, kout,
                 d_out));
  return ZKG_OK;
}

// BN254 point arithmetic with FP64-pipe products unless ZKB_G1_DPF=0 (BLS12-381 stays on the
// integer pipes: its 8-limb FP64 product made these kernels slower, 55.0 vs 43.3 ms at 2^14)
static const bool g_g1_dpf = [] {
  const char* v = std::getenv("ZKB_G1_DPF");
  return v ? std::atoi(v) != 0 : true;
}();

template <class C, int NL>
static zkg_status g1_fft_launch(Context& cx, int jac, int m, const uint64_t* gen, const uint32_t* d_src,
                                uint32_t* d_out, int inverse, cudaStream_t st) {
  if constexpr (C::ID == 0) {
    if (g_g1_dpf) return g1_fft_run<typename DpfCurve<C>::type, C, NL>(cx, jac, m, gen, d_src, d_out, inverse, st);
  }
  return g1_fft_run<C, C, NL>(cx, jac, m, gen, d_src, d_out, inverse, st);
}

static zkg_status g1_fft_check(zkg_curve curve, int m, const void* gen, const void* src, const void* tgt) {
  if (curve != ZKG_BN254 && curve != ZKG_BLS12_381) return set_status(ZKG_ERR_ARG, "g1_fft", "unknown curve");
  if (m < 0 || m > 26) return set_status(ZKG_ERR_ARG, "g1_fft", "m out of range [0, 26]");
  if (!gen || !src || !tgt) return set_status(ZKG_ERR_ARG, "g1_fft", "null pointer");
  return ZKG_OK;
}

template <class C, int NL>
static zkg_status g1_fft_host(int jac, int m, const uint64_t* gen, const uint64_t* src, uint64_t* tgt, int inverse) {
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  const size_t n = (size_t)1 << m, pb = 3 * NL * 8;
  uint32_t* d_io = nullptr;
  ZKB_CUDA(cudaMalloc(&d_io, n * pb));
  const cudaStream_t st = cx.compute();
  zkg_status rc = ZKG_OK;
  rc = copy_h2d(cx, d_io, src, n * pb, st);
  if (rc == ZKG_OK) rc = g1_fft_launch<C, NL>(cx, jac, m, gen, d_io, d_io, inverse, st);
  if (rc == ZKG_OK) rc = copy_d2h(cx, tgt, d_io, n * pb, st);
  if (rc == ZKG_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = set_status(ZKG_ERR_CUDA, "g1_fft", "sync");
  cudaFree(d_io);
  return rc == ZKG_OK ? set_status(ZKG_OK, nullptr, nullptr) : rc;
}

template <class C, int NL>
static zkg_status g1_fft_dev(int jac, int m, const uint64_t* gen, const uint64_t* d_src, uint64_t* d_tgt, int inverse) {
  if ((reinterpret_cast<uintptr_t>(d_src) | reinterpret_cast<uintptr_t>(d_tgt)) & 15)
    return set_status(ZKG_ERR_ARG, "g1_fft_device", "device buffers must be 16-byte aligned");
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  if (!cx.user_stream) ZKB_CUDA(cudaDeviceSynchronize());
  const cudaStream_t st = cx.compute();
  ZKB_TRY((g1_fft_launch<C, NL>(cx, jac, m, gen, reinterpret_cast<const uint32_t*>(d_src),
                                reinterpret_cast<uint32_t*>(d_tgt), inverse, st)));
  ZKB_CUDA(cudaStreamSynchronize(st));
  return set_status(ZKG_OK, nullptr, nullptr);
}

// ------------------------------------------------------------------------ binary MSM host side
struct BinPlan {
  int windowed = 0;   // 0: direct madds; 1: subset-sum tables of c columns
  int c = 1;
  int G = 1;          // partial sums per row
  int cw = 0;         // columns per chunk (a multiple of c)
};

// Cost per column in field products: direct = rows * (1/2) * 10 (one madd per selected base at
// density 1/2); windowed = ((2^c - 1 - c) * 10 + rows * (1 - 2^-c) * 14) / c (table madds plus
// one full addition per row and window).
static BinPlan bin_plan(int nrows, int npoints, int nl, int sm_count) {
  BinPlan P;
  double best = 5.0 * nrows;
  for (int c = 2; c <= 12; c++) {
    const double cost = ((double)((1 << c) - 1 - c) * 10.0 + nrows * (1.0 - std::ldexp(1.0, -c)) * 14.0) / c;
    if (cost < best * 0.95) { best = cost; P.windowed = 1; P.c = c; }
  }
  const size_t xb = 4 * (size_t)nl * 8;
  // chunk: coefficients <= 32 MiB, bases <= 32 MiB, tables <= 256 MiB
  size_t cw = std::min<size_t>((size_t)npoints, ((size_t)32 << 20) / std::max(1, nrows));
  cw = std::min<size_t>(cw, ((size_t)32 << 20) / (2 * (size_t)nl * 8));
  if (P.windowed) cw = std::min<size_t>(cw, (((size_t)256 << 20) / (xb << P.c)) * P.c);
  cw = std::max<size_t>(cw, (size_t)P.c);
  cw = (cw + P.c - 1) / P.c * P.c;
  P.cw = (int)cw;
  const long units = P.windowed ? (long)(cw / P.c) : (long)cw;   // per-row work items in a chunk
  const long target = (long)sm_count * 512;                      // threads to keep the SMs busy
  long G = (target + nrows - 1) / nrows;
  G = std::max(1L, std::min(G, units));
  G = std::min(G, 65536L);
  P.G = (int)G;
  return P;
}

// Runs the chunk loop. get_chunk(q, col0, cw, &coeffs, &ld, &bases) makes chunk q's coefficient
// rows (ld bytes apart) and bases available to the compute stream.
template <class C, int NL, class Get>
static zkg_status bin_run(Context& cx, const BinPlan& P, int nrows, int npoints, char* ws, cudaStream_t st,
                          Get get_chunk, int kind, uint32_t* d_out) {
  using F = typename C::Fp;
  const size_t xb = 4 * NL * 8;
  uint32_t* partial = reinterpret_cast<uint32_t*>(ws);
  ws += rup256((size_t)nrows * P.G * xb);
  uint32_t* table = reinterpret_cast<uint32_t*>(ws);
  const dim3 blk(128);
  const size_t nthr = (size_t)nrows * P.G;
  const int nchunks = (npoints + P.cw - 1) / P.cw;
  for (int q = 0; q < nchunks; q++) {
    const int col0 = q * P.cw;
    const int cw = std::min(P.cw, npoints - col0);
    const uint8_t* coeffs = nullptr;
    size_t ld = 0;
    const uint32_t* bases = nullptr;
    ZKB_TRY(get_chunk(q, col0, cw, &coeffs, &ld, &bases));
    if (!P.windowed) {
      ZKB_TRY(launch("bin_direct", k_bin_direct<C>, dim3((unsigned)((nthr + 127) / 128)), blk, 0, st, nrows, cw,
                     coeffs, ld, bases, P.G, partial, q == 0 ? 1 : 0));
    } else {
      const int nwin = (cw + P.c - 1) / P.c;
      for (int l = 0; l < P.c; l++) {
        const size_t nt = (size_t)nwin << l;
        ZKB_TRY(launch("bin_table", k_bin_table<C>, dim3((unsigned)((nt + 127) / 128)), blk, 0, st, nwin, P.c, l, cw,
                       bases, table));
      }
      ZKB_TRY(launch("bin_rows", k_bin_rows<C>, dim3((unsigned)((nthr + 127) / 128)), blk, 0, st, nrows, nwin, P.c,
                     cw, coeffs, ld, (const uint32_t*)table, P.G, partial, q == 0 ? 1 : 0));
    }
    ZKB_TRY(get_chunk(-1 - q, 0, 0, nullptr, nullptr, nullptr));   // chunk q's inputs are consumed
  }
  // reduce G partials per row: 256 per block per pass
  int L = P.G;
  uint32_t* in = partial;
  uint32_t* tmp = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(table));   // reuse the table region
  while (L > 1) {
    const int B = (L + 255) / 256;
    ZKB_TRY(launch("xyzz_reduce", k_xyzz_reduce<C>, dim3((unsigned)B, (unsigned)nrows), blk, 0, st, L, B,
                   (const uint32_t*)in, tmp));
    std::swap(in, tmp);
    L = B;
  }
  ZKB_TRY(launch("xyzz_write", k_xyzz_write<C>, dim3((unsigned)((nrows + 127) / 128)), blk, 0, st, nrows, kind,
                 (const uint32_t*)in, d_out));
  (void)sizeof(F);
  return ZKG_OK;
}

template <int NL>
static size_t bin_ws_bytes(const BinPlan& P, int nrows) {
  const size_t xb = 4 * NL * 8;
  const size_t part = rup256((size_t)nrows * P.G * xb);
  const size_t nwin = (size_t)(P.cw + P.c - 1) / P.c;
  size_t tab = P.windowed ? rup256((nwin << P.c) * xb) : 0;
  tab = std::max(tab, part);   // the reduction's ping-pong buffer reuses the table region
  return part + tab;
}

static zkg_status bin_check(zkg_curve curve, int kind, int nrows, int npoints, const void* rows, const void* bases,
                            const void* out) {
  if (curve != ZKG_BN254 && curve != ZKG_BLS12_381) return set_status(ZKG_ERR_ARG, "msm_binary", "unknown curve");
  if (kind < ZKG_OUT_PROJ || kind > ZKG_OUT_AFFINE) return set_status(ZKG_ERR_ARG, "msm_binary", "bad output kind");
  if (nrows < 0 || npoints < 0) return set_status(ZKG_ERR_ARG, "msm_binary", "negative size");
  if (nrows > 0 && (!out || (npoints > 0 && (!rows || !bases))))
    return set_status(ZKG_ERR_ARG, "msm_binary", "null pointer");
  return ZKG_OK;
}

template <class C, int NL>
static zkg_status bin_host(const host::Field<NL>& Fp, int kind, int nrows, int npoints, const uint8_t* const* rows,
                           const uint64_t* grps, uint64_t* tgt) {
  const int ow = (kind == ZKG_OUT_AFFINE ? 2 : 3) * NL;
  if (nrows == 0) return set_status(ZKG_OK, nullptr, nullptr);
  if (npoints == 0) {
    for (int r = 0; r < nrows; r++) host::xyzz_write<NL>(Fp, host::xyzz_inf<NL>(), kind, tgt + (size_t)r * ow);
    return set_status(ZKG_OK, nullptr, nullptr);
  }
  for (int r = 0; r < nrows; r++)
    if (!rows[r]) return set_status(ZKG_ERR_ARG, "msm_binary", "null coefficient row");
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  const BinPlan P = bin_plan(nrows, npoints, NL, cx.sm_count);
  const size_t bb = 2 * NL * 8;
  const size_t coef_chunk = rup256((size_t)nrows * P.cw), base_chunk = rup256((size_t)P.cw * bb);
  const size_t out_bytes = rup256((size_t)nrows * ow * 8);
  const size_t stage = coef_chunk + base_chunk;   // one pinned / device staging slot
  const size_t bytes = 2 * stage + out_bytes + bin_ws_bytes<NL>(P, nrows);
  ZKB_TRY(cx.arena.reserve(bytes));
  cx.arena.reset();
  char* dstage = static_cast<char*>(cx.arena.take(2 * stage));
  uint32_t* d_out = static_cast<uint32_t*>(cx.arena.take(out_bytes));
  char* ws = static_cast<char*>(cx.arena.take(bytes - 2 * stage - out_bytes));
  if (!dstage || !d_out || !ws) return set_status(ZKG_ERR_NOMEM, "msm_binary", "arena");
  ZKB_TRY(pinned_reserve(cx, std::max(2 * stage, out_bytes)));
  char* pin = static_cast<char*>(cx.pinned);
  const cudaStream_t st = cx.compute();
  cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_used[2] = {nullptr, nullptr};
  for (int b = 0; b < 2; b++) {
    ZKB_CUDA(cudaEventCreateWithFlags(&ev_copied[b], cudaEventDisableTiming));
    ZKB_CUDA(cudaEventCreateWithFlags(&ev_used[b], cudaEventDisableTiming));
  }
  // earlier work on the compute stream may still use the arena
  ZKB_CUDA(cudaEventRecord(ev_used[0], st));
  ZKB_CUDA(cudaEventRecord(ev_used[1], st));
  bool pending[2] = {false, false};
  auto get_chunk = [&](int q, int col0, int cw, const uint8_t** coeffs, size_t* ld,
                       const uint32_t** bases) -> zkg_status {
    if (q < 0) {   // chunk -1 - q consumed by the kernels just queued
      const int b = (-1 - q) & 1;
      ZKB_CUDA(cudaEventRecord(ev_used[b], st));
      return ZKG_OK;
    }
    const int b = q & 1;
    char* hp = pin + b * stage;
    char* dp = dstage + b * stage;
    if (pending[b]) ZKB_CUDA(cudaEventSynchronize(ev_copied[b]));   // pinned slot b is free again
    for (int r = 0; r < nrows; r++) std::memcpy(hp + (size_t)r * P.cw, rows[r] + col0, (size_t)cw);
    std::memcpy(hp + coef_chunk, grps + (size_t)col0 * 2 * NL, (size_t)cw * bb);
    ZKB_CUDA(cudaStreamWaitEvent(cx.copy_stream, ev_used[b], 0));
    ZKB_CUDA(cudaMemcpyAsync(dp, hp, coef_chunk + (size_t)cw * bb, cudaMemcpyHostToDevice, cx.copy_stream));
    ZKB_CUDA(cudaEventRecord(ev_copied[b], cx.copy_stream));
    pending[b] = true;
    ZKB_CUDA(cudaStreamWaitEvent(st, ev_copied[b], 0));
    *coeffs = reinterpret_cast<const uint8_t*>(dp);
    *ld = (size_t)P.cw;
    *bases = reinterpret_cast<const uint32_t*>(dp + coef_chunk);
    return ZKG_OK;
  };
  zkg_status rc = bin_run<C, NL>(cx, P, nrows, npoints, ws, st, get_chunk, kind, d_out);
  if (rc == ZKG_OK) {
    // the pinned slots may still feed a copy; wait for all of them before reusing pinned memory
    if (cudaStreamSynchronize(cx.copy_stream) != cudaSuccess) rc = set_status(ZKG_ERR_CUDA, "msm_binary", "copy sync");
  }
  if (rc == ZKG_OK && cudaMemcpyAsync(pin, d_out, (size_t)nrows * ow * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    rc = set_status(ZKG_ERR_CUDA, "msm_binary", "output copy");
  if (rc == ZKG_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = set_status(ZKG_ERR_CUDA, "msm_binary", "sync");
  if (rc == ZKG_OK) std::memcpy(tgt, pin, (size_t)nrows * ow * 8);
  if (rc != ZKG_OK) {
    cudaStreamSynchronize(cx.copy_stream);
    cudaStreamSynchronize(st);
  }
  for (int b = 0; b < 2; b++) {
    cudaEventDestroy(ev_copied[b]);
    cudaEventDestroy(ev_used[b]);
  }
  return rc == ZKG_OK ? set_status(ZKG_OK, nullptr, nullptr) : rc;
}

template <class C, int NL>
static zkg_status bin_dev(int kind, int nrows, int npoints, const uint8_t* d_coeffs, size_t ld, const uint64_t* d_bases,
                          uint64_t* d_out) {
  if (nrows == 0) return set_status(ZKG_OK, nullptr, nullptr);
  if (npoints > 0 && ld < (size_t)npoints) return set_status(ZKG_ERR_ARG, "msm_binary_device", "ld < npoints");
  if ((reinterpret_cast<uintptr_t>(d_bases) | reinterpret_cast<uintptr_t>(d_out)) & 15)
    return set_status(ZKG_ERR_ARG, "msm_binary_device", "device buffers must be 16-byte aligned");
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  if (!cx.user_stream) ZKB_CUDA(cudaDeviceSynchronize());
  const cudaStream_t st = cx.compute();
  const dim3 blk(128);
  if (npoints == 0) {
    // every row is the identity: write it through the same conversion kernel
    const size_t xb = 4 * NL * 8;
    ZKB_TRY(cx.arena.reserve((size_t)nrows * xb));
    cx.arena.reset();
    uint32_t* z = static_cast<uint32_t*>(cx.arena.take((size_t)nrows * xb));
    if (!z) return set_status(ZKG_ERR_NOMEM, "msm_binary_device", "arena");
    ZKB_CUDA(cudaMemsetAsync(z, 0, (size_t)nrows * xb, st));
    ZKB_TRY(launch("xyzz_write", k_xyzz_write<C>, dim3((unsigned)((nrows + 127) / 128)), blk, 0, st, nrows, kind,
                   (const uint32_t*)z, reinterpret_cast<uint32_t*>(d_out)));
    ZKB_CUDA(cudaStreamSynchronize(st));
    return set_status(ZKG_OK, nullptr, nullptr);
  }
  const BinPlan P = bin_plan(nrows, npoints, NL, cx.sm_count);
  const size_t bytes = bin_ws_bytes<NL>(P, nrows);
  ZKB_TRY(cx.arena.reserve(bytes));
  cx.arena.reset();
  char* ws = static_cast<char*>(cx.arena.take(bytes));
  if (!ws) return set_status(ZKG_ERR_NOMEM, "msm_binary_device", "arena");
  auto get_chunk = [&](int q, int col0, int cw, const uint8_t** coeffs, size_t* pld,
                       const uint32_t** bases) -> zkg_status {
    if (q < 0) return ZKG_OK;
    (void)cw;
    *coeffs = d_coeffs + col0;
    *pld = ld;
    *bases = reinterpret_cast<const uint32_t*>(d_bases + (size_t)col0 * 2 * NL);
    return ZKG_OK;
  };
  ZKB_TRY((bin_run<C, NL>(cx, P, nrows, npoints, ws, st, get_chunk, kind, reinterpret_cast<uint32_t*>(d_out))));
  ZKB_CUDA(cudaStreamSynchronize(st));
  return set_status(ZKG_OK, nullptr, nullptr);
}

}  // namespace zkb

using namespace zkb;

extern "C" zkg_status zkg_g1_fft(zkg_curve curve, int jac, int m, const uint64_t* gen, const uint64_t* src,
                                 uint64_t* tgt, int inverse) {
  ZKB_TRY(g1_fft_check(curve, m, gen, src, tgt));
  if (curve == ZKG_BN254) return g1_fft_host<BN254, 4>(jac ? 1 : 0, m, gen, src, tgt, inverse ? 1 : 0);
  return g1_fft_host<BLS12_381, 6>(jac ? 1 : 0, m, gen, src, tgt, inverse ? 1 : 0);
}

extern "C" zkg_status zkg_g1_fft_device(zkg_curve curve, int jac, int m, const uint64_t* gen, const uint64_t* d_src,
                                        uint64_t* d_tgt, int inverse) {
  ZKB_TRY(g1_fft_check(curve, m, gen, d_src, d_tgt));
  if (curve == ZKG_BN254) return g1_fft_dev<BN254, 4>(jac ? 1 : 0, m, gen, d_src, d_tgt, inverse ? 1 : 0);
  return g1_fft_dev<BLS12_381, 6>(jac ? 1 : 0, m, gen, d_src, d_tgt, inverse ? 1 : 0);
}

extern "C" zkg_status zkg_msm_binary(zkg_curve curve, int out_kind, int nrows, int npoints,
                                     const uint8_t* const* rows, const uint64_t* bases, uint64_t* out) {
  ZKB_TRY(bin_check(curve, out_kind, nrows, npoints, rows, bases, out));
  if (curve == ZKG_BN254) return bin_host<BN254, 4>(host::BN_FP, out_kind, nrows, npoints, rows, bases, out);
  return bin_host<BLS12_381, 6>(host::BLS_FP, out_kind, nrows, npoints, rows, bases, out);
}

extern "C" zkg_status zkg_msm_binary_device(zkg_curve curve, int out_kind, int nrows, int npoints,
                                            const uint8_t* d_coeffs, size_t ld, const uint64_t* d_bases,
                                            uint64_t* d_out) {
  ZKB_TRY(bin_check(curve, out_kind, nrows, npoints, d_coeffs, d_bases, d_out));
  if (curve == ZKG_BN254) return bin_dev<BN254, 4>(out_kind, nrows, npoints, d_coeffs, ld, d_bases, d_out);
  return bin_dev<BLS12_381, 6>(out_kind, nrows, npoints, d_coeffs, ld, d_bases, d_out);
}
