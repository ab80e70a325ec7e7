// Element-wise field operations on device buffers, for direct tests of the field arithmetic that
// every kernel is built on: the 32-bit-limb CIOS product (zkb_field.cuh) and the FP64-pipe
// product (zkb_dpf.cuh), over BN254 / BLS12-381 Fp and Fr.
//
// Reference: bn128_Fp_mont_mul (lib/cbits/curves/fields/mont/bn128_Fp_mont.c:189),
// bls12_381_Fp_mont_mul (bls12_381_Fp_mont.c:203), the Fr twins (bn128_Fr_mont.c:189,
// bls12_381_Fr_mont.c:189), and their add / sub / neg / sqr. Elements are the reference's
// Montgomery form (radix R = 2^256, or 2^384 for BLS12-381 Fp), fully reduced.
//
// On the FP64 path the operands are moved into that product's radix R' = 2^(52 L) and back with
// the same exact conversions the MSM and NTT use (x R -> mont'(x R, R'^2 / R) = x R';
// x R' -> mont'(x R', R) = x R), so the result is directly comparable with the reference's.
// Path 2 (Fp only) runs the MSM bucket pipeline's redundant-range arithmetic (values in
// [0, 2p), zkb_field.cuh) on operands given in both representatives x and x + p. Path 3 runs the
// FP64 product in the reference's own radix (EXACT fields, zkb_dpf.cuh) with no conversions.
#include "zkb_dpf.cuh"
#include "zkb_runtime.h"

namespace zkb {

enum FieldTestOp {
  FT_MUL = 0,       // a b R^-1                       (the reference's mont_mul)
  FT_SQR = 1,       // a^2 R^-1
  FT_ADD = 2,       // a + b mod p
  FT_SUB = 3,       // a - b mod p
  FT_NEG = 4,       // -a mod p
  FT_RAW_DPF = 5,   // a b R'^-1 (FP64 product without radix conversions; path ignored)
  FT_PAIR_A = 6,    // first product of a paired call  (a b, path 1: paired FP64 products)
  FT_PAIR_B = 7,    // second product of a paired call (b a)
  FT_SQR_PAIR = 8,  // first square of a paired square call (a^2)
};

// path 2: the MSM pipeline's redundant range (lazy field PL, values in [0, 2p)): operands are
// lifted to x + p for odd indices (the other representative), the operation runs on the lazy
// type, and the result is made canonical.
template <class P, class PL>
__device__ Fe<P> field_test_lazy(int op, uint32_t i, const Fe<P>& x0, const Fe<P>& y0, const Fe<PL>& kin,
                                 const Fe<PL>& kout) {
  auto lift = [&](const Fe<P>& v, bool up) {
    Fe<PL> w;
    uint32_t c = 0;
    for (int k = 0; k < P::N; k++) {
      const uint64_t t = (uint64_t)v.v[k] + (up ? P::mod(k) : 0u) + c;
      w.v[k] = (uint32_t)t;
      c = (uint32_t)(t >> 32);
    }
    return w;
  };
  const Fe<PL> x = lift(x0, i & 1), y = lift(y0, (i >> 1) & 1);
  Fe<PL> r;
  switch (op) {
    case FT_MUL: r = fe_mul(x, fe_mul(y, kin)); break;
    case FT_SQR: r = fe_mul(fe_sqr(fe_mul(x, kin)), kout); break;
    case FT_ADD: r = fe_add(x, y); break;
    case FT_SUB: r = fe_sub(x, y); break;
    case FT_NEG: r = fe_neg(x); break;
    case FT_PAIR_A:
    case FT_PAIR_B: {
      Fe<PL> u, v;
      fe_mul2(u, x, fe_mul(y, kin), v, y, fe_mul(x, kin));
      r = op == FT_PAIR_A ? u : v;
      break;
    }
    case FT_SQR_PAIR: {
      Fe<PL> u, v;
      fe_sqr2(u, fe_mul(x, kin), v, fe_mul(y, kin));
      r = fe_mul(u, kout);
      break;
    }
    default: r = fe_zero<PL>(); break;
  }
  // every result must be in [0, 2p) before it is made canonical
  bool below2p = true;
  {
    uint32_t bw = 0;
    for (int k = 0; k < P::N; k++) {
      const uint64_t t = (uint64_t)r.v[k] - red_mod<PL>(k) - bw;
      bw = (uint32_t)(t >> 63);
    }
    below2p = bw != 0;
  }
  const Fe<PL> c = fe_canon(r);
  Fe<P> o;
  for (int k = 0; k < P::N; k++) o.v[k] = below2p ? c.v[k] : 0xffffffffu;   // all-ones flags a range error
  return o;
}

// path 3: FP64 products in the reference's own radix (EXACT field PE): no conversions
template <class P, class PE>
__device__ Fe<P> field_test_exact(int op, const Fe<P>& x0, const Fe<P>& y0) {
  Fe<PE> x, y, r;
  for (int k = 0; k < P::N; k++) { x.v[k] = x0.v[k]; y.v[k] = y0.v[k]; }
  switch (op) {
    case FT_MUL: r = fe_mul(x, y); break;
    case FT_SQR: r = fe_sqr(x); break;
    case FT_ADD: r = fe_add(x, y); break;
    case FT_SUB: r = fe_sub(x, y); break;
    case FT_NEG: r = fe_neg(x); break;
    case FT_PAIR_A:
    case FT_PAIR_B: {
      Fe<PE> u, v;
      fe_mul2(u, x, y, v, y, x);
      r = op == FT_PAIR_A ? u : v;
      break;
    }
    case FT_SQR_PAIR: {
      Fe<PE> u, v;
      fe_sqr2(u, x, v, y);
      r = u;
      break;
    }
    default: r = fe_zero<PE>(); break;
  }
  Fe<P> o;
  for (int k = 0; k < P::N; k++) o.v[k] = r.v[k];
  return o;
}

template <class P, class PD, class PL, class PE>
__global__ void k_field_test(int op, int path, uint32_t n, const uint32_t* __restrict__ a,
                             const uint32_t* __restrict__ b, uint32_t* __restrict__ out, Fe<PD> kin, Fe<PD> kout) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Fe<P> x = fe_load<P>(a + (size_t)i * P::N);
  const Fe<P> y = b ? fe_load<P>(b + (size_t)i * P::N) : fe_zero<P>();
  Fe<P> r;
  if (path == 3) {
    fe_store<P>(out + (size_t)i * P::N, field_test_exact<P, PE>(op, x, y));
    return;
  }
  if constexpr (lazy_v<PL>) {
    if (path == 2) {
      Fe<PL> ki, ko;
      for (int k = 0; k < P::N; k++) { ki.v[k] = kin.v[k]; ko.v[k] = kout.v[k]; }
      fe_store<P>(out + (size_t)i * P::N, field_test_lazy<P, PL>(op, i, x, y, ki, ko));
      return;
    }
  }
  // word-level reinterpretation between the two flavours of one field (same modulus and words)
  auto toD = [](const Fe<P>& v) { Fe<PD> w; for (int k = 0; k < P::N; k++) w.v[k] = v.v[k]; return w; };
  auto fromD = [](const Fe<PD>& v) { Fe<P> w; for (int k = 0; k < P::N; k++) w.v[k] = v.v[k]; return w; };
  switch (op) {
    case FT_MUL:
      if (path == 0) r = fe_mul(x, y);
      else r = fromD(fe_mul(toD(x), fe_mul(toD(y), kin)));
      break;
    case FT_SQR:
      if (path == 0) r = fe_sqr(x);
      else r = fromD(fe_mul(fe_sqr(fe_mul(toD(x), kin)), kout));
      break;
    case FT_ADD: r = path == 0 ? fe_add(x, y) : fromD(fe_add(toD(x), toD(y))); break;
    case FT_SUB: r = path == 0 ? fe_sub(x, y) : fromD(fe_sub(toD(x), toD(y))); break;
    case FT_NEG: r = path == 0 ? fe_neg(x) : fromD(fe_neg(toD(x))); break;
    case FT_RAW_DPF: r = fromD(fe_mul(toD(x), toD(y))); break;
    case FT_PAIR_A:
    case FT_PAIR_B:
      if (path == 0) {
        Fe<P> u, v;
        fe_mul2(u, x, y, v, y, x);
        r = op == FT_PAIR_A ? u : v;
      } else {
        const Fe<PD> xd = fe_mul(toD(x), kin), yd = fe_mul(toD(y), kin);
        Fe<PD> u, v;
        fe_mul2(u, toD(x), yd, v, toD(y), xd);
        r = fromD(op == FT_PAIR_A ? u : v);
      }
      break;
    case FT_SQR_PAIR:
      if (path == 0) {
        Fe<P> u, v;
        fe_sqr2(u, x, v, y);
        r = u;
      } else {
        Fe<PD> u, v;
        fe_sqr2(u, fe_mul(toD(x), kin), v, fe_mul(toD(y), kin));
        r = fromD(fe_mul(u, kout));
      }
      break;
    default: r = fe_zero<P>(); break;
  }
  fe_store<P>(out + (size_t)i * P::N, r);
}

// 2^e mod p as field words (a standard integer: an operand of mont'(., .), not a value in
// either radix)
template <class PD, int NL>
static Fe<PD> pow2_words(const host::Field<NL>& F, int e) {
  host::El<NL> x = host::zero<NL>();
  x.v[0] = 1;
  for (int i = 0; i < e; i++) x = host::add(F, x, x);
  Fe<PD> out;
  for (int w = 0; w < PD::N; w++) out.v[w] = (uint32_t)(x.v[w >> 1] >> (32 * (w & 1)));
  return out;
}

template <class P, class PD, class PL, class PE, int NL>
static zkg_status field_test(const host::Field<NL>& F, int op, int path, int n, const uint64_t* d_a,
                             const uint64_t* d_b, uint64_t* d_out) {
  const bool path_ok = path == 0 || path == 1 || path == 3 || (path == 2 && lazy_v<PL>);
  if (n < 0 || op < 0 || op > 8 || !path_ok || (path >= 2 && op == FT_RAW_DPF) || (n > 0 && (!d_a || !d_out)))
    return set_status(ZKG_ERR_ARG, "zkg_field_test_device", "bad arguments");
  if (n > 0 && !d_b && (op == FT_MUL || op == FT_ADD || op == FT_SUB || op == FT_RAW_DPF || op == FT_PAIR_A ||
                        op == FT_PAIR_B || op == FT_SQR_PAIR))
    return set_status(ZKG_ERR_ARG, "zkg_field_test_device", "operation needs b");
  if (n == 0) return set_status(ZKG_OK, nullptr, nullptr);
  Context* cx = nullptr;
  ZKB_TRY(get_context(&cx));
  std::lock_guard<std::mutex> lk(cx->mu);
  constexpr int L = D52<PD>::L;
  const Fe<PD> kin = pow2_words<PD, NL>(F, 2 * 52 * L - 32 * PD::N);   // R'^2 / R
  const Fe<PD> kout = pow2_words<PD, NL>(F, 32 * PD::N);               // R
  const cudaStream_t st = cx->compute();
  ZKB_TRY(launch("field_test", k_field_test<P, PD, PL, PE>, dim3(((uint32_t)n + 255) / 256), dim3(256), 0, st, op, path,
                 (uint32_t)n, reinterpret_cast<const uint32_t*>(d_a), reinterpret_cast<const uint32_t*>(d_b),
                 reinterpret_cast<uint32_t*>(d_out), kin, kout));
  ZKB_CUDA(cudaStreamSynchronize(st));
  return set_status(ZKG_OK, nullptr, nullptr);
}

// Product-throughput probe: every thread runs four independent chains of the MSM bucket
// pipeline's field product (the exact-radix FP64 product on the redundant range [0, 2p), in
// pairs through fe_mul2 as the point formulas call it), a_j <- a_j b_j. The rate it measures is
// the ceiling of any kernel whose work is these products.
template <class P>
__global__ void __launch_bounds__(256) k_product_probe(uint32_t* out, int iters) {
  Fe<P> a[4], b[4];
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int w = 0; w < P::N; w++) {
      a[j].v[w] = (w == P::N - 1) ? 0u : (threadIdx.x * 2654435761u + 97u * j + w);
      b[j].v[w] = (w == P::N - 1) ? 0u : (blockIdx.x * 40503u + 131u * j + 7u * w + 1u);
    }
  for (int i = 0; i < iters; i++) {
    fe_mul2(a[0], a[0], b[0], a[1], a[1], b[1]);
    fe_mul2(a[2], a[2], b[2], a[3], a[3], b[3]);
  }
  uint32_t x = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) x ^= a[j].v[0];
  if (x == 0x9e3779b9u) out[0] = x;   // keeps the chains live
}

template <class P>
static double product_probe() {
  Context* cx = nullptr;
  if (get_context(&cx) != ZKG_OK) return -1.0;
  std::lock_guard<std::mutex> lk(cx->mu);
  uint32_t* d = nullptr;
  if (cudaMalloc(&d, 64) != cudaSuccess) return -1.0;
  const int iters = 256, threads = 256, blocks = cx->sm_count * 4;
  double best = 0.0;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(cx->ev_a, cx->stream);
    k_product_probe<P><<<blocks, threads, 0, cx->stream>>>(d, iters);
    g_launches.fetch_add(1);
    cudaEventRecord(cx->ev_b, cx->stream);
    if (cudaStreamSynchronize(cx->stream) != cudaSuccess) { cudaFree(d); return -1.0; }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, cx->ev_a, cx->ev_b);
    const double n = (double)blocks * threads * iters * 4.0;
    if (rep > 0 && ms > 0) best = std::max(best, n / (ms * 1e-3));
  }
  cudaFree(d);
  return best;
}

}  // namespace zkb

extern "C" double zkg_product_probe(zkg_curve curve) {
  if (curve == ZKG_BN254) return zkb::product_probe<zkb::BnFpLE>();
  if (curve == ZKG_BLS12_381) return zkb::product_probe<zkb::BlsFpLE>();
  return -1.0;
}

extern "C" zkg_status zkg_field_test_device(zkg_curve curve, int field, int path, int op, int n, const uint64_t* d_a,
                                            const uint64_t* d_b, uint64_t* d_out) {
  using namespace zkb;
  if (curve == ZKG_BN254 && field == 0)
    return field_test<BnFp, BnFpD, BnFpL, BnFpE, 4>(host::BN_FP, op, path, n, d_a, d_b, d_out);
  if (curve == ZKG_BN254 && field == 1)
    return field_test<BnFr, BnFrD, BnFrD, BnFrE, 4>(host::BN_FR, op, path, n, d_a, d_b, d_out);
  if (curve == ZKG_BLS12_381 && field == 0)
    return field_test<BlsFp, BlsFpD, BlsFpL, BlsFpE, 6>(host::BLS_FP, op, path, n, d_a, d_b, d_out);
  if (curve == ZKG_BLS12_381 && field == 1)
    return field_test<BlsFr, BlsFrD, BlsFrD, BlsFrE, 4>(host::BLS_FR, op, path, n, d_a, d_b, d_out);
  return set_status(ZKG_ERR_ARG, "zkg_field_test_device", "unknown curve or field");
}
