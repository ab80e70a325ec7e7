// Device generation of G1 points k_i * G (affine, Montgomery), used to build benchmark and test
// inputs the way the reference's tests do (rndG1 = k*G,
// lib/src/ZK/Algebra/Curves/BN128/G1/Affine.hs; scalar multiplication
// lib/cbits/curves/g1/affine/bn128_G1_affine.c:235).
//
// Fixed-base comb: T[j][v] = v * 16^j * G for j < 64, v < 16 is built once on the host in
// XYZZ coordinates; each thread adds one table entry per 4-bit digit of its scalar and converts
// the sum to affine with a Fermat inversion.
#include <cstring>
#include <vector>

#include "zkb_curve.cuh"
#include "zkb_host_ec.h"
#include "zkb_runtime.h"

namespace zkb {

template <class C>
__global__ void k_g1_gen_mul(int n, const uint64_t* __restrict__ ks, const uint32_t* __restrict__ table,
                             uint32_t* __restrict__ out) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* k = reinterpret_cast<const uint32_t*>(ks + 4 * (size_t)i);
  Xyzz<F> acc = xyzz_inf<F>();
  for (int j = 0; j < 64; j++) {
    const uint32_t d = (__ldg(k + (j >> 3)) >> (4 * (j & 7))) & 15u;
    if (d) xyzz_add(acc, xyzz_load<F>(table + ((size_t)j * 16 + d) * XW));
  }
  uint32_t* o = out + (size_t)i * 2 * F::N;
  if (xyzz_is_inf(acc)) {
    fe_store<F>(o, fe_zero<F>());
    fe_store<F>(o + F::N, fe_zero<F>());
    return;
  }
  const Fe<F> d = fe_inv_fermat(fe_mul(acc.ZZ, acc.ZZZ));
  fe_store<F>(o, fe_mul(acc.X, fe_mul(d, acc.ZZZ)));
  fe_store<F>(o + F::N, fe_mul(acc.Y, fe_mul(d, acc.ZZ)));
}

template <int NL>
static std::vector<uint64_t> comb_table(const host::Field<NL>& F, const uint64_t* gx_std, const uint64_t* gy_std) {
  using host::El;
  El<NL> x, y;
  std::memcpy(x.v, gx_std, 8 * NL);
  std::memcpy(y.v, gy_std, 8 * NL);
  host::Xyzz<NL> base;
  base.X = host::from_std(F, x);
  base.Y = host::from_std(F, y);
  base.ZZ = host::one(F);
  base.ZZZ = host::one(F);
  std::vector<uint64_t> tab((size_t)64 * 16 * 4 * NL, 0);
  for (int j = 0; j < 64; j++) {
    host::Xyzz<NL> acc = host::xyzz_inf<NL>();
    for (int v = 0; v < 16; v++) {
      uint64_t* p = tab.data() + ((size_t)j * 16 + v) * 4 * NL;
      std::memcpy(p, acc.X.v, 8 * NL);
      std::memcpy(p + NL, acc.Y.v, 8 * NL);
      std::memcpy(p + 2 * NL, acc.ZZ.v, 8 * NL);
      std::memcpy(p + 3 * NL, acc.ZZZ.v, 8 * NL);
      acc = host::xyzz_add(F, acc, base);
    }
    for (int d = 0; d < 4; d++) base = host::xyzz_dbl(F, base);
  }
  return tab;
}

// G1 generators in standard form: BN254 (1, 2); BLS12-381 as in
// lib/cbits/curves/g1/affine/bls12_381_G1_affine.c:33 (there in Montgomery form)
static const uint64_t BN_GX[4] = {1, 0, 0, 0}, BN_GY[4] = {2, 0, 0, 0};
static const uint64_t BLS_GX[6] = {0xfb3af00adb22c6bbULL, 0x6c55e83ff97a1aefULL, 0xa14e3a3f171bac58ULL,
                                   0xc3688c4f9774b905ULL, 0x2695638c4fa9ac0fULL, 0x17f1d3a73197d794ULL};
static const uint64_t BLS_GY[6] = {0x0caa232946c5e7e1ULL, 0xd03cc744a2888ae4ULL, 0x00db18cb2c04b3edULL,
                                   0xfcf5e095d5d00af6ULL, 0xa09e30ed741d8ae4ULL, 0x08b3f481e3aaa0f1ULL};

template <class C, int NL>
static zkg_status gen_mul(const host::Field<NL>& F, const uint64_t* gx, const uint64_t* gy, int n,
                          const uint64_t* d_ks, uint64_t* d_out) {
  if (n < 0 || (n > 0 && (!d_ks || !d_out))) return set_status(ZKG_ERR_ARG, "g1_gen_mul", "bad arguments");
  if (n == 0) return ZKG_OK;
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  const std::vector<uint64_t> tab = comb_table<NL>(F, gx, gy);
  uint32_t* d_tab = nullptr;
  ZKB_CUDA(cudaMalloc(&d_tab, tab.size() * 8));
  zkg_status st = ZKG_OK;
  if (cudaMemcpy(d_tab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
    st = set_status(ZKG_ERR_CUDA, "g1_gen_mul", "table upload");
  if (st == ZKG_OK) cudaDeviceSynchronize();
  if (st == ZKG_OK)
    st = launch("g1_gen_mul", k_g1_gen_mul<C>, dim3((n + 127) / 128), dim3(128), 0, cx.stream, n, d_ks,
                (const uint32_t*)d_tab, reinterpret_cast<uint32_t*>(d_out));
  if (st == ZKG_OK && cudaStreamSynchronize(cx.stream) != cudaSuccess)
    st = set_status(ZKG_ERR_CUDA, "g1_gen_mul", "sync");
  cudaFree(d_tab);
  return st == ZKG_OK ? set_status(ZKG_OK, nullptr, nullptr) : st;
}

}  // namespace zkb

extern "C" zkg_status zkg_g1_gen_mul_device(zkg_curve curve, int n, const uint64_t* d_scalars_std,
                                            uint64_t* d_out_affine) {
  if (curve == ZKG_BN254)
    return zkb::gen_mul<zkb::BN254, 4>(zkb::host::BN_FP, zkb::BN_GX, zkb::BN_GY, n, d_scalars_std, d_out_affine);
  if (curve == ZKG_BLS12_381)
    return zkb::gen_mul<zkb::BLS12_381, 6>(zkb::host::BLS_FP, zkb::BLS_GX, zkb::BLS_GY, n, d_scalars_std,
                                           d_out_affine);
  return zkb::set_status(ZKG_ERR_ARG, "zkg_g1_gen_mul_device", "unknown curve");
}
