// Drop-in entry points with the reference's names and signatures (lib/cbits, see
// include/zkb200.h for the per-symbol citations). They forward to the native zkg_* calls.
//
// The reference returns void and aborts (assert) when it cannot allocate
// (lib/cbits/curves/g1/proj/bn128_G1_proj.c:508,517; lib/cbits/curves/poly/mont/
// bn128_poly_mont.c:458,469). These wrappers likewise report a failed call on stderr and
// abort, so a failure is never silent. With ZKB200_NO_ABORT set in the environment they
// return instead, leaving the status in zkg_last_status() and tgt holding the infinity
// encoding (MSM) or zeros (NTT).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/zkb200.h"

namespace {

void fail(const char* fn, zkg_status s, uint64_t* tgt, size_t fill_words, int fill_byte) {
  std::fprintf(stderr, "zkb200: %s failed (status %d): %s\n", fn, s, zkg_last_error());
  if (!std::getenv("ZKB200_NO_ABORT")) std::abort();
  if (tgt && fill_words) std::memset(tgt, fill_byte, fill_words * 8);
}

void msm(const char* fn, zkg_curve curve, int nlp, int mont, zkg_out_kind kind, int npoints, const uint64_t* expos,
         const uint64_t* grps, uint64_t* tgt, int expo_nlimbs) {
  const zkg_status s = zkg_msm(curve, npoints, expos, expo_nlimbs, mont, grps, kind, tgt);
  if (s != ZKG_OK) fail(fn, s, tgt, (kind == ZKG_OUT_AFFINE ? 2 : 3) * nlp, kind == ZKG_OUT_AFFINE ? 0xff : 0);
}

void ntt(const char* fn, zkg_curve curve, int m, const uint64_t* gen, const uint64_t* src, uint64_t* tgt, int inv) {
  const zkg_status s = zkg_ntt(curve, m, gen, src, tgt, inv);
  if (s != ZKG_OK) fail(fn, s, tgt, (m >= 0 && m <= 28) ? ((size_t)4 << m) : 0, 0);
}

}  // namespace

#define ZKB_MSM_ENTRY(name, curve, nlp, mont, kind)                                                        \
  extern "C" void name(int npoints, const uint64_t* expos, const uint64_t* grps, uint64_t* tgt, int expo_nlimbs) { \
    msm(#name, curve, nlp, mont, kind, npoints, expos, grps, tgt, expo_nlimbs);                            \
  }

ZKB_MSM_ENTRY(bn128_G1_proj_MSM_std_coeff_proj_out, ZKG_BN254, 4, 0, ZKG_OUT_PROJ)
ZKB_MSM_ENTRY(bn128_G1_proj_MSM_mont_coeff_proj_out, ZKG_BN254, 4, 1, ZKG_OUT_PROJ)
ZKB_MSM_ENTRY(bn128_G1_proj_MSM_std_coeff_affine_out, ZKG_BN254, 4, 0, ZKG_OUT_AFFINE)
ZKB_MSM_ENTRY(bn128_G1_proj_MSM_mont_coeff_affine_out, ZKG_BN254, 4, 1, ZKG_OUT_AFFINE)
ZKB_MSM_ENTRY(bn128_G1_jac_MSM_std_coeff_jac_out, ZKG_BN254, 4, 0, ZKG_OUT_JAC)
ZKB_MSM_ENTRY(bn128_G1_jac_MSM_mont_coeff_jac_out, ZKG_BN254, 4, 1, ZKG_OUT_JAC)
ZKB_MSM_ENTRY(bn128_G1_jac_MSM_std_coeff_affine_out, ZKG_BN254, 4, 0, ZKG_OUT_AFFINE)
ZKB_MSM_ENTRY(bn128_G1_jac_MSM_mont_coeff_affine_out, ZKG_BN254, 4, 1, ZKG_OUT_AFFINE)

ZKB_MSM_ENTRY(bls12_381_G1_proj_MSM_std_coeff_proj_out, ZKG_BLS12_381, 6, 0, ZKG_OUT_PROJ)
ZKB_MSM_ENTRY(bls12_381_G1_proj_MSM_mont_coeff_proj_out, ZKG_BLS12_381, 6, 1, ZKG_OUT_PROJ)
ZKB_MSM_ENTRY(bls12_381_G1_proj_MSM_std_coeff_affine_out, ZKG_BLS12_381, 6, 0, ZKG_OUT_AFFINE)
ZKB_MSM_ENTRY(bls12_381_G1_proj_MSM_mont_coeff_affine_out, ZKG_BLS12_381, 6, 1, ZKG_OUT_AFFINE)
ZKB_MSM_ENTRY(bls12_381_G1_jac_MSM_std_coeff_jac_out, ZKG_BLS12_381, 6, 0, ZKG_OUT_JAC)
ZKB_MSM_ENTRY(bls12_381_G1_jac_MSM_mont_coeff_jac_out, ZKG_BLS12_381, 6, 1, ZKG_OUT_JAC)
ZKB_MSM_ENTRY(bls12_381_G1_jac_MSM_std_coeff_affine_out, ZKG_BLS12_381, 6, 0, ZKG_OUT_AFFINE)
ZKB_MSM_ENTRY(bls12_381_G1_jac_MSM_mont_coeff_affine_out, ZKG_BLS12_381, 6, 1, ZKG_OUT_AFFINE)

extern "C" void bn128_poly_mont_ntt_forward(int m, const uint64_t* gen, const uint64_t* src, uint64_t* tgt) {
  ntt("bn128_poly_mont_ntt_forward", ZKG_BN254, m, gen, src, tgt, 0);
}
extern "C" void bn128_poly_mont_ntt_inverse(int m, const uint64_t* gen, const uint64_t* src, uint64_t* tgt) {
  ntt("bn128_poly_mont_ntt_inverse", ZKG_BN254, m, gen, src, tgt, 1);
}
extern "C" void bls12_381_poly_mont_ntt_forward(int m, const uint64_t* gen, const uint64_t* src, uint64_t* tgt) {
  ntt("bls12_381_poly_mont_ntt_forward", ZKG_BLS12_381, m, gen, src, tgt, 0);
}
extern "C" void bls12_381_poly_mont_ntt_inverse(int m, const uint64_t* gen, const uint64_t* src, uint64_t* tgt) {
  ntt("bls12_381_poly_mont_ntt_inverse", ZKG_BLS12_381, m, gen, src, tgt, 1);
}


#define ZKB_SHIFTED_ENTRY(name, curve, inv)                                                              \
  extern "C" void name(const uint64_t* eta, int m, const uint64_t* gen, const uint64_t* src, uint64_t* tgt) { \
    const zkg_status s = zkg_ntt_shifted(curve, eta, m, gen, src, tgt, inv);                              \
    if (s != ZKG_OK) fail(#name, s, tgt, (m >= 0 && m <= 28) ? ((size_t)4 << m) : 0, 0);                \
  }
ZKB_SHIFTED_ENTRY(bn128_poly_mont_ntt_forward_shifted, ZKG_BN254, 0)
ZKB_SHIFTED_ENTRY(bn128_poly_mont_ntt_inverse_shifted, ZKG_BN254, 1)
ZKB_SHIFTED_ENTRY(bls12_381_poly_mont_ntt_forward_shifted, ZKG_BLS12_381, 0)
ZKB_SHIFTED_ENTRY(bls12_381_poly_mont_ntt_inverse_shifted, ZKG_BLS12_381, 1)

#define ZKB_ASYM_ENTRY(name, curve)                                                                      \
  extern "C" void name(int m_src, int m_tgt, const uint64_t* gen_src, const uint64_t* gen_tgt, const uint64_t* src, \
                       uint64_t* tgt) {                                                                  \
    const zkg_status s = zkg_ntt_asymmetric(curve, m_src, m_tgt, gen_src, gen_tgt, src, tgt);            \
    if (s != ZKG_OK) fail(#name, s, tgt, (m_tgt >= 0 && m_tgt <= 28) ? ((size_t)4 << m_tgt) : 0, 0);     \
  }
ZKB_ASYM_ENTRY(bn128_poly_mont_ntt_forward_asymmetric, ZKG_BN254)
ZKB_ASYM_ENTRY(bls12_381_poly_mont_ntt_forward_asymmetric, ZKG_BLS12_381)

// Binary MSMs (coefficients are bytes, non-zero = 1) and multi-row binary MSMs
#define ZKB_BIN_ENTRY(name, curve, nlp, kind)                                                              \
  extern "C" void name(int npoints, const uint8_t* expos, const uint64_t* grps, uint64_t* tgt) {           \
    const uint8_t* rows[1] = {expos};                                                                     \
    const zkg_status s = zkg_msm_binary(curve, kind, 1, npoints, rows, grps, tgt);                        \
    if (s != ZKG_OK) fail(#name, s, tgt, (kind == ZKG_OUT_AFFINE ? 2 : 3) * nlp, kind == ZKG_OUT_AFFINE ? 0xff : 0); \
  }
#define ZKB_MULTI_BIN_ENTRY(name, curve, nlp, kind)                                                        \
  extern "C" void name(int nrows, int npoints, const uint8_t** expos, const uint64_t* grps, uint64_t* tgt) { \
    const zkg_status s = zkg_msm_binary(curve, kind, nrows, npoints, expos, grps, tgt);                   \
    if (s != ZKG_OK)                                                                                      \
      fail(#name, s, tgt, nrows > 0 ? (size_t)nrows * (kind == ZKG_OUT_AFFINE ? 2 : 3) * nlp : 0,          \
           kind == ZKG_OUT_AFFINE ? 0xff : 0);                                                            \
  }
ZKB_BIN_ENTRY(bn128_G1_proj_MSM_binary_coeff_proj_out, ZKG_BN254, 4, ZKG_OUT_PROJ)
ZKB_BIN_ENTRY(bn128_G1_proj_MSM_binary_coeff_affine_out, ZKG_BN254, 4, ZKG_OUT_AFFINE)
ZKB_BIN_ENTRY(bn128_G1_jac_MSM_binary_coeff_jac_out, ZKG_BN254, 4, ZKG_OUT_JAC)
ZKB_BIN_ENTRY(bn128_G1_jac_MSM_binary_coeff_affine_out, ZKG_BN254, 4, ZKG_OUT_AFFINE)
ZKB_BIN_ENTRY(bls12_381_G1_proj_MSM_binary_coeff_proj_out, ZKG_BLS12_381, 6, ZKG_OUT_PROJ)
ZKB_BIN_ENTRY(bls12_381_G1_proj_MSM_binary_coeff_affine_out, ZKG_BLS12_381, 6, ZKG_OUT_AFFINE)
ZKB_BIN_ENTRY(bls12_381_G1_jac_MSM_binary_coeff_jac_out, ZKG_BLS12_381, 6, ZKG_OUT_JAC)
ZKB_BIN_ENTRY(bls12_381_G1_jac_MSM_binary_coeff_affine_out, ZKG_BLS12_381, 6, ZKG_OUT_AFFINE)
ZKB_MULTI_BIN_ENTRY(bn128_G1_proj_multi_MSM_binary_coeff_proj_out, ZKG_BN254, 4, ZKG_OUT_PROJ)
ZKB_MULTI_BIN_ENTRY(bn128_G1_proj_multi_MSM_binary_coeff_affine_out, ZKG_BN254, 4, ZKG_OUT_AFFINE)
ZKB_MULTI_BIN_ENTRY(bn128_G1_jac_multi_MSM_binary_coeff_jac_out, ZKG_BN254, 4, ZKG_OUT_JAC)
ZKB_MULTI_BIN_ENTRY(bn128_G1_jac_multi_MSM_binary_coeff_affine_out, ZKG_BN254, 4, ZKG_OUT_AFFINE)
ZKB_MULTI_BIN_ENTRY(bls12_381_G1_proj_multi_MSM_binary_coeff_proj_out, ZKG_BLS12_381, 6, ZKG_OUT_PROJ)
ZKB_MULTI_BIN_ENTRY(bls12_381_G1_proj_multi_MSM_binary_coeff_affine_out, ZKG_BLS12_381, 6, ZKG_OUT_AFFINE)
ZKB_MULTI_BIN_ENTRY(bls12_381_G1_jac_multi_MSM_binary_coeff_jac_out, ZKG_BLS12_381, 6, ZKG_OUT_JAC)
ZKB_MULTI_BIN_ENTRY(bls12_381_G1_jac_multi_MSM_binary_coeff_affine_out, ZKG_BLS12_381, 6, ZKG_OUT_AFFINE)

// G1 group FFTs over projective or Jacobian points; outputs normalised
#define ZKB_G1_FFT_ENTRY(name, curve, nlp, jac, inv)                                                       \
  extern "C" void name(int m, const uint64_t* gen, const uint64_t* src, uint64_t* tgt) {                 \
    const zkg_status s = zkg_g1_fft(curve, jac, m, gen, src, tgt, inv);                                   \
    if (s != ZKG_OK) fail(#name, s, tgt, (m >= 0 && m <= 26) ? ((size_t)3 * nlp << m) : 0, 0);            \
  }
ZKB_G1_FFT_ENTRY(bn128_G1_proj_fft_forward, ZKG_BN254, 4, 0, 0)
ZKB_G1_FFT_ENTRY(bn128_G1_proj_fft_inverse, ZKG_BN254, 4, 0, 1)
ZKB_G1_FFT_ENTRY(bn128_G1_jac_fft_forward, ZKG_BN254, 4, 1, 0)
ZKB_G1_FFT_ENTRY(bn128_G1_jac_fft_inverse, ZKG_BN254, 4, 1, 1)
ZKB_G1_FFT_ENTRY(bls12_381_G1_proj_fft_forward, ZKG_BLS12_381, 6, 0, 0)
ZKB_G1_FFT_ENTRY(bls12_381_G1_proj_fft_inverse, ZKG_BLS12_381, 6, 0, 1)
ZKB_G1_FFT_ENTRY(bls12_381_G1_jac_fft_forward, ZKG_BLS12_381, 6, 1, 0)
ZKB_G1_FFT_ENTRY(bls12_381_G1_jac_fft_inverse, ZKG_BLS12_381, 6, 1, 1)
