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
#include "zkb_ntt.h"

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
  if (s != ZKG_OK) fail(fn, s, tgt, (m >= 0 && m <= zkb::NTT_MMAX) ? ((size_t)4 << m) : 0, 0);
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
    if (s != ZKG_OK) fail(#name, s, tgt, (m >= 0 && m <= zkb::NTT_MMAX) ? ((size_t)4 << m) : 0, 0);                \
  }
ZKB_SHIFTED_ENTRY(bn128_poly_mont_ntt_forward_shifted, ZKG_BN254, 0)
ZKB_SHIFTED_ENTRY(bn128_poly_mont_ntt_inverse_shifted, ZKG_BN254, 1)
ZKB_SHIFTED_ENTRY(bls12_381_poly_mont_ntt_forward_shifted, ZKG_BLS12_381, 0)
ZKB_SHIFTED_ENTRY(bls12_381_poly_mont_ntt_inverse_shifted, ZKG_BLS12_381, 1)

#define ZKB_ASYM_ENTRY(name, curve)                                                                      \
  extern "C" void name(int m_src, int m_tgt, const uint64_t* gen_src, const uint64_t* gen_tgt, const uint64_t* src, \
                       uint64_t* tgt) {                                                                  \
    const zkg_status s = zkg_ntt_asymmetric(curve, m_src, m_tgt, gen_src, gen_tgt, src, tgt);            \
    if (s != ZKG_OK) fail(#name, s, tgt, (m_tgt >= 0 && m_tgt <= zkb::NTT_MMAX) ? ((size_t)4 << m_tgt) : 0, 0);     \
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

// Fr vector operations (*_arr_mont_*). Arithmetic runs on the GPU through zkg_fr_*; copies and
// constant fills are host memory moves, as in the reference.
namespace {

const uint64_t FR_ONE[2][4] = {
    {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL},   // BN254 R mod r
    {0x00000001fffffffeULL, 0x5884b7fa00034802ULL, 0x998c4fefecbc4ff5ULL, 0x1824b159acc5056fULL}};  // BLS12-381

void arr_map(const char* fn, zkg_curve curve, int op, int n, const uint64_t* a, const uint64_t* b, const uint64_t* c,
             const uint64_t* ka, const uint64_t* kb, uint64_t* tgt) {
  const zkg_status s = zkg_fr_map(curve, op, n, a, b, c, ka, kb, tgt);
  if (s != ZKG_OK) fail(fn, s, tgt, n > 0 ? (size_t)4 * n : 0, 0);
}

uint8_t arr_pred(const char* fn, zkg_curve curve, int which, int n, const uint64_t* a, const uint64_t* b) {
  int r = 0;
  const zkg_status s = zkg_fr_predicate(curve, which, n, a, b, &r);
  if (s != ZKG_OK) {
    fail(fn, s, nullptr, 0, 0);
    return 0;
  }
  return (uint8_t)(r ? 1 : 0);
}

}  // namespace

#define ZKB_ARR_ENTRIES(P, CURVE, CI)                                                                          \
  extern "C" uint8_t P##_arr_mont_is_valid(int n, const uint64_t* src) {                                     \
    return arr_pred(#P "_arr_mont_is_valid", CURVE, 0, n, src, nullptr);                                      \
  }                                                                                                          \
  extern "C" uint8_t P##_arr_mont_is_zero(int n, const uint64_t* src) {                                      \
    return arr_pred(#P "_arr_mont_is_zero", CURVE, 1, n, src, nullptr);                                       \
  }                                                                                                          \
  extern "C" uint8_t P##_arr_mont_is_one(int n, const uint64_t* src) {                                       \
    return arr_pred(#P "_arr_mont_is_one", CURVE, 2, n, src, nullptr);                                        \
  }                                                                                                          \
  extern "C" uint8_t P##_arr_mont_is_equal(int n, const uint64_t* src1, const uint64_t* src2) {              \
    return arr_pred(#P "_arr_mont_is_equal", CURVE, 3, n, src1, src2);                                        \
  }                                                                                                          \
  extern "C" void P##_arr_mont_set_zero(int n, uint64_t* tgt) {                                              \
    if (n > 0) std::memset(tgt, 0, (size_t)32 * n);                                                          \
  }                                                                                                          \
  extern "C" void P##_arr_mont_set_one(int n, uint64_t* tgt) {                                               \
    for (int i = 0; i < n; i++) std::memcpy(tgt + (size_t)4 * i, FR_ONE[CI], 32);                            \
  }                                                                                                          \
  extern "C" void P##_arr_mont_set_const(int n, const uint64_t* src, uint64_t* tgt) {                        \
    for (int i = 0; i < n; i++) std::memcpy(tgt + (size_t)4 * i, src, 32);                                   \
  }                                                                                                          \
  extern "C" void P##_arr_mont_copy(int n, const uint64_t* src, uint64_t* tgt) {                             \
    if (n > 0) std::memcpy(tgt, src, (size_t)32 * n);                                                        \
  }                                                                                                          \
  extern "C" void P##_arr_mont_append(int n1, int n2, const uint64_t* src1, const uint64_t* src2, uint64_t* tgt) { \
    if (n1 > 0) std::memcpy(tgt, src1, (size_t)32 * n1);                                                     \
    if (n2 > 0) std::memcpy(tgt + (size_t)4 * (n1 > 0 ? n1 : 0), src2, (size_t)32 * n2);                     \
  }                                                                                                          \
  extern "C" void P##_arr_mont_concat(int K, int* ns, const uint64_t** srcs, uint64_t* tgt) {                \
    uint64_t* q = tgt;                                                                                       \
    for (int k = 0; k < K; k++) {                                                                            \
      if (ns[k] > 0) std::memcpy(q, srcs[k], (size_t)32 * ns[k]);                                            \
      q += (size_t)4 * (ns[k] > 0 ? ns[k] : 0);                                                              \
    }                                                                                                        \
  }                                                                                                          \
  extern "C" void P##_arr_mont_from_std(int n, const uint64_t* src, uint64_t* tgt) {                         \
    arr_map(#P "_arr_mont_from_std", CURVE, ZKG_FR_FROM_STD, n, src, 0, 0, 0, 0, tgt);                        \
  }                                                                                                          \
  extern "C" void P##_arr_mont_to_std(int n, const uint64_t* src, uint64_t* tgt) {                           \
    arr_map(#P "_arr_mont_to_std", CURVE, ZKG_FR_TO_STD, n, src, 0, 0, 0, 0, tgt);                            \
  }                                                                                                          \
  extern "C" void P##_arr_mont_neg(int n, const uint64_t* src, uint64_t* tgt) {                              \
    arr_map(#P "_arr_mont_neg", CURVE, ZKG_FR_NEG, n, src, 0, 0, 0, 0, tgt);                                  \
  }                                                                                                          \
  extern "C" void P##_arr_mont_add(int n, const uint64_t* src1, const uint64_t* src2, uint64_t* tgt) {       \
    arr_map(#P "_arr_mont_add", CURVE, ZKG_FR_ADD, n, src1, src2, 0, 0, 0, tgt);                              \
  }                                                                                                          \
  extern "C" void P##_arr_mont_sub(int n, const uint64_t* src1, const uint64_t* src2, uint64_t* tgt) {       \
    arr_map(#P "_arr_mont_sub", CURVE, ZKG_FR_SUB, n, src1, src2, 0, 0, 0, tgt);                              \
  }                                                                                                          \
  extern "C" void P##_arr_mont_sqr(int n, const uint64_t* src, uint64_t* tgt) {                              \
    arr_map(#P "_arr_mont_sqr", CURVE, ZKG_FR_SQR, n, src, 0, 0, 0, 0, tgt);                                  \
  }                                                                                                          \
  extern "C" void P##_arr_mont_mul(int n, const uint64_t* src1, const uint64_t* src2, uint64_t* tgt) {       \
    arr_map(#P "_arr_mont_mul", CURVE, ZKG_FR_MUL, n, src1, src2, 0, 0, 0, tgt);                              \
  }                                                                                                          \
  extern "C" void P##_arr_mont_inv(int n, const uint64_t* src, uint64_t* tgt) {                              \
    arr_map(#P "_arr_mont_inv", CURVE, ZKG_FR_INV, n, src, 0, 0, 0, 0, tgt);                                  \
  }                                                                                                          \
  extern "C" void P##_arr_mont_div(int n, const uint64_t* src1, const uint64_t* src2, uint64_t* tgt) {       \
    arr_map(#P "_arr_mont_div", CURVE, ZKG_FR_DIV, n, src1, src2, 0, 0, 0, tgt);                              \
  }                                                                                                          \
  extern "C" void P##_arr_mont_mul_add(int n, const uint64_t* src1, const uint64_t* src2, const uint64_t* src3, \
                                       uint64_t* tgt) {                                                      \
    arr_map(#P "_arr_mont_mul_add", CURVE, ZKG_FR_MUL_ADD, n, src1, src2, src3, 0, 0, tgt);                   \
  }                                                                                                          \
  extern "C" void P##_arr_mont_mul_sub(int n, const uint64_t* src1, const uint64_t* src2, const uint64_t* src3, \
                                       uint64_t* tgt) {                                                      \
    arr_map(#P "_arr_mont_mul_sub", CURVE, ZKG_FR_MUL_SUB, n, src1, src2, src3, 0, 0, tgt);                   \
  }                                                                                                          \
  extern "C" void P##_arr_mont_neg_inplace(int n, uint64_t* tgt) {                                           \
    arr_map(#P "_arr_mont_neg_inplace", CURVE, ZKG_FR_NEG, n, tgt, 0, 0, 0, 0, tgt);                          \
  }                                                                                                          \
  extern "C" void P##_arr_mont_add_inplace(int n, uint64_t* tgt, const uint64_t* src2) {                     \
    arr_map(#P "_arr_mont_add_inplace", CURVE, ZKG_FR_ADD, n, tgt, src2, 0, 0, 0, tgt);                       \
  }                                                                                                          \
  extern "C" void P##_arr_mont_sub_inplace(int n, uint64_t* tgt, const uint64_t* src2) {                     \
    arr_map(#P "_arr_mont_sub_inplace", CURVE, ZKG_FR_SUB, n, tgt, src2, 0, 0, 0, tgt);                       \
  }                                                                                                          \
  extern "C" void P##_arr_mont_sqr_inplace(int n, uint64_t* tgt) {                                           \
    arr_map(#P "_arr_mont_sqr_inplace", CURVE, ZKG_FR_SQR, n, tgt, 0, 0, 0, 0, tgt);                          \
  }                                                                                                          \
  extern "C" void P##_arr_mont_mul_inplace(int n, uint64_t* tgt, const uint64_t* src2) {                     \
    arr_map(#P "_arr_mont_mul_inplace", CURVE, ZKG_FR_MUL, n, tgt, src2, 0, 0, 0, tgt);                       \
  }                                                                                                          \
  extern "C" void P##_arr_mont_inv_inplace(int n, uint64_t* tgt) {                                           \
    arr_map(#P "_arr_mont_inv_inplace", CURVE, ZKG_FR_INV, n, tgt, 0, 0, 0, 0, tgt);                          \
  }                                                                                                          \
  extern "C" void P##_arr_mont_div_inplace(int n, uint64_t* tgt, const uint64_t* src2) {                     \
    arr_map(#P "_arr_mont_div_inplace", CURVE, ZKG_FR_DIV, n, tgt, src2, 0, 0, 0, tgt);                       \
  }                                                                                                          \
  extern "C" void P##_arr_mont_sub_inplace_reverse(int n, uint64_t* tgt, const uint64_t* src1) {             \
    arr_map(#P "_arr_mont_sub_inplace_reverse", CURVE, ZKG_FR_SUB, n, src1, tgt, 0, 0, 0, tgt);               \
  }                                                                                                          \
  extern "C" void P##_arr_mont_dot_prod(int n, const uint64_t* src1, const uint64_t* src2, uint64_t* tgt) {  \
    const zkg_status s = zkg_fr_dot(CURVE, n, src1, src2, tgt);                                              \
    if (s != ZKG_OK) fail(#P "_arr_mont_dot_prod", s, tgt, 4, 0);                                            \
  }                                                                                                          \
  extern "C" void P##_arr_mont_powers(int n, const uint64_t* coeffA, const uint64_t* coeffB, uint64_t* tgt) { \
    arr_map(#P "_arr_mont_powers", CURVE, ZKG_FR_POWERS, n, 0, 0, 0, coeffA, coeffB, tgt);                    \
  }                                                                                                          \
  extern "C" void P##_arr_mont_mul_by_powers(int n, const uint64_t* coeffA, const uint64_t* coeffB,          \
                                             const uint64_t* src, uint64_t* tgt) {                           \
    arr_map(#P "_arr_mont_mul_by_powers", CURVE, ZKG_FR_MUL_BY_POWERS, n, src, 0, 0, coeffA, coeffB, tgt);    \
  }                                                                                                          \
  extern "C" void P##_arr_mont_sparse_matrix_mul(int N, int K, const uint64_t* row_idxs, const uint64_t* col_idxs, \
                                                 const uint64_t* coeffs, const uint64_t* src, uint64_t* tgt) { \
    const zkg_status s = zkg_fr_sparse_matrix_mul(CURVE, N, K, row_idxs, col_idxs, coeffs, src, tgt);        \
    if (s != ZKG_OK) fail(#P "_arr_mont_sparse_matrix_mul", s, tgt, N > 0 ? (size_t)4 * N : 0, 0);           \
  }                                                                                                          \
  extern "C" void P##_arr_mont_scale(int n, const uint64_t* coeff, const uint64_t* src2, uint64_t* tgt) {    \
    arr_map(#P "_arr_mont_scale", CURVE, ZKG_FR_SCALE, n, src2, 0, 0, coeff, 0, tgt);                         \
  }                                                                                                          \
  extern "C" void P##_arr_mont_scale_inplace(int n, const uint64_t* coeff, uint64_t* tgt) {                  \
    arr_map(#P "_arr_mont_scale_inplace", CURVE, ZKG_FR_SCALE, n, tgt, 0, 0, coeff, 0, tgt);                  \
  }                                                                                                          \
  extern "C" void P##_arr_mont_Ax_plus_y(int n, const uint64_t* coeffA, const uint64_t* src1, const uint64_t* src2, \
                                         uint64_t* tgt) {                                                    \
    arr_map(#P "_arr_mont_Ax_plus_y", CURVE, ZKG_FR_AXPY, n, src1, src2, 0, coeffA, 0, tgt);                  \
  }                                                                                                          \
  extern "C" void P##_arr_mont_Ax_plus_y_inplace(int n, const uint64_t* coeffA, uint64_t* tgt, const uint64_t* src2) { \
    arr_map(#P "_arr_mont_Ax_plus_y_inplace", CURVE, ZKG_FR_AXPY, n, tgt, src2, 0, coeffA, 0, tgt);           \
  }                                                                                                          \
  extern "C" void P##_arr_mont_Ax_plus_By(int n, const uint64_t* coeffA, const uint64_t* coeffB, const uint64_t* src1, \
                                          const uint64_t* src2, uint64_t* tgt) {                             \
    arr_map(#P "_arr_mont_Ax_plus_By", CURVE, ZKG_FR_AXPBY, n, src1, src2, 0, coeffA, coeffB, tgt);           \
  }                                                                                                          \
  extern "C" void P##_arr_mont_Ax_plus_By_inplace(int n, const uint64_t* coeffA, const uint64_t* coeffB, uint64_t* tgt, \
                                                  const uint64_t* src2) {                                    \
    arr_map(#P "_arr_mont_Ax_plus_By_inplace", CURVE, ZKG_FR_AXPBY, n, tgt, src2, 0, coeffA, coeffB, tgt);    \
  }

ZKB_ARR_ENTRIES(bn128, ZKG_BN254, 0)
ZKB_ARR_ENTRIES(bls12_381, ZKG_BLS12_381, 1)
