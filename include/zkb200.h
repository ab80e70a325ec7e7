/*
 * zkb200 -- B200 (sm_100a) implementation of zikkurat-algebra's two data-parallel hot paths:
 * Pippenger multi-scalar multiplication on BN254 / BLS12-381 G1, and the radix-2 NTT over
 * their scalar fields Fr.
 *
 * Part 1 declares the drop-in entry points. They have the exact names, signatures and
 * argument meaning of the reference's generated C (lib/cbits), so the Haskell FFI imports
 * (foreign import ccall unsafe ...) and C callers link against libzkb200.so unchanged.
 * All buffers are caller-owned HOST memory; the call copies inputs to the GPU, computes there
 * and copies the result back before returning. Data layout is the reference's: little-endian
 * 64-bit limbs, Montgomery form (R = 2^256 for BN254 Fp/Fr and BLS12-381 Fr, R = 2^384 for
 * BLS12-381 Fp), affine points x|y with input infinity (0,0).
 *
 * Part 2 is the native C ABI (zkg_*) with status codes, device-pointer variants and
 * helpers. Every entry point is plain C: pointers, sizes, ints. No CUDA or torch types.
 */
#ifndef ZKB200_H
#define ZKB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ============================================================ Part 1: drop-in entry points */

/* MSM: tgt = sum_i expos[i] * grps[i].
 *   npoints     number of points (>= 0)
 *   expos       npoints scalars of expo_nlimbs 64-bit limbs each; "std" = plain integers
 *               (any value, all 64*expo_nlimbs bits are used), "mont" = Montgomery Fr elements
 *               (expo_nlimbs must be 4, as in the reference, which reads 4 limbs per scalar)
 *   grps        npoints affine Montgomery points, 2*NLIMBS_P limbs each (BN254 8, BLS12-381 12)
 *   tgt         proj_out: 3*NLIMBS_P limbs (infinity = (0,1,0));
 *               jac_out: 3*NLIMBS_P limbs (infinity = (1,1,0));
 *               affine_out: 2*NLIMBS_P limbs (infinity = all 0xff bytes).
 * Finite projective / Jacobian results are returned normalised (Z = 1). The reference may
 * return another representative of the same point; equality (normalise, then compare)
 * holds, and affine outputs are bit-identical. */

/* replaces lib/cbits/curves/g1/proj/bn128_G1_proj.c:597  (declared bn128_G1_proj.h:43) */
void bn128_G1_proj_MSM_std_coeff_proj_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bn128_G1_proj.c:631  (bn128_G1_proj.h:44) */
void bn128_G1_proj_MSM_mont_coeff_proj_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bn128_G1_proj.c:656  (bn128_G1_proj.h:46) */
void bn128_G1_proj_MSM_std_coeff_affine_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bn128_G1_proj.c:669  (bn128_G1_proj.h:47) */
void bn128_G1_proj_MSM_mont_coeff_affine_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces lib/cbits/curves/g1/jac/bn128_G1_jac.c:646  (bn128_G1_jac.h:43) */
void bn128_G1_jac_MSM_std_coeff_jac_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bn128_G1_jac.c:680  (bn128_G1_jac.h:44) */
void bn128_G1_jac_MSM_mont_coeff_jac_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bn128_G1_jac.c:705  (bn128_G1_jac.h:46) */
void bn128_G1_jac_MSM_std_coeff_affine_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bn128_G1_jac.c:718  (bn128_G1_jac.h:47) */
void bn128_G1_jac_MSM_mont_coeff_affine_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);

/* replaces lib/cbits/curves/g1/proj/bls12_381_G1_proj.c:598  (bls12_381_G1_proj.h:43) */
void bls12_381_G1_proj_MSM_std_coeff_proj_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bls12_381_G1_proj.c:632  (bls12_381_G1_proj.h:44) */
void bls12_381_G1_proj_MSM_mont_coeff_proj_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bls12_381_G1_proj.c:657  (bls12_381_G1_proj.h:46) */
void bls12_381_G1_proj_MSM_std_coeff_affine_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bls12_381_G1_proj.c:670  (bls12_381_G1_proj.h:47) */
void bls12_381_G1_proj_MSM_mont_coeff_affine_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces lib/cbits/curves/g1/jac/bls12_381_G1_jac.c:646  (bls12_381_G1_jac.h:43) */
void bls12_381_G1_jac_MSM_std_coeff_jac_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bls12_381_G1_jac.c:680  (bls12_381_G1_jac.h:44) */
void bls12_381_G1_jac_MSM_mont_coeff_jac_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bls12_381_G1_jac.c:705  (bls12_381_G1_jac.h:46) */
void bls12_381_G1_jac_MSM_std_coeff_affine_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);
/* replaces bls12_381_G1_jac.c:718  (bls12_381_G1_jac.h:47) */
void bls12_381_G1_jac_MSM_mont_coeff_affine_out(int npoints, const uint64_t *expos, const uint64_t *grps, uint64_t *tgt, int expo_nlimbs);

/* NTT over Fr, natural order in and out, N = 2^m elements of 4 limbs (Montgomery).
 *   forward: tgt[k] = sum_i src[i] * gen^(i*k)       (radix-2 DIT network of the reference)
 *   inverse: tgt = (1/2)^m * DIF network with gen^-1 (for a generator of order 2^m this is
 *            tgt[i] = N^-1 * sum_k src[k] * gen^(-i*k))
 * gen is the Montgomery-form generator of the size-2^m subgroup. src and tgt must not overlap. */
/* replaces lib/cbits/curves/poly/mont/bn128_poly_mont.c:452  (bn128_poly_mont.h:27) */
void bn128_poly_mont_ntt_forward(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_poly_mont.c:601  (bn128_poly_mont.h:28) */
void bn128_poly_mont_ntt_inverse(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces lib/cbits/curves/poly/mont/bls12_381_poly_mont.c:452  (bls12_381_poly_mont.h:27) */
void bls12_381_poly_mont_ntt_forward(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_poly_mont.c:601  (bls12_381_poly_mont.h:28) */
void bls12_381_poly_mont_ntt_inverse(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);

/* Coset NTTs (evaluations of f(eta x); coefficients of f with f(eta^-1 w^k) = src[k]):
 *   forward_shifted: NTT of src[i] * eta^i;  inverse_shifted: inverse NTT, then output i times eta^i.
 * Asymmetric NTT: the size-2^m_src polynomial src evaluated on the size-2^m_tgt subgroup; for
 * k < K = 2^(m_tgt - m_src), tgt[i K + k] = NTT_{gen_src}(src[j] gen_tgt^(k j))[i]. */
/* replaces lib/cbits/curves/poly/mont/bn128_poly_mont.c:477  (bn128_poly_mont.h:30) */
void bn128_poly_mont_ntt_forward_shifted(const uint64_t *eta, int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_poly_mont.c:626  (bn128_poly_mont.h:31) */
void bn128_poly_mont_ntt_inverse_shifted(const uint64_t *eta, int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_poly_mont.c:492  (bn128_poly_mont.h:33) */
void bn128_poly_mont_ntt_forward_asymmetric(int m_src, int m_tgt, const uint64_t *gen_src, const uint64_t *gen_tgt, const uint64_t *src, uint64_t *tgt);
/* replaces lib/cbits/curves/poly/mont/bls12_381_poly_mont.c:477  (bls12_381_poly_mont.h:30) */
void bls12_381_poly_mont_ntt_forward_shifted(const uint64_t *eta, int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_poly_mont.c:626  (bls12_381_poly_mont.h:31) */
void bls12_381_poly_mont_ntt_inverse_shifted(const uint64_t *eta, int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_poly_mont.c:492  (bls12_381_poly_mont.h:33) */
void bls12_381_poly_mont_ntt_forward_asymmetric(int m_src, int m_tgt, const uint64_t *gen_src, const uint64_t *gen_tgt, const uint64_t *src, uint64_t *tgt);

/* Binary MSMs: tgt = sum of the grps[i] whose byte expos[i] is non-zero (any non-zero byte
 * counts as 1, as in the reference). Multi-row form: row r of the nrows x npoints byte matrix
 * (expos[r] points to npoints bytes) gives tgt[r]; tgt holds nrows points of the output kind.
 * Output encodings as for the MSMs above (proj / jac normalised, affine infinity all 0xff). */
/* replaces lib/cbits/curves/g1/proj/bn128_G1_proj.c:684  (bn128_G1_proj.h:45) */
void bn128_G1_proj_MSM_binary_coeff_proj_out(int npoints, const uint8_t *expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bn128_G1_proj.c:694  (bn128_G1_proj.h:48) */
void bn128_G1_proj_MSM_binary_coeff_affine_out(int npoints, const uint8_t *expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bn128_G1_proj.c:718  (bn128_G1_proj.h:52) */
void bn128_G1_proj_multi_MSM_binary_coeff_proj_out(int nrows, int npoints, const uint8_t **expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bn128_G1_proj.c:774  (bn128_G1_proj.h:53) */
void bn128_G1_proj_multi_MSM_binary_coeff_affine_out(int nrows, int npoints, const uint8_t **expos, const uint64_t *grps, uint64_t *tgt);
/* replaces lib/cbits/curves/g1/jac/bn128_G1_jac.c:733  (bn128_G1_jac.h:45) */
void bn128_G1_jac_MSM_binary_coeff_jac_out(int npoints, const uint8_t *expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bn128_G1_jac.c:743  (bn128_G1_jac.h:48) */
void bn128_G1_jac_MSM_binary_coeff_affine_out(int npoints, const uint8_t *expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bn128_G1_jac.c:767  (bn128_G1_jac.h:52) */
void bn128_G1_jac_multi_MSM_binary_coeff_jac_out(int nrows, int npoints, const uint8_t **expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bn128_G1_jac.c:823  (bn128_G1_jac.h:53) */
void bn128_G1_jac_multi_MSM_binary_coeff_affine_out(int nrows, int npoints, const uint8_t **expos, const uint64_t *grps, uint64_t *tgt);
/* replaces lib/cbits/curves/g1/proj/bls12_381_G1_proj.c:685  (bls12_381_G1_proj.h:45) */
void bls12_381_G1_proj_MSM_binary_coeff_proj_out(int npoints, const uint8_t *expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bls12_381_G1_proj.c:695  (bls12_381_G1_proj.h:48) */
void bls12_381_G1_proj_MSM_binary_coeff_affine_out(int npoints, const uint8_t *expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bls12_381_G1_proj.c:719  (bls12_381_G1_proj.h:52) */
void bls12_381_G1_proj_multi_MSM_binary_coeff_proj_out(int nrows, int npoints, const uint8_t **expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bls12_381_G1_proj.c:775  (bls12_381_G1_proj.h:53) */
void bls12_381_G1_proj_multi_MSM_binary_coeff_affine_out(int nrows, int npoints, const uint8_t **expos, const uint64_t *grps, uint64_t *tgt);
/* replaces lib/cbits/curves/g1/jac/bls12_381_G1_jac.c:733  (bls12_381_G1_jac.h:45) */
void bls12_381_G1_jac_MSM_binary_coeff_jac_out(int npoints, const uint8_t *expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bls12_381_G1_jac.c:743  (bls12_381_G1_jac.h:48) */
void bls12_381_G1_jac_MSM_binary_coeff_affine_out(int npoints, const uint8_t *expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bls12_381_G1_jac.c:767  (bls12_381_G1_jac.h:52) */
void bls12_381_G1_jac_multi_MSM_binary_coeff_jac_out(int nrows, int npoints, const uint8_t **expos, const uint64_t *grps, uint64_t *tgt);
/* replaces bls12_381_G1_jac.c:823  (bls12_381_G1_jac.h:53) */
void bls12_381_G1_jac_multi_MSM_binary_coeff_affine_out(int nrows, int npoints, const uint8_t **expos, const uint64_t *grps, uint64_t *tgt);

/* G1 group FFT over N = 2^m points (projective X|Y|Z, x = X/Z, in *_G1_proj_*; Jacobian,
 * x = X/Z^2, y = Y/Z^3, in *_G1_jac_*), infinity Z = 0:
 *   forward: tgt[k] = sum_i [gen^(ik)] src[i]  (the NTT's DIT network with points);
 *   inverse: the DIF network with gen^-1 and (1/2)^m (for gen of order 2^m,
 *            tgt[i] = N^-1 sum_k [gen^(-ik)] src[k]).
 * gen is a Montgomery Fr element. Outputs are normalised as the reference does: (x, y, 1),
 * infinity (0, 1, 0), in both coordinate systems. */
/* replaces lib/cbits/curves/g1/proj/bn128_G1_proj.c:831  (bn128_G1_proj.h:54) */
void bn128_G1_proj_fft_forward(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_G1_proj.c:893  (bn128_G1_proj.h:55) */
void bn128_G1_proj_fft_inverse(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces lib/cbits/curves/g1/jac/bn128_G1_jac.c:880  (bn128_G1_jac.h:54) */
void bn128_G1_jac_fft_forward(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_G1_jac.c:942  (bn128_G1_jac.h:55) */
void bn128_G1_jac_fft_inverse(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces lib/cbits/curves/g1/proj/bls12_381_G1_proj.c:832  (bls12_381_G1_proj.h:54) */
void bls12_381_G1_proj_fft_forward(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_G1_proj.c:894  (bls12_381_G1_proj.h:55) */
void bls12_381_G1_proj_fft_inverse(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces lib/cbits/curves/g1/jac/bls12_381_G1_jac.c:880  (bls12_381_G1_jac.h:54) */
void bls12_381_G1_jac_fft_forward(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_G1_jac.c:942  (bls12_381_G1_jac.h:55) */
void bls12_381_G1_jac_fft_inverse(int m, const uint64_t *gen, const uint64_t *src, uint64_t *tgt);

/* Fr vector operations (*_arr_mont_*): element-wise over n Montgomery Fr elements (4 limbs each),
 * same results as the reference, including its edge behaviour: *_inv / *_div use one batch
 * inversion, so a zero anywhere in the inverted array makes every output zero; *_mul_by_powers
 * leaves tgt[0] unwritten and sets tgt[i] = src[i] * A * B^(i-1) for i >= 1; *_sparse_matrix_mul
 * is declared here though the reference's header omits it (it is defined and bound by the FFI).
 * Copies and constant fills (set_*, copy, append, concat) are plain host memory moves. */
/* replaces lib/cbits/curves/array/mont/bn128_arr_mont.c:26  (bn128_arr_mont.h:3) */
uint8_t bn128_arr_mont_is_valid(int n, const uint64_t *src);
/* replaces bn128_arr_mont.c:34  (bn128_arr_mont.h:4) */
uint8_t bn128_arr_mont_is_zero(int n, const uint64_t *src);
/* replaces bn128_arr_mont.c:43  (bn128_arr_mont.h:5) */
uint8_t bn128_arr_mont_is_one(int n, const uint64_t *src);
/* replaces bn128_arr_mont.c:51  (bn128_arr_mont.h:6) */
uint8_t bn128_arr_mont_is_equal(int n, const uint64_t *src1, const uint64_t *src2);
/* replaces bn128_arr_mont.c:59  (bn128_arr_mont.h:7) */
void bn128_arr_mont_set_zero(int n, uint64_t *tgt);
/* replaces bn128_arr_mont.c:63  (bn128_arr_mont.h:8) */
void bn128_arr_mont_set_one(int n, uint64_t *tgt);
/* replaces bn128_arr_mont.c:67  (bn128_arr_mont.h:9) */
void bn128_arr_mont_set_const(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_arr_mont.c:71  (bn128_arr_mont.h:10) */
void bn128_arr_mont_copy(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_arr_mont.c:94  (bn128_arr_mont.h:12) */
void bn128_arr_mont_from_std(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_arr_mont.c:98  (bn128_arr_mont.h:13) */
void bn128_arr_mont_to_std(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_arr_mont.c:77  (bn128_arr_mont.h:15) */
void bn128_arr_mont_append(int n1, int n2, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bn128_arr_mont.c:85  (bn128_arr_mont.h:16) */
void bn128_arr_mont_concat(int K, int *ns, const uint64_t **srcs, uint64_t *tgt);
/* replaces bn128_arr_mont.c:103  (bn128_arr_mont.h:18) */
void bn128_arr_mont_neg(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_arr_mont.c:107  (bn128_arr_mont.h:19) */
void bn128_arr_mont_add(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bn128_arr_mont.c:111  (bn128_arr_mont.h:20) */
void bn128_arr_mont_sub(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bn128_arr_mont.c:115  (bn128_arr_mont.h:21) */
void bn128_arr_mont_sqr(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_arr_mont.c:119  (bn128_arr_mont.h:22) */
void bn128_arr_mont_mul(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bn128_arr_mont.c:123  (bn128_arr_mont.h:23) */
void bn128_arr_mont_inv(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_arr_mont.c:127  (bn128_arr_mont.h:24) */
void bn128_arr_mont_div(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bn128_arr_mont.c:151  (bn128_arr_mont.h:26) */
void bn128_arr_mont_neg_inplace(int n, uint64_t *tgt);
/* replaces bn128_arr_mont.c:155  (bn128_arr_mont.h:27) */
void bn128_arr_mont_add_inplace(int n, uint64_t *tgt, const uint64_t *src2);
/* replaces bn128_arr_mont.c:159  (bn128_arr_mont.h:28) */
void bn128_arr_mont_sub_inplace(int n, uint64_t *tgt, const uint64_t *src2);
/* replaces bn128_arr_mont.c:167  (bn128_arr_mont.h:29) */
void bn128_arr_mont_sqr_inplace(int n, uint64_t *tgt);
/* replaces bn128_arr_mont.c:171  (bn128_arr_mont.h:30) */
void bn128_arr_mont_mul_inplace(int n, uint64_t *tgt, const uint64_t *src2);
/* replaces bn128_arr_mont.c:175  (bn128_arr_mont.h:31) */
void bn128_arr_mont_inv_inplace(int n, uint64_t *tgt);
/* replaces bn128_arr_mont.c:179  (bn128_arr_mont.h:32) */
void bn128_arr_mont_div_inplace(int n, uint64_t *tgt, const uint64_t *src2);
/* replaces bn128_arr_mont.c:163  (bn128_arr_mont.h:33) */
void bn128_arr_mont_sub_inplace_reverse(int n, uint64_t *tgt, const uint64_t *src1);
/* replaces bn128_arr_mont.c:136  (bn128_arr_mont.h:35) */
void bn128_arr_mont_mul_add(int n, const uint64_t *src1, const uint64_t *src2, const uint64_t *src3, uint64_t *tgt);
/* replaces bn128_arr_mont.c:144  (bn128_arr_mont.h:36) */
void bn128_arr_mont_mul_sub(int n, const uint64_t *src1, const uint64_t *src2, const uint64_t *src3, uint64_t *tgt);
/* replaces bn128_arr_mont.c:187  (bn128_arr_mont.h:38) */
void bn128_arr_mont_dot_prod(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bn128_arr_mont.c:199  (bn128_arr_mont.h:39) */
void bn128_arr_mont_powers(int n, const uint64_t *coeffA, const uint64_t *coeffB, uint64_t *tgt);
/* replaces bn128_arr_mont.c:208  (bn128_arr_mont.h:40) */
void bn128_arr_mont_mul_by_powers(int n, const uint64_t *coeffA, const uint64_t *coeffB, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_arr_mont.c:226  (not in the header) */
void bn128_arr_mont_sparse_matrix_mul(int N, int K, const uint64_t *row_idxs, const uint64_t *col_idxs, const uint64_t *coeffs, const uint64_t *src, uint64_t *tgt);
/* replaces bn128_arr_mont.c:239  (bn128_arr_mont.h:42) */
void bn128_arr_mont_scale(int n, const uint64_t *coeff, const uint64_t *src2, uint64_t *tgt);
/* replaces bn128_arr_mont.c:243  (bn128_arr_mont.h:43) */
void bn128_arr_mont_scale_inplace(int n, const uint64_t *coeff, uint64_t *tgt);
/* replaces bn128_arr_mont.c:247  (bn128_arr_mont.h:45) */
void bn128_arr_mont_Ax_plus_y(int n, const uint64_t *coeffA, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bn128_arr_mont.c:254  (bn128_arr_mont.h:46) */
void bn128_arr_mont_Ax_plus_y_inplace(int n, const uint64_t *coeffA, uint64_t *tgt, const uint64_t *src2);
/* replaces bn128_arr_mont.c:261  (bn128_arr_mont.h:48) */
void bn128_arr_mont_Ax_plus_By(int n, const uint64_t *coeffA, const uint64_t *coeffB, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bn128_arr_mont.c:271  (bn128_arr_mont.h:49) */
void bn128_arr_mont_Ax_plus_By_inplace(int n, const uint64_t *coeffA, const uint64_t *coeffB, uint64_t *tgt, const uint64_t *src2);
/* replaces lib/cbits/curves/array/mont/bls12_381_arr_mont.c:26  (bls12_381_arr_mont.h:3) */
uint8_t bls12_381_arr_mont_is_valid(int n, const uint64_t *src);
/* replaces bls12_381_arr_mont.c:34  (bls12_381_arr_mont.h:4) */
uint8_t bls12_381_arr_mont_is_zero(int n, const uint64_t *src);
/* replaces bls12_381_arr_mont.c:43  (bls12_381_arr_mont.h:5) */
uint8_t bls12_381_arr_mont_is_one(int n, const uint64_t *src);
/* replaces bls12_381_arr_mont.c:51  (bls12_381_arr_mont.h:6) */
uint8_t bls12_381_arr_mont_is_equal(int n, const uint64_t *src1, const uint64_t *src2);
/* replaces bls12_381_arr_mont.c:59  (bls12_381_arr_mont.h:7) */
void bls12_381_arr_mont_set_zero(int n, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:63  (bls12_381_arr_mont.h:8) */
void bls12_381_arr_mont_set_one(int n, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:67  (bls12_381_arr_mont.h:9) */
void bls12_381_arr_mont_set_const(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:71  (bls12_381_arr_mont.h:10) */
void bls12_381_arr_mont_copy(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:94  (bls12_381_arr_mont.h:12) */
void bls12_381_arr_mont_from_std(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:98  (bls12_381_arr_mont.h:13) */
void bls12_381_arr_mont_to_std(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:77  (bls12_381_arr_mont.h:15) */
void bls12_381_arr_mont_append(int n1, int n2, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:85  (bls12_381_arr_mont.h:16) */
void bls12_381_arr_mont_concat(int K, int *ns, const uint64_t **srcs, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:103  (bls12_381_arr_mont.h:18) */
void bls12_381_arr_mont_neg(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:107  (bls12_381_arr_mont.h:19) */
void bls12_381_arr_mont_add(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:111  (bls12_381_arr_mont.h:20) */
void bls12_381_arr_mont_sub(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:115  (bls12_381_arr_mont.h:21) */
void bls12_381_arr_mont_sqr(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:119  (bls12_381_arr_mont.h:22) */
void bls12_381_arr_mont_mul(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:123  (bls12_381_arr_mont.h:23) */
void bls12_381_arr_mont_inv(int n, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:127  (bls12_381_arr_mont.h:24) */
void bls12_381_arr_mont_div(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:151  (bls12_381_arr_mont.h:26) */
void bls12_381_arr_mont_neg_inplace(int n, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:155  (bls12_381_arr_mont.h:27) */
void bls12_381_arr_mont_add_inplace(int n, uint64_t *tgt, const uint64_t *src2);
/* replaces bls12_381_arr_mont.c:159  (bls12_381_arr_mont.h:28) */
void bls12_381_arr_mont_sub_inplace(int n, uint64_t *tgt, const uint64_t *src2);
/* replaces bls12_381_arr_mont.c:167  (bls12_381_arr_mont.h:29) */
void bls12_381_arr_mont_sqr_inplace(int n, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:171  (bls12_381_arr_mont.h:30) */
void bls12_381_arr_mont_mul_inplace(int n, uint64_t *tgt, const uint64_t *src2);
/* replaces bls12_381_arr_mont.c:175  (bls12_381_arr_mont.h:31) */
void bls12_381_arr_mont_inv_inplace(int n, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:179  (bls12_381_arr_mont.h:32) */
void bls12_381_arr_mont_div_inplace(int n, uint64_t *tgt, const uint64_t *src2);
/* replaces bls12_381_arr_mont.c:163  (bls12_381_arr_mont.h:33) */
void bls12_381_arr_mont_sub_inplace_reverse(int n, uint64_t *tgt, const uint64_t *src1);
/* replaces bls12_381_arr_mont.c:136  (bls12_381_arr_mont.h:35) */
void bls12_381_arr_mont_mul_add(int n, const uint64_t *src1, const uint64_t *src2, const uint64_t *src3, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:144  (bls12_381_arr_mont.h:36) */
void bls12_381_arr_mont_mul_sub(int n, const uint64_t *src1, const uint64_t *src2, const uint64_t *src3, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:187  (bls12_381_arr_mont.h:38) */
void bls12_381_arr_mont_dot_prod(int n, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:199  (bls12_381_arr_mont.h:39) */
void bls12_381_arr_mont_powers(int n, const uint64_t *coeffA, const uint64_t *coeffB, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:208  (bls12_381_arr_mont.h:40) */
void bls12_381_arr_mont_mul_by_powers(int n, const uint64_t *coeffA, const uint64_t *coeffB, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:226  (not in the header) */
void bls12_381_arr_mont_sparse_matrix_mul(int N, int K, const uint64_t *row_idxs, const uint64_t *col_idxs, const uint64_t *coeffs, const uint64_t *src, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:239  (bls12_381_arr_mont.h:42) */
void bls12_381_arr_mont_scale(int n, const uint64_t *coeff, const uint64_t *src2, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:243  (bls12_381_arr_mont.h:43) */
void bls12_381_arr_mont_scale_inplace(int n, const uint64_t *coeff, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:247  (bls12_381_arr_mont.h:45) */
void bls12_381_arr_mont_Ax_plus_y(int n, const uint64_t *coeffA, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:254  (bls12_381_arr_mont.h:46) */
void bls12_381_arr_mont_Ax_plus_y_inplace(int n, const uint64_t *coeffA, uint64_t *tgt, const uint64_t *src2);
/* replaces bls12_381_arr_mont.c:261  (bls12_381_arr_mont.h:48) */
void bls12_381_arr_mont_Ax_plus_By(int n, const uint64_t *coeffA, const uint64_t *coeffB, const uint64_t *src1, const uint64_t *src2, uint64_t *tgt);
/* replaces bls12_381_arr_mont.c:271  (bls12_381_arr_mont.h:49) */
void bls12_381_arr_mont_Ax_plus_By_inplace(int n, const uint64_t *coeffA, const uint64_t *coeffB, uint64_t *tgt, const uint64_t *src2);

/* ================================================================ Part 2: native C ABI */

typedef int zkg_status;
#define ZKG_OK               0
#define ZKG_ERR_ARG          1   /* invalid argument (size, limb count, null pointer) */
#define ZKG_ERR_CUDA         2   /* a CUDA runtime call failed (see zkg_last_error) */
#define ZKG_ERR_NOMEM        3   /* device memory could not be reserved */
#define ZKG_ERR_UNSUPPORTED  4   /* argument combination the reference leaves undefined */
#define ZKG_ERR_TIMEOUT      5   /* a wait's deadline passed (the awaited work is still pending) */

typedef int zkg_curve;
#define ZKG_BN254      0
#define ZKG_BLS12_381  1

typedef int zkg_out_kind;
#define ZKG_OUT_PROJ    0
#define ZKG_OUT_JAC     1
#define ZKG_OUT_AFFINE  2

/* MSM on host buffers (what the drop-in entry points call). */
zkg_status zkg_msm(zkg_curve curve, int npoints, const uint64_t *expos, int expo_nlimbs,
                   int expos_mont, const uint64_t *grps, zkg_out_kind kind, uint64_t *tgt);

/* MSM on device-resident inputs (d_expos, d_grps are device pointers); the result is
 * written to the HOST buffer tgt. The call is synchronous. */
zkg_status zkg_msm_device(zkg_curve curve, int npoints, const uint64_t *d_expos, int expo_nlimbs,
                          int expos_mont, const uint64_t *d_grps, zkg_out_kind kind, uint64_t *tgt);

/* NTT on host buffers (what the drop-in entry points call). m in [0, 30], the bound of the
 * reference's `int N = 1 << m` (bn128_poly_mont.c:453; the reference itself aborts from m = 27,
 * where its int buffer size overflows). Any generator. 2^30 points need about 140 GB of device
 * memory with the transform's twiddle table and scratch; a shortfall returns ZKG_ERR_NOMEM. */
zkg_status zkg_ntt(zkg_curve curve, int m, const uint64_t *gen, const uint64_t *src,
                   uint64_t *tgt, int inverse);

/* Shifted (coset) and asymmetric NTTs on host buffers (what the drop-in entry points call). */
zkg_status zkg_ntt_shifted(zkg_curve curve, const uint64_t *eta, int m, const uint64_t *gen, const uint64_t *src,
                           uint64_t *tgt, int inverse);
zkg_status zkg_ntt_asymmetric(zkg_curve curve, int m_src, int m_tgt, const uint64_t *gen_src, const uint64_t *gen_tgt,
                              const uint64_t *src, uint64_t *tgt);

/* NTT on device buffers d_src -> d_tgt (device pointers, non-overlapping); gen is a host
 * pointer to the Montgomery generator. Synchronous. */
zkg_status zkg_ntt_device(zkg_curve curve, int m, const uint64_t *gen, const uint64_t *d_src,
                          uint64_t *d_tgt, int inverse);

/* NTT on device buffers that allocates nothing. No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc, such as code running beside a framework memory pool that
 * owns the device memory, or a host application that gives this library no device-memory quota.
 * Same arguments and results as zkg_ntt_device, with m <= 16 (larger m is rejected with
 * ZKG_ERR_ARG). All scratch lives in one fixed 4 MiB + 24 KiB array in the library's device
 * image, which every GPU that loads the library holds until the process exits. Calls share the
 * array and are serialised. Every call synchronises the whole device (it waits for all earlier
 * device work before it starts, copies its tables with blocking copies and waits for its own
 * kernels before it returns), so it must not be called while any stream capture is active in
 * the process. */
zkg_status zkg_ntt_device_noalloc(zkg_curve curve, int m, const uint64_t *gen, const uint64_t *d_src,
                                  uint64_t *d_tgt, int inverse);

/* Element-wise field arithmetic on device buffers of n elements (the reference's Montgomery form,
 * fully reduced; 4 or 6 limbs), for direct tests of the arithmetic every kernel is built on.
 * field: 0 = Fp, 1 = Fr. path: 0 = 32-bit-limb products, 1 = FP64-pipe products (operands moved
 * into that product's radix and back with the same exact conversions the MSM and NTT use),
 * 2 (Fp only) = the MSM bucket pipeline's redundant range [0, 2p) with FP64 products (operands
 * at odd indices of a and at indices 2, 3 mod 4 of b are taken as x + p; results made canonical,
 * all-ones words if a result left [0, 2p)), 3 = FP64-pipe products in the reference's own radix
 * (no conversions; op 5 not available).
 * op: 0 mul (bn128_Fp_mont.c:189, bls12_381_Fp_mont.c:203, Fr twins), 1 sqr, 2 add, 3 sub,
 * 4 neg, 5 raw FP64 product a b 2^-(52 L) (path ignored), 6 / 7 first / second product of a
 * paired call (a b and b a), 8 first square of a paired square call. d_b may be null for
 * 1 and 4. Synchronous. */
zkg_status zkg_field_test_device(zkg_curve curve, int field, int path, int op, int n, const uint64_t *d_a,
                                 const uint64_t *d_b, uint64_t *d_out);

/* Device-side generation of affine points k_i * G (G the curve's G1 generator) for
 * standard-form scalars k_i (4 limbs each); output in the affine Montgomery layout.
 * Infinity (k_i = 0 mod r) is written as (0,0). For building test and benchmark inputs. */
zkg_status zkg_g1_gen_mul_device(zkg_curve curve, int n, const uint64_t *d_scalars_std,
                                 uint64_t *d_out_affine);

/* ------------------------------------------------------------------- G1 group FFT, binary MSMs
 * zkg_g1_fft: host buffers of 2^m points (3 * NLIMBS_P limbs each, projective when jac == 0,
 * Jacobian otherwise), gen a Montgomery Fr element (host pointer); outputs normalised
 * projective / Jacobian (same bytes). m in [0, 26]. src and tgt may be the same buffer.
 * zkg_g1_fft_device: the same on device buffers (16-byte aligned).
 * zkg_msm_binary: nrows binary MSMs over one base set; rows[r] points to npoints host bytes;
 * out receives nrows points of out_kind. zkg_msm_binary_device: device coefficient matrix,
 * row r at d_coeffs + r * ld (ld >= npoints), device bases and output. */
zkg_status zkg_g1_fft(zkg_curve curve, int jac, int m, const uint64_t *gen, const uint64_t *src,
                      uint64_t *tgt, int inverse);
zkg_status zkg_g1_fft_device(zkg_curve curve, int jac, int m, const uint64_t *gen, const uint64_t *d_src,
                             uint64_t *d_tgt, int inverse);
zkg_status zkg_msm_binary(zkg_curve curve, zkg_out_kind out_kind, int nrows, int npoints,
                          const uint8_t *const *rows, const uint64_t *bases, uint64_t *out);
zkg_status zkg_msm_binary_device(zkg_curve curve, zkg_out_kind out_kind, int nrows, int npoints,
                                 const uint8_t *d_coeffs, size_t ld, const uint64_t *d_bases, uint64_t *d_out);

/* ------------------------------------------------------------------- Fr vector operations
 * zkg_fr_map computes out[i] = op(a[i], b[i], c[i]; A, B) on host buffers of n Montgomery Fr
 * elements; zkg_fr_map_device on device buffers (16-byte aligned; in-place use allowed). A and B
 * (coeff_a, coeff_b) are single host elements. Operations (the inputs each reads):
 *   FROM_STD a*R, TO_STD a/R, NEG -a, SQR a^2, INV batch 1/a (all zero if some a[i] = 0)  [a]
 *   ADD a+b, SUB a-b, MUL a*b, DIV a * batch 1/b                                          [a, b]
 *   MUL_ADD a*b+c, MUL_SUB a*b-c                                                          [a, b, c]
 *   SCALE A*a [a, A]; AXPY A*a+b [a, b, A]; AXPBY A*a+B*b [a, b, A, B]
 *   POWERS A*B^i [A, B]; MUL_BY_POWERS out[i] = a[i]*A*B^(i-1) for i >= 1, out[0] kept [a, A, B]
 * zkg_fr_dot: sum a[i]*b[i] into out (4 host limbs). zkg_fr_predicate: which = 0 all valid (< r),
 * 1 all zero, 2 all one, 3 a == b; *result = 1 or 0. zkg_fr_sparse_matrix_mul: tgt (N elements)
 * = A*src for the K non-zeros (row, col, coeff); the device form takes the length M of src. */
#define ZKG_FR_FROM_STD       0
#define ZKG_FR_TO_STD         1
#define ZKG_FR_NEG            2
#define ZKG_FR_ADD            3
#define ZKG_FR_SUB            4
#define ZKG_FR_SQR            5
#define ZKG_FR_MUL            6
#define ZKG_FR_INV            7
#define ZKG_FR_DIV            8
#define ZKG_FR_MUL_ADD        9
#define ZKG_FR_MUL_SUB        10
#define ZKG_FR_SCALE          11
#define ZKG_FR_AXPY           12
#define ZKG_FR_AXPBY          13
#define ZKG_FR_POWERS         14
#define ZKG_FR_MUL_BY_POWERS  15
zkg_status zkg_fr_map(zkg_curve curve, int op, int n, const uint64_t *a, const uint64_t *b, const uint64_t *c,
                      const uint64_t *coeff_a, const uint64_t *coeff_b, uint64_t *out);
zkg_status zkg_fr_map_device(zkg_curve curve, int op, int n, const uint64_t *d_a, const uint64_t *d_b,
                             const uint64_t *d_c, const uint64_t *coeff_a, const uint64_t *coeff_b, uint64_t *d_out);
zkg_status zkg_fr_dot(zkg_curve curve, int n, const uint64_t *a, const uint64_t *b, uint64_t *out);
zkg_status zkg_fr_dot_device(zkg_curve curve, int n, const uint64_t *d_a, const uint64_t *d_b, uint64_t *out);
zkg_status zkg_fr_predicate(zkg_curve curve, int which, int n, const uint64_t *a, const uint64_t *b, int *result);
zkg_status zkg_fr_predicate_device(zkg_curve curve, int which, int n, const uint64_t *d_a, const uint64_t *d_b,
                                   int *result);
zkg_status zkg_fr_sparse_matrix_mul(zkg_curve curve, int N, int K, const uint64_t *rows, const uint64_t *cols,
                                    const uint64_t *coeffs, const uint64_t *src, uint64_t *tgt);
zkg_status zkg_fr_sparse_matrix_mul_device(zkg_curve curve, int N, int K, const uint64_t *d_rows,
                                           const uint64_t *d_cols, const uint64_t *d_coeffs, const uint64_t *d_src,
                                           int M, uint64_t *d_tgt);

/* ------------------------------------------------------------------ resident base set
 * A base set (the SRS-like points every MSM of a prover reuses: examples/KZG.hs:80 takes
 * prefixes of one set) uploaded to the device once and kept there in the form the MSM pipeline
 * reads. zkg_bases_upload copies n affine
 * Montgomery points from host memory (on_device = 0, pageable or page-locked) or from a device
 * buffer (on_device = 1); the handle owns its copy. zkg_msm_resident runs an MSM over the first
 * npoints bases with device-resident scalars, zkg_msm_resident_host with host scalars (copied
 * each call); both take the arguments and give the results of zkg_msm_device / zkg_msm.
 * zkg_batch_create_resident and zkg_server_create_resident build a batch / commit server on the
 * set, so neither copies nor converts bases again. The handle must outlive its batches and
 * servers. */
typedef struct zkg_bases zkg_bases;
zkg_status zkg_bases_upload(zkg_curve curve, const uint64_t *bases, int n, int on_device, zkg_bases **out);
zkg_status zkg_bases_destroy(zkg_bases *h);
int zkg_bases_count(const zkg_bases *h);
zkg_status zkg_msm_resident(zkg_bases *h, int npoints, const uint64_t *d_expos, int expo_nlimbs, int expos_mont,
                            zkg_out_kind kind, uint64_t *tgt);
zkg_status zkg_msm_resident_host(zkg_bases *h, int npoints, const uint64_t *expos, int expo_nlimbs,
                                 int expos_mont, zkg_out_kind kind, uint64_t *tgt);

/* ------------------------------------------------------------------- batched mode
 * Many MSMs (against prefixes of one device-resident base set: request i uses bases[0, n_i),
 * the KZG pattern of committing polynomials of several degrees) and NTTs of uneven sizes run as
 * one CUDA graph. The MSMs share one segmented pipeline (each with its own window width). Two
 * forms, with the same results: graph branches (the default, measured faster on B200), where the
 * NTTs run on parallel streams beside the MSM pipeline; and the persistent form
 * (zkg_batch_set_mode(b, 1) or ZKB_BATCH_PERSISTENT=1), where the bulk of the work runs in ONE
 * persistent kernel whose CTAs drain a device work queue holding every MSM's share of the bucket
 * accumulation and every tile of every NTT pass (a pass's tiles wait, with a bounded spin, until
 * the pass before is complete). The first zkg_batch_run builds the plan and captures the graph;
 * later runs replay it on the same (device) input and output buffers, whose contents may change
 * between runs. MSM results (affine, host memory) are written when zkg_batch_run returns. The
 * 32-bit-product pipelines always use graph branches.
 * zkg_batch_set_wait_limit (before the first run): polls a pass waits for the one before it
 * (default 2^24, about 2 s) before the run fails with ZKG_ERR_TIMEOUT; inject_stall != 0 makes
 * one pass wait for a tile that never comes (tests of that path). zkg_batch_persistent reports
 * whether the batch runs the persistent kernel (1), its grid and its number of tasks. */
typedef struct zkg_batch zkg_batch;
zkg_status zkg_batch_create(zkg_curve curve, const uint64_t *d_bases, int n_bases, zkg_batch **out);
zkg_status zkg_batch_create_resident(zkg_bases *h, zkg_batch **out);
zkg_status zkg_batch_add_msm(zkg_batch *b, int n, const uint64_t *d_scalars_mont, uint64_t *out_affine);
zkg_status zkg_batch_add_ntt(zkg_batch *b, int m, const uint64_t *gen, const uint64_t *d_src, uint64_t *d_tgt,
                             int inverse);
zkg_status zkg_batch_run(zkg_batch *b);
/* device time (ms) of the last zkg_batch_run's graph */
float zkg_batch_last_ms(const zkg_batch *b);
zkg_status zkg_batch_set_wait_limit(zkg_batch *b, uint32_t polls, int inject_stall);
int zkg_batch_persistent(const zkg_batch *b, int *grid, uint32_t *tasks);
/* before the first run: 1 = persistent kernel, 0 = NTTs as parallel graph branches beside the MSM
 * pipeline (the default); results are the same */
zkg_status zkg_batch_set_mode(zkg_batch *b, int persistent);
zkg_status zkg_batch_destroy(zkg_batch *b);

/* -------------------------------------------------------------------- served mode
 * A commit server: each request is the KZG commit of 2^k evaluations (inverse NTT on the size-2^k
 * subgroup, then MSM of the Montgomery coefficients against bases[0, 2^k) of a resident base set).
 * Whenever one of `slots` streams is free, the oldest pending request whose device memory fits
 * into `hbm_budget` bytes is admitted (a request can be overtaken by younger ones at most 16
 * times, then it is admitted next); admitted requests overlap on the GPU and a request is
 * finished as soon as its own stream completes (continuous batching). `values` (host, pinned for
 * asynchronous copies) and `out_affine` must stay valid until zkg_server_wait returns. Latency
 * is measured from zkg_server_submit to completion.
 * After a failure every pending ticket completes with the error status (no wait blocks forever),
 * requests already running finish, and new submissions return the error.
 * zkg_server_wait_for waits at most timeout_ms (< 0: no limit) and returns ZKG_ERR_TIMEOUT if the
 * request is still pending (the ticket stays valid). zkg_server_inject_failure makes the
 * admission `admission` places from now fail on the host as a launch error would (testing of the
 * failure path; < 0 disarms it). */
typedef struct zkg_server zkg_server;
zkg_status zkg_server_create(zkg_curve curve, const uint64_t *d_bases, int n_bases, int k_min, int k_max,
                             size_t hbm_budget, int slots, zkg_server **out);
zkg_status zkg_server_create_resident(zkg_bases *h, int k_min, int k_max, size_t hbm_budget, int slots,
                                      zkg_server **out);
zkg_status zkg_server_submit(zkg_server *s, int k, const uint64_t *values, uint64_t *out_affine, uint64_t *ticket);
zkg_status zkg_server_wait(zkg_server *s, uint64_t ticket, double *latency_ms);
zkg_status zkg_server_wait_for(zkg_server *s, uint64_t ticket, double timeout_ms, double *latency_ms);
zkg_status zkg_server_inject_failure(zkg_server *s, long admission);
zkg_status zkg_server_stats(zkg_server *s, uint64_t *completed, int *max_inflight, size_t *peak_bytes);
zkg_status zkg_server_destroy(zkg_server *s);

/* ------------------------------------------------------------------------ autotuner
 * zkg_autotune_msm tunes the MSM for every n = 2^L, L in [log_min, log_max], on the given
 * device-resident bases (random scalars): the window width around the cost model's choice, then
 * the accumulation chunk length, the running-sum group size and the prefetch depth (coordinate
 * search, each setting timed on the device). chosen[L - log_min] receives the window width (may
 * be NULL); zkg_msm_tuned_config reports all four settings of a size (0 / -1 = default rule;
 * returns 1 when the size is tuned, 0 when not, -1 on bad arguments).
 * zkg_autotune_ntt times the NTT's largest pass size (6..11) per m.
 * Tuned settings apply to every later call of the process on that curve and size, the drop-in
 * entry points included. With the environment variable ZKG_TUNE_CACHE naming a file they are
 * also written there and read back by later processes on a GPU with the same SM count. Results
 * never depend on tuning. */
zkg_status zkg_autotune_msm(zkg_curve curve, const uint64_t *d_bases, int n_bases, int log_min, int log_max,
                            int *chosen);
int zkg_msm_tuned_window(zkg_curve curve, int log_n);
int zkg_msm_tuned_config(zkg_curve curve, int log_n, int *c, int *chunk_len, int *group, int *prefetch);
zkg_status zkg_autotune_ntt(zkg_curve curve, int m_min, int m_max, int *chosen);

/* MSM window width override (0 = automatic choice by size). Returns the previous value. */
int zkg_set_msm_window(int c);
/* Number of point-range parts (1..4, 0 = automatic) a host-buffer MSM is split into so that
 * copies overlap computation. Returns the previous value. Results do not depend on it. */
int zkg_set_msm_parts(int parts);
/* Affine tree levels of the bucket accumulation (0 = none, -1 = automatic by size) and the output
 * slots per tree thread (its simultaneous-inversion batch; 0 keeps the current value, -1 returns
 * to the automatic choice, >= 4 otherwise). Returns the previous level setting. Results do not
 * depend on either. */
int zkg_set_msm_tree(int levels, int slots_per_thread);
/* Window width the automatic rule picks for a curve and size. */
int zkg_msm_window_for(zkg_curve curve, int npoints);
/* Largest NTT pass (log2 of the per-pass network size, 1..11; default 8; 0 = back to the
 * default and the autotuner's per-size choices). Returns the previous value. Results do not
 * depend on it. */
int zkg_set_ntt_kmax(int k);

zkg_status zkg_last_status(void);
const char *zkg_last_error(void);
/* Device time in milliseconds of the compute kernels of the last MSM, NTT or Fr element-wise
 * (zkg_fr_map*) call. */
float zkg_last_kernel_ms(void);
/* Number of kernels the library launched since load (all calls). */
uint64_t zkg_kernel_launches(void);
/* Releases cached device memory and plans of the current device. */
zkg_status zkg_release_cache(void);
/* Compute stream for subsequent calls on the current device: a cudaStream_t passed as an opaque
 * pointer (NULL = the library's own stream). With a caller stream, device-pointer calls do not
 * synchronise the whole device first; inputs must be ready on that stream. */
zkg_status zkg_set_stream(void *stream);
/* Device time (ms) of the phases of the last MSM: sort, level-1 accumulation, folding levels,
 * bucket reduction. Returns the number of values written (<= max). */
int zkg_last_phase_ms(float *out, int max);
/* Measured 32-bit multiply-add (IMAD) throughput of the current device, instructions per second
 * (independent mad.lo.u32 chains on every SM): the denominator of the MSM/NTT roofline. */
double zkg_imad_probe(void);
/* Measured issue rate (instructions per second, whole device) of one instruction kind in
 * independent dependency chains: 0 mad.lo.u32, 1 mad.hi.u32, 2 mad.wide.u32, 3 fma.rn.f64. */
double zkg_pipe_probe(int kind);
/* Measured throughput (products per second, whole device) of the MSM bucket pipeline's Fp
 * product (exact-radix FP64 product on the redundant range, in pairs as the point formulas call
 * it) in independent chains: the ceiling of the bucket accumulation, whose work is these products. */
double zkg_product_probe(zkg_curve curve);
/* Window width, window count and number of bucket mixed additions of the last MSM. */
int zkg_msm_last_info(int *c, int *nwin, uint64_t *additions);

#ifdef __cplusplus
}
#endif

#endif /* ZKB200_H */
