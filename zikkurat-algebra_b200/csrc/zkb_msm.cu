// Pippenger MSM on G1 for BN254 and BLS12-381, B200 (sm_100a).
//
// Reference: lib/cbits/curves/g1/proj/bn128_G1_proj.c:506-586 (unsigned c-bit windows over all
// 64*expo_nlimbs scalar bits, one bucket array per window filled by mixed additions, running
// sum, c doublings per window) and the Montgomery / affine / Jacobian wrappers :597-673,
// lib/cbits/curves/g1/jac/bn128_G1_jac.c:646-720. The sum computed is the same group element;
// the schedule is the GPU's:
//
//   1. digits+hist   per point (Montgomery scalars converted to standard form in registers):
//                    signed c-bit digits (buckets 1..2^(c-1), sign folded into the point),
//                    per-(window,bucket) counts by atomics; each digit and the value its count
//                    increment returned (its rank in the segment) are stored window-major
//   2. scan          exclusive prefix sum of the counts -> one segment per (window, bucket)
//   3. scatter       point indices (+ sign bit) placed at segment offset + rank, window after
//                    window, no atomics
//   4. affine tree   (BLS12-381, long segments) the first levels as affine pair sums with one
//                    simultaneous inversion per level (zkb_msm_tree.cuh)
//   5. accumulate    equal-length chunks of the segmented array, one chunk per thread:
//                    mixed additions of affine bases (the next one prefetched into shared
//                    memory by cp.async) into an XYZZ accumulator, products on the FP64 pipe
//                    (zkb_dpf.cuh). Complete segments go straight to the bucket array;
//                    segments cut by a chunk boundary leave partial sums in slots.
//   6. merge, fold   a segment cut across at most 9 chunks is summed from its slots by one
//                    thread (nearly every cut segment at large n spans two); longer ones are
//                    folded by levels, again in equal chunks, so any digit distribution is
//                    load balanced.
//   7. bucket reduce (the point-range parts of a host-buffer MSM summed first, in one parallel
//                    pass) per (window, group of K buckets) running sums (T_g, R_g), then per
//                    window the plain sums U_R = sum R_g and U_k = sum_{g: bit k of g} T_g,
//                    so that sum_b b*S_b = U_R + K * sum_k 2^k U_k needs no doublings on
//                    the GPU
//   8. host tail     Horner over windows and bits, normalisation, output encoding.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>
#include <vector>

#include "zkb_curve.cuh"
#include "zkb_dpf.cuh"
#include "zkb_host_ec.h"
#include "zkb_ntt.h"
#include "zkb_batch_work.h"
#include "zkb_msm_accum.cuh"
#include "zkb_msm_tree.cuh"
#include "zkb_runtime.h"

namespace zkb {

static constexpr int MAX_LEVELS = 12;
static constexpr int MAX_TREE = 8;   // affine tree levels (zkb_msm_tree.cuh)

struct LevelHist {
  int n;
  uint32_t L[MAX_LEVELS];
};

// ------------------------------------------------------------------------ scalar handling

// Montgomery Fr scalars (4 limbs) -> standard form (the reference's to_std per scalar,
// bn128_G1_proj.c:638-642)
template <class C>
__global__ void k_msm_scalar_from_mont(int n, const uint64_t* __restrict__ in, uint32_t* __restrict__ out) {
  using Fr = typename C::Fr;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Fe<Fr> a = fe_load_nc<Fr>(reinterpret_cast<const uint32_t*>(in) + 8 * (size_t)i);
  fe_store<Fr>(out + 8 * (size_t)i, fe_from_mont(a));
}

// c bits of a scalar (nw 32-bit words) starting at bit `bit`; bits past the end read as 0
__device__ __forceinline__ uint32_t scalar_bits(const uint32_t* __restrict__ w, int nw, int bit, int c) {
  const int wi = bit >> 5, sh = bit & 31;
  const uint64_t lo = wi < nw ? __ldg(w + wi) : 0u;
  const uint64_t hi = wi + 1 < nw ? __ldg(w + wi + 1) : 0u;
  return (uint32_t)(((lo | (hi << 32)) >> sh) & ((1ull << c) - 1));
}

// signed digit for window `win` given the running carry; returns bucket (0 = none)
__device__ __forceinline__ uint32_t next_digit(const uint32_t* w, int nw, int win, int c,
                                               uint32_t& carry, uint32_t& neg) {
  const uint32_t raw = scalar_bits(w, nw, win * c, c) + carry;
  const uint32_t half = 1u << (c - 1);
  if (raw > half) {
    carry = 1;
    neg = 1;
    return (1u << c) - raw;
  }
  carry = 0;
  neg = 0;
  return raw;
}

// dig (optional): every (window, point) digit, window-major, as bucket | sign << 31 (bucket 0 = no
// entry), for k_msm_scatter_d
// rank (with dig): the entry's position within its (window, bucket) segment, the value its count
// increment returned, so the scatter needs no atomics
__global__ void k_msm_hist(int n, const uint32_t* __restrict__ scal, int nw, int c, int nwin,
                           uint32_t B, uint32_t* __restrict__ cnt, uint32_t* chk = nullptr,
                           uint32_t* __restrict__ dig = nullptr, uint32_t* __restrict__ rank = nullptr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* w = scal + (size_t)nw * i;
  uint32_t carry = 0, neg;
  for (int win = 0; win < nwin; win++) {
    uint32_t b = next_digit(w, nw, win, c, carry, neg);
    if (chk && b > B) { atomicOr(chk, 1u); b = 0; }
    if (dig) {
      dig[(size_t)win * n + i] = b | (b ? neg << 31 : 0u);
      if (b) rank[(size_t)win * n + i] = atomicAdd(cnt + (size_t)win * B + (b - 1), 1u);
    } else if (b) {
      atomicAdd(cnt + (size_t)win * B + (b - 1), 1u);
    }
  }
}

// The histogram for Montgomery Fr scalars with stored digits: each thread converts its scalar to
// standard form in registers (the reference's to_std, bn128_G1_proj.c:638-642), so no standard
// copy of the scalars is written or read back.
template <class C>
__global__ void k_msm_hist_mont(int n, const uint64_t* __restrict__ in, int c, int nwin, uint32_t B,
                                uint32_t* __restrict__ cnt, uint32_t* chk, uint32_t* __restrict__ dig,
                                uint32_t* __restrict__ rank) {
  using Fr = typename C::Fr;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Fe<Fr> sv = fe_from_mont(fe_load_nc<Fr>(reinterpret_cast<const uint32_t*>(in) + 8 * (size_t)i));
  uint32_t carry = 0;
  const uint32_t half = 1u << (c - 1);
  for (int win = 0; win < nwin; win++) {
    const int bit = win * c, wi = bit >> 5, sh = bit & 31;
    uint64_t pair = 0;   // words wi, wi + 1 of the scalar (past the end: 0)
#pragma unroll
    for (int k = 0; k < 8; k++) {
      if (k == wi) pair |= sv.v[k];
      if (k == wi + 1) pair |= (uint64_t)sv.v[k] << 32;
    }
    const uint32_t raw = (uint32_t)((pair >> sh) & ((1ull << c) - 1)) + carry;
    const uint32_t neg = raw > half ? 1u : 0u;
    carry = neg;
    uint32_t b = neg ? (1u << c) - raw : raw;
    if (chk && b > B) { atomicOr(chk, 1u); b = 0; }
    dig[(size_t)win * n + i] = b | (b ? neg << 31 : 0u);
    if (b) rank[(size_t)win * n + i] = atomicAdd(cnt + (size_t)win * B + (b - 1), 1u);
  }
}

// Window-major scatter from the stored digits and ranks (grid y = window): coalesced 4-byte reads
// per (window, point), the entry's position = its segment's offset + its rank, no atomics
__global__ void k_msm_scatter_d(int n, const uint32_t* __restrict__ dig, const uint32_t* __restrict__ rank,
                                uint32_t B, const uint32_t* __restrict__ off, uint32_t* __restrict__ entries,
                                uint32_t* chk, uint32_t total) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int win = blockIdx.y;
  if (i >= n) return;
  const uint32_t v = __ldg(dig + (size_t)win * n + i);
  const uint32_t b = v & 0x7fffffffu;
  if (b) {
    const uint32_t pos = __ldg(off + (size_t)win * B + (b - 1)) + __ldg(rank + (size_t)win * n + i);
    if (chk && pos >= total) { atomicOr(chk, CHK_ENTRY); return; }
    entries[pos] = (uint32_t)i | (v & 0x80000000u);
  }
}

__global__ void k_msm_scatter(int n, const uint32_t* __restrict__ scal, int nw, int c, int nwin,
                              uint32_t B, uint32_t* __restrict__ cursor, uint32_t* __restrict__ entries) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* w = scal + (size_t)nw * i;
  uint32_t carry = 0, neg;
  for (int win = 0; win < nwin; win++) {
    const uint32_t b = next_digit(w, nw, win, c, carry, neg);
    if (b) {
      const uint32_t pos = atomicAdd(cursor + (size_t)win * B + (b - 1), 1u);
      entries[pos] = (uint32_t)i | (neg << 31);
    }
  }
}

// Window-major digits. The carry into window w of the signed recoding above is a function of the
// scalar's low w*c bits alone: with digits in (-2^(c-1), 2^(c-1)], the digits of windows below
// w represent exactly the values in (-H_w + S_w - 2^(wc), H_w] with H_w = sum_{j<w} 2^(jc + c - 1)
// and S_w = sum_{j<w} 2^(jc), so carry_w = [ (s mod 2^(wc)) > H_w ]. Each (window, point) digit is
// then computed on its own, and the histogram and scatter run one window after another (grid y =
// window): a window's 4-byte entries (n * 4 bytes) stay in L2 until their sectors are complete,
// instead of all windows' entries being written at random over the whole array.
static constexpr int HT_WORDS = 480;   // H_w tables up to nwin * nw words
struct CarryTable {
  uint32_t h[HT_WORDS];   // word k of H_w at [w * nw + k]
};

__device__ __forceinline__ uint32_t carry_into(const uint32_t* __restrict__ w, int nw, int win, int c,
                                               const uint32_t* __restrict__ H) {
  const int bits = win * c;
  if (bits == 0) return 0;
  const int top = min((bits - 1) >> 5, nw - 1);
  for (int k = top; k >= 0; k--) {
    uint32_t sw = __ldg(w + k);
    if (k == ((bits - 1) >> 5) && (bits & 31)) sw &= (1u << (bits & 31)) - 1u;
    const uint32_t hw = H[k];
    if (sw != hw) return sw > hw ? 1u : 0u;
  }
  return 0;
}

__device__ __forceinline__ uint32_t digit_at(const uint32_t* __restrict__ w, int nw, int win, int c,
                                             const CarryTable& T, uint32_t& neg) {
  const uint32_t raw = scalar_bits(w, nw, win * c, c) + carry_into(w, nw, win, c, T.h + win * nw);
  const uint32_t half = 1u << (c - 1);
  neg = raw > half ? 1u : 0u;
  return neg ? (1u << c) - raw : raw;
}

// chk (device bounds checks, null = off): bucket b in [1, B], scatter position below `total`
__global__ void k_msm_hist_w(int n, const uint32_t* __restrict__ scal, int nw, int c, uint32_t B, const CarryTable T,
                             uint32_t* __restrict__ cnt, uint32_t* chk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int win = blockIdx.y;
  if (i >= n) return;
  uint32_t neg;
  const uint32_t b = digit_at(scal + (size_t)nw * i, nw, win, c, T, neg);
  if (chk && b > B) { atomicOr(chk, CHK_BUCKET); return; }
  if (b) atomicAdd(cnt + (size_t)win * B + (b - 1), 1u);
}

__global__ void k_msm_scatter_w(int n, const uint32_t* __restrict__ scal, int nw, int c, uint32_t B, const CarryTable T,
                                uint32_t* __restrict__ cursor, uint32_t* __restrict__ entries, uint32_t* chk,
                                uint32_t total) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int win = blockIdx.y;
  if (i >= n) return;
  uint32_t neg;
  const uint32_t b = digit_at(scal + (size_t)nw * i, nw, win, c, T, neg);
  if (chk && b > B) { atomicOr(chk, CHK_BUCKET); return; }
  if (b) {
    const uint32_t pos = atomicAdd(cursor + (size_t)win * B + (b - 1), 1u);
    if (chk && pos >= total) { atomicOr(chk, CHK_ENTRY); return; }
    entries[pos] = (uint32_t)i | (neg << 31);
  }
}

// H_w for every window (host side); false when the table does not fit CarryTable
static bool make_carry_table(int nwin, int nw, int c, CarryTable& T) {
  if ((size_t)nwin * nw > (size_t)HT_WORDS) return false;
  std::memset(T.h, 0, sizeof(T.h));
  for (int w = 0; w < nwin; w++)
    for (int j = 0; j < w; j++) {
      const int bit = j * c + c - 1;
      if ((bit >> 5) < nw) T.h[w * nw + (bit >> 5)] |= 1u << (bit & 31);
    }
  return true;
}

// --------------------------------------------------------------------------------- scan
// Exclusive prefix sum of n u32 counts in three launches (blocks of 4096 elements).
static constexpr int SCAN_T = 1024, SCAN_E = 4;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sm_warp, uint32_t& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) sm_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < (int)(blockDim.x >> 5) ? sm_warp[lane] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, d);
      if (lane >= d) s += y;
    }
    sm_warp[lane] = s;   // inclusive warp-prefix
  }
  __syncthreads();
  total = sm_warp[(blockDim.x >> 5) - 1];
  const uint32_t before = wid ? sm_warp[wid - 1] : 0u;
  return before + x - v;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_blocks(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                        uint32_t* __restrict__ bsums, uint32_t n) {
  __shared__ uint32_t smw[32];
  const size_t base = (size_t)blockIdx.x * SCAN_T * SCAN_E + (size_t)threadIdx.x * SCAN_E;
  uint32_t v[SCAN_E], s = 0;
#pragma unroll
  for (int e = 0; e < SCAN_E; e++) {
    v[e] = (base + e < n) ? in[base + e] : 0u;
    s += v[e];
  }
  uint32_t total;
  uint32_t pre = block_excl_scan(s, smw, total);
#pragma unroll
  for (int e = 0; e < SCAN_E; e++) {
    if (base + e < n) out[base + e] = pre;
    pre += v[e];
  }
  if (threadIdx.x == 0) bsums[blockIdx.x] = total;
}

// single block: exclusive scan of up to SCAN_T*SCAN_E block totals; bsums[nb] = grand total
__global__ void __launch_bounds__(SCAN_T) k_scan_top(uint32_t* __restrict__ bsums, uint32_t nb) {
  __shared__ uint32_t smw[32];
  const uint32_t base = threadIdx.x * SCAN_E;
  uint32_t v[SCAN_E], s = 0;
#pragma unroll
  for (int e = 0; e < SCAN_E; e++) {
    v[e] = (base + e < nb) ? bsums[base + e] : 0u;
    s += v[e];
  }
  uint32_t total;
  uint32_t pre = block_excl_scan(s, smw, total);
#pragma unroll
  for (int e = 0; e < SCAN_E; e++) {
    if (base + e < nb) bsums[base + e] = pre;
    pre += v[e];
  }
  if (threadIdx.x == 0) bsums[nb] = total;
}

__global__ void k_scan_add(uint32_t* __restrict__ out, uint32_t* __restrict__ cursor,
                           const uint32_t* __restrict__ bsums, uint32_t n, uint32_t nb) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const uint32_t v = out[i] + bsums[i / (SCAN_T * SCAN_E)];
    out[i] = v;
    cursor[i] = v;
  }
  if (i == 0) out[n] = bsums[nb];
}

// ------------------------------------------------------------------ bucket accumulation
// (accum_block and its helpers: zkb_msm_accum.cuh)

template <class C, int PF, int NT = 256, int MINB = (C::ID == 0 ? 2 : 1)>
__global__ void __launch_bounds__(NT, MINB) k_msm_accum(const uint32_t* __restrict__ entries,
                                                   const uint32_t* __restrict__ off, uint32_t nseg,
                                                   uint32_t nchunks, uint32_t L, const uint32_t* __restrict__ bases,
                                                   uint32_t* __restrict__ bsum, uint32_t* __restrict__ skey,
                                                   uint32_t* __restrict__ spt, uint32_t* chk, uint32_t npts) {
  // PF > 0: the next PF - 1 bases are prefetched into shared memory (PF stages, piece q of
  // thread j at [stage][q][j]) by cp.async instead of into registers
  __shared__ uint4 pf[PF > 0 ? PF * (C::Fp::N / 2) * NT : 1];
  accum_block<C, PF, NT>(blockIdx.x, entries, off, nseg, nchunks, L, bases, bsum, skey, spt, pf, chk, npts);
}

// One block of NT threads per SM (registers up to 65536 / NT per thread), prefetch stages in
// dynamic shared memory (PF * Q * NT 16-byte pieces, above the 48 KB static limit for NT > 384).
template <class C, int NT, int PF = 2>
__global__ void __launch_bounds__(NT, 1) k_msm_accum_w(const uint32_t* __restrict__ entries,
                                                       const uint32_t* __restrict__ off, uint32_t nseg,
                                                       uint32_t nchunks, uint32_t L, const uint32_t* __restrict__ bases,
                                                       uint32_t* __restrict__ bsum, uint32_t* __restrict__ skey,
                                                       uint32_t* __restrict__ spt, uint32_t* chk, uint32_t npts) {
  extern __shared__ uint4 pf_dyn[];
  accum_block<C, PF, NT>(blockIdx.x, entries, off, nseg, nchunks, L, bases, bsum, skey, spt, pf_dyn, chk, npts);
}

// Cut segments that span at most RUN_MAX + 1 level-1 chunks (with ~64-entry segments and
// ~128-entry chunks, nearly every cut segment spans two) are summed here into the bucket array,
// one thread per segment start, and their slots are cleared, so the fold levels only carry
// longer segments. A cut segment s starting in chunk t leaves its B partial in slot 2t + 1 and
// the A partial of every later chunk it reaches in slot 2t' (a chunk inside s routes its whole
// sum as A); it ends in chunk (off[s + 1] - 1) / L.
static constexpr uint32_t RUN_MAX = 8;
template <class C>
__global__ void __launch_bounds__(256, 2) k_msm_pair_merge(const uint32_t* __restrict__ off, uint32_t nchunks,
                                                           uint32_t L, uint32_t* __restrict__ skey,
                                                           const uint32_t* __restrict__ spt,
                                                           uint32_t* __restrict__ bsum, uint32_t* chk,
                                                           uint32_t nseg) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t + 1 >= nchunks) return;
  const uint32_t s = skey[2 * t + 1];
  if (s == INVALID) return;
  if (chk && s >= nseg) { atomicOr(chk, CHK_SEGMENT); return; }
  const uint32_t last = (__ldg(off + s + 1) - 1) / L;   // chunk holding the segment's last entry
  if (last - t > RUN_MAX) return;                       // left to the fold levels
  Xyzz<F> acc = xyzz_load<F>(spt + (size_t)(2 * t + 1) * XW);
  for (uint32_t u = t + 1; u <= last; u++) {
    xyzz_add_paired(acc, xyzz_load<F>(spt + (size_t)(2 * u) * XW));
    skey[2 * u] = INVALID;   // A slots of chunks t+1..last: no other thread reads or writes them
  }
  xyzz_store<F>(bsum + (size_t)s * XW, acc);
  skey[2 * t + 1] = INVALID;
}

// ---------------------------------------------------------- the FP64-product pipeline
// With BN254D / BLS12_381D (the curves over BnFpD / BlsFpD of zkb_dpf.cuh) the bucket pipeline
// (accumulation, folds, bucket reduction) runs unchanged but with FP64-pipe products, on values
// in the radix R' = 2^(52 L). Bases enter that radix once per MSM (x R -> mont'(x R, R'^2 / R)
// = x R'); the per-window sums U leave it once (x R' -> mont'(x R', R) = x R), so the host tail
// and the output encodings are unchanged. Both conversions are exact field products.
// affine points, radix R -> R' (the identity (0, 0) stays (0, 0))
template <class CD>
__global__ void k_msm_bases_to_dpf(uint32_t n, const uint32_t* __restrict__ src, const Fe<typename CD::Fp> kin,
                                   uint32_t* __restrict__ dst) {
  using FD = typename CD::Fp;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Affine<FD> a = affine_load<FD>(src + (size_t)i * 2 * FD::N);
  fe_store<FD>(dst + (size_t)i * 2 * FD::N, fe_mul(a.x, kin));
  fe_store<FD>(dst + (size_t)i * 2 * FD::N + FD::N, fe_mul(a.y, kin));
}

// XYZZ points in place, radix R' -> R
template <class CD>
__global__ void k_msm_xyzz_from_dpf(uint32_t n, uint32_t* __restrict__ pts, const Fe<typename CD::Fp> kout) {
  using FD = typename CD::Fp;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 4 * n) return;
  uint32_t* q = pts + (size_t)i * FD::N;
  fe_store<FD>(q, fe_canon(fe_mul(fe_load<FD>(q), kout)));
}



// Fold partial sums left by the previous level. Slots carry their segment id (INVALID for an
// unused slot); the range of segment s at this level follows from its range one level down:
// chunks cs..ce of length L_prev hold its pieces at slots 2cs+1 .. 2ce.
template <class C>
__global__ void __launch_bounds__(256) k_msm_seg_level(const uint32_t* __restrict__ ikey,
                                                       const uint32_t* __restrict__ ipt, uint32_t Y, uint32_t L,
                                                       uint32_t nchunks, LevelHist hist,
                                                       const uint32_t* __restrict__ off,
                                                       uint32_t* __restrict__ bsum, uint32_t* __restrict__ okey,
                                                       uint32_t* __restrict__ opt) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nchunks) return;
  const uint64_t start = (uint64_t)t * L;
  const uint64_t end = min(start + L, (uint64_t)Y);
  uint32_t keyA = INVALID, keyB = INVALID;
  uint32_t cur = INVALID;
  Xyzz<F> acc = xyzz_inf<F>();
  auto flush = [&](uint32_t s) {
    uint64_t lo = __ldg(off + s), hi = __ldg(off + s + 1);
    for (int j = 0; j < hist.n; j++) {
      const uint64_t cs = lo / hist.L[j], ce = (hi - 1) / hist.L[j];
      lo = 2 * cs + 1;
      hi = 2 * ce + 1;
    }
    route_run<F>(s, acc, lo, hi, start, L, t, bsum, opt, keyA, keyB);
  };
  for (uint64_t y = start; y < end; y++) {
    const uint32_t k = __ldg(ikey + y);
    if (k == INVALID) continue;
    if (k != cur) {
      if (cur != INVALID) flush(cur);
      cur = k;
      acc = xyzz_inf<F>();
    }
    xyzz_add_paired(acc, xyzz_load<F>(ipt + y * XW));
  }
  if (cur != INVALID) flush(cur);
  okey[2 * (size_t)t] = keyA;
  okey[2 * (size_t)t + 1] = keyB;
}

// ------------------------------------------------------------------------- bucket reduce

// Bucket arrays of up to four point-range parts of one MSM (same window layout); a bucket's sum
// is the sum of its non-empty per-part entries.
struct PartSet {
  int n;
  const uint32_t* bsum[4];
  const uint32_t* off[4];   // segment offsets (empty segments skipped); null: every segment present
};

// Sum of the parts' bucket arrays into `out` (which may be part 0's own array), one thread per
// bucket: the parts of a pipelined host-buffer MSM merge in one parallel pass, so the running sums
// that follow read one array (merging inside their sequential chains cost 1 ms at 2^22)
template <class C>
__global__ void k_msm_merge_parts(PartSet parts, uint32_t nseg, uint32_t* __restrict__ out) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  Xyzz<F> acc = xyzz_inf<F>();
  for (int q = 0; q < parts.n; q++)
    if (__ldg(parts.off[q] + s) != __ldg(parts.off[q] + s + 1)) xyzz_add_paired(acc, xyzz_load<F>(parts.bsum[q] + (size_t)s * XW));
  xyzz_store<F>(out + (size_t)s * XW, acc);
}

// thread (w, g): buckets j = g*K .. g*K+K-1 of window w (bucket number j+1):
// T = sum S_j, R = sum (j - g*K + 1) S_j (running sum from the top)
template <class C>
__global__ void __launch_bounds__(128) k_msm_bucket_rs(PartSet parts, uint32_t B, uint32_t nwin, uint32_t K,
                                                       uint32_t G, uint32_t* __restrict__ Tout,
                                                       uint32_t* __restrict__ Rout) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nwin * G) return;
  const uint32_t w = t / G, g = t % G;
  Xyzz<F> T = xyzz_inf<F>(), R = xyzz_inf<F>();
  for (int l = (int)K - 1; l >= 0; l--) {
    const size_t s = (size_t)w * B + (size_t)g * K + l;
    for (int q = 0; q < parts.n; q++)
      if (!parts.off[q] || __ldg(parts.off[q] + s) != __ldg(parts.off[q] + s + 1))
        xyzz_add_paired(T, xyzz_load<F>(parts.bsum[q] + s * XW));
    xyzz_add_paired(R, T);
  }
  xyzz_store<F>(Tout + (size_t)t * XW, T);
  xyzz_store<F>(Rout + (size_t)t * XW, R);
}

// block (w, k): k < gbits -> U_k = sum over g with bit k set of T_g; k == gbits -> sum of R_g
template <class C>
__global__ void __launch_bounds__(256, 2) k_msm_bucket_bits(const uint32_t* __restrict__ Tin,
                                                         const uint32_t* __restrict__ Rin, uint32_t G,
                                                         int gbits, uint32_t* __restrict__ U) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  extern __shared__ uint4 smem_u4[];
  uint32_t* sm = reinterpret_cast<uint32_t*>(smem_u4);
  const uint32_t w = blockIdx.x, k = blockIdx.y;
  Xyzz<F> acc = xyzz_inf<F>();
  for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) {
    if ((int)k < gbits) {
      if ((g >> k) & 1u) xyzz_add_paired(acc, xyzz_load<F>(Tin + ((size_t)w * G + g) * XW));
    } else {
      xyzz_add_paired(acc, xyzz_load<F>(Rin + ((size_t)w * G + g) * XW));
    }
  }
  xyzz_store<F>(sm + threadIdx.x * XW, acc);
  __syncthreads();
  for (uint32_t half = blockDim.x >> 1; half > 0; half >>= 1) {
    if (threadIdx.x < half) {
      Xyzz<F> a = xyzz_load<F>(sm + threadIdx.x * XW);
      xyzz_add_paired(a, xyzz_load<F>(sm + (threadIdx.x + half) * XW));
      xyzz_store<F>(sm + threadIdx.x * XW, a);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) xyzz_store<F>(U + ((size_t)w * (gbits + 1) + k) * XW, xyzz_canon(xyzz_load<F>(sm)));
}

// ---------------------------------------------------------------------------- planning

static int g_window_override = 0;
// tuning knobs (ZKB_MSM_L1: level-1 chunk length, entries per accumulation thread; ZKB_MSM_K1: buckets per
// running-sum group, a power of two); read once from the environment
static int env_int(const char* name, int dflt) {
  const char* v = std::getenv(name);
  return v ? std::atoi(v) : dflt;
}
static int g_tune_L1 = env_int("ZKB_MSM_L1", 0);
// bucket accumulation on the FP64 pipe (zkb_dpf.cuh); ZKB_MSM_DPF=0 selects the 32-bit-limb kernel
static int g_msm_dpf = env_int("ZKB_MSM_DPF", 1);
static int g_tune_K1 = env_int("ZKB_MSM_K1", 0);
// stages of the accumulation's base prefetch through shared memory (cp.async; ZKB_MSM_PF = 2 or
// 3), 0 = prefetch of the next base into registers
static int g_msm_pf = env_int("ZKB_MSM_PF", 2);
// window-major digit histogram and scatter (ZKB_MSM_WMAJOR=0: point-major, all windows per thread)
static int g_msm_wmajor = env_int("ZKB_MSM_WMAJOR", 1);
static int g_msm_hist_wmajor = env_int("ZKB_MSM_HIST_WMAJOR", 0);
// the histogram stores every digit for the window-major scatter (ZKB_MSM_DIGITS=0: the scatter
// re-derives each digit from its scalar)
static int g_msm_digits = env_int("ZKB_MSM_DIGITS", 1);
static const bool g_msm_pf_env = std::getenv("ZKB_MSM_PF") != nullptr;

// Tuned settings per curve and round(log2 n), from zkg_autotune_msm or the persisted tuning
// cache: window width, level-1 chunk length, running-sum group size, prefetch stages (0 / -1 =
// the default rule). An environment knob, when set, wins over a tuned value.
struct MsmTune {
  int c = 0, L1 = 0, K1 = 0, pf = -1;
  int tree = 0;   // affine tree levels + 1 (0 = the default rule)
};
static MsmTune g_tune[2][32];
static std::once_flag g_tune_once[2];

static int round_log2(uint64_t n);
static MsmTune& msm_tune(int curve, int lg) {
  std::call_once(g_tune_once[curve], [curve] {
    const int sms = device_sm_count();
    for (int l = 0; l < 32; l++) {
      int v[5];
      if (tune_cache_get("msm", curve, l, sms, v, 4)) {
        g_tune[curve][l].c = v[0];
        g_tune[curve][l].L1 = v[1];
        g_tune[curve][l].K1 = v[2];
        g_tune[curve][l].pf = v[3];
        if (tune_cache_get("msm", curve, l, sms, v, 5)) g_tune[curve][l].tree = v[4];   // entries before the tree: 4 values
      }
    }
  });
  return g_tune[curve][lg < 0 ? 0 : (lg > 31 ? 31 : lg)];
}

// Buckets per running-sum group of the bucket reduction. Each group is one thread's sequential
// chain of 2 K1 additions: long groups keep the bucket_bits tail small (2^22 points: 32 measured
// best), but for small MSMs (few windows x buckets) they leave the GPU idle, so K1 shrinks until
// nwin * B / K1 reaches 16 K threads.
static uint32_t pick_k1(uint32_t nwin, uint32_t B, int tuned = 0) {
  if (g_tune_K1 > 0) return std::min<uint32_t>(B, (uint32_t)g_tune_K1);
  if (tuned > 0) return std::min<uint32_t>(B, (uint32_t)tuned);
  uint32_t k = 32;
  while (k > 2 && (uint64_t)nwin * B / k < 16384) k >>= 1;
  return std::min<uint32_t>(B, k);
}

static int ilog2_floor(uint64_t x) {
  int r = -1;
  while (x) { x >>= 1; r++; }
  return r;
}

// Cost model: nwin * (n madds + 2^(c-1) buckets * w madd-equivalents) + per-window tail. w = 2.8
// for BN254; 3.5 for BLS12-381, whose affine tree levels make an entry cheaper against a bucket's
// running-sum additions (measured at 2^22: c = 16 29.5 ms, the 2.8 rule's c = 18 33.8 ms).
static double bucket_weight(int curve) { return curve == ZKG_BLS12_381 ? 3.5 : 2.8; }
static int auto_window(int n, int scalar_bits, double w) {
  if (n <= 1) return 2;
  double best = 1e300;
  int bestc = 2;
  for (int c = 2; c <= 20; c++) {
    const int nwin = (scalar_bits + 1 + c - 1) / c;
    const double cost = (double)nwin * ((double)n + w * (double)(1u << (c - 1)) + 4000.0);
    if (cost < best) { best = cost; bestc = c; }
  }
  return bestc;
}

// ------------------------------------------------------------------------- window tuning

static int round_log2(uint64_t n) { return n > 1 ? ilog2_floor(n + (n >> 1)) : 0; }

static int pick_window(int curve, int n, int scalar_bits) {
  if (g_window_override > 0) return g_window_override;
  if (n > 1) {
    const MsmTune& T = msm_tune(curve, round_log2((uint64_t)n));
    if (T.c > 0) return T.c;
  }
  return auto_window(n, scalar_bits, bucket_weight(curve));
}

// Affine tree levels before the chunk accumulation (zkb_msm_tree.cuh). ZKB_MSM_TREE = the number
// of levels (0 = none). By default BLS12-381 runs trees by the entries per bucket segment e:
// none below 64, then log2(e) - 4 levels up to three (measured at c = 16: 2^18 and 2^20 points,
// e = 32: the tree costs 0-40%; 2^21, e = 64: 2 levels 15.9 ms against 17.1; 2^22, e = 128:
// 3 levels 28.5 ms against 33.1). BN254 runs none (its mixed addition is cheap enough that the
// levels' extra passes over memory cancel their fewer products: 14.3-14.4 ms at 2^22 either way).
// ZKB_MSM_TREE_B: output slots per tree thread (its simultaneous-inversion batch); by default 64
// from e = 128 (2^22: 28.5 ms against 29.0 with 32), 32 below.
static int g_tree_env = env_int("ZKB_MSM_TREE", -1);
static uint32_t g_tree_B = (uint32_t)std::max(0, env_int("ZKB_MSM_TREE_B", 0));   // 0: by e

template <class C>
static int pick_tree(uint64_t total, uint32_t nseg, int tuned) {
  if constexpr (radix_conv_v<typename C::Fp>) {
    return 0;   // the tree's inversion works in the reference's radix
  } else {
    int k = g_tree_env >= 0 ? g_tree_env : tuned - 1;
    if (k < 0) {
      const uint64_t e = total / std::max<uint32_t>(1, nseg);
      if (C::Fp::N == 8 || e < 64) return 0;
      k = std::min(3, ilog2_floor(e) - 4);
    }
    return std::max(0, std::min(k, MAX_TREE));
  }
}
static uint32_t pick_tree_slots(uint64_t total, uint32_t nseg) {
  if (g_tree_B) return std::max<uint32_t>(4, g_tree_B);
  return total / std::max<uint32_t>(1, nseg) >= 128 ? 64u : 32u;
}

// Launch shape of the accumulation (ZKB_MSM_ACCUM_SHAPE): 0 = 256-thread blocks, two per SM for
// BN254 (128 registers per thread, the paired products spill); otherwise one block per SM of
// 1: 256 threads (255 registers), 2: 384 (170), 3: 320 (204), 4: 448 (146), 5: 512 (128).
// BLS12-381 (96-byte bases, more registers per product) uses shape 1 for every shape but 0.
static int g_accum_shape = env_int("ZKB_MSM_ACCUM_SHAPE", 2);

template <class C>
static int accum_shape() {
  const int s = g_accum_shape < 0 || g_accum_shape > 5 ? 2 : g_accum_shape;
  return (s >= 2 && C::Fp::N != 8) ? 1 : s;
}
static int accum_threads(int shape) {
  static const int nt[6] = {256, 256, 384, 320, 448, 512};
  return nt[shape];
}
template <class C, int NT, int PF = 2>
static int accum_w_occupancy() {
  const size_t smem = (size_t)PF * (C::Fp::N / 2) * NT * 16;
  if (cudaFuncSetAttribute(k_msm_accum_w<C, NT, PF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return 0;
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_msm_accum_w<C, NT, PF>, NT, smem) != cudaSuccess) return 0;
  return b;
}

// Threads of k_msm_accum<C> resident on the whole GPU at once (one "wave").
template <class C>
static uint64_t accum_wave() {
  static const uint64_t w = [] {
    int dev = 0, sms = 148, blocks = 1;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
      sms = 148;
    const int shape = accum_shape<C>();
    cudaError_t e = cudaSuccess;
    if (shape == 0) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_msm_accum<C, 2>, 256, 0);
    else if (shape == 1) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_msm_accum<C, 2, 256, 1>, 256, 0);
    else if constexpr (C::Fp::N == 8) {
      blocks = shape == 2 ? accum_w_occupancy<C, 384>() : shape == 3 ? accum_w_occupancy<C, 320>()
             : shape == 4 ? accum_w_occupancy<C, 448>() : accum_w_occupancy<C, 512>();
      accum_w_occupancy<C, 384, 3>();   // the three-stage form's shared-memory limit
    }
    if (e != cudaSuccess || blocks < 1) blocks = 1;
    return (uint64_t)sms * (uint64_t)blocks * (uint64_t)accum_threads(shape);
  }();
  return w;
}

template <class C>
static zkg_status launch_accum(uint32_t nch, cudaStream_t st, const uint32_t* ent, const uint32_t* off, uint32_t nseg,
                               uint32_t L, const uint32_t* bases, uint32_t* bsum, uint32_t* key, uint32_t* pt,
                               int pf = -1, uint32_t* chk = nullptr, uint32_t npts = 0) {
  if (pf < 0) pf = g_msm_pf;
  const dim3 g((nch + 255) / 256);
  if constexpr (C::Fp::N == 8) {   // three stages of 96-byte BLS12-381 bases exceed 48 KB of shared memory
    if (pf >= 3 && accum_shape<C>() == 2) {
      accum_wave<C>();
      return launch("msm_accum", k_msm_accum_w<C, 384, 3>, dim3((nch + 383) / 384), dim3(384),
                    (size_t)3 * (C::Fp::N / 2) * 384 * 16, st, ent, off, nseg, nch, L, bases, bsum, key, pt, chk,
                    npts);
    }
    if (pf >= 3) return launch("msm_accum", k_msm_accum<C, 3>, g, dim3(256), 0, st, ent, off, nseg, nch, L, bases, bsum, key, pt, chk, npts);
  }
  if (pf >= 1) {
    const int shape = accum_shape<C>();
    if (shape == 1)
      return launch("msm_accum", k_msm_accum<C, 2, 256, 1>, g, dim3(256), 0, st, ent, off, nseg, nch, L, bases, bsum,
                    key, pt, chk, npts);
    if constexpr (C::Fp::N == 8) {
      if (shape >= 2) {
        accum_wave<C>();   // sets the kernels' shared-memory limit
        const int nt = accum_threads(shape);
        const size_t smem = (size_t)2 * (C::Fp::N / 2) * nt * 16;
        const dim3 gw((nch + nt - 1) / nt);
#define ZKB_ACCUM_W(NTV)                                                                                \
  return launch("msm_accum", k_msm_accum_w<C, NTV>, gw, dim3(NTV), smem, st, ent, off, nseg, nch, L, bases, \
                bsum, key, pt, chk, npts);
        if (nt == 384) ZKB_ACCUM_W(384)
        if (nt == 320) ZKB_ACCUM_W(320)
        if (nt == 448) ZKB_ACCUM_W(448)
        ZKB_ACCUM_W(512)
#undef ZKB_ACCUM_W
      }
    }
    return launch("msm_accum", k_msm_accum<C, 2>, g, dim3(256), 0, st, ent, off, nseg, nch, L, bases, bsum, key, pt, chk, npts);
  }
  return launch("msm_accum", k_msm_accum<C, 0>, g, dim3(256), 0, st, ent, off, nseg, nch, L, bases, bsum, key, pt, chk, npts);
}

// Level-1 chunk length (entries per accumulation thread) for `total` entries: about 128, with the
// thread count a whole number of waves, so no SM idles through a partial last wave; below eight
// entries per thread of one wave, chunks of 8. tuned > 0: a tuned length.
static uint32_t chunk_len(uint64_t total, uint64_t wave, int tuned = 0) {
  if (g_tune_L1 > 0) return (uint32_t)g_tune_L1;
  if (tuned > 0) return (uint32_t)tuned;
  if (total <= wave * 8) return 8;
  const uint64_t k = std::max<uint64_t>(1, (total + wave * 64) / (wave * 128));   // round(total / (128 wave))
  return (uint32_t)((total + k * wave - 1) / (k * wave));
}

struct MsmPlan {
  int n = 0, c = 0, nwin = 0, nw = 0;
  uint32_t B = 0, nseg = 0;
  uint64_t total_max = 0;   // nwin * n
  int L1 = 64;
  int nlev = 0;             // levels after the first
  uint32_t Llev[MAX_LEVELS];
  uint64_t Ylev[MAX_LEVELS];   // slot positions read by level k (k >= 2)
  uint32_t nch[MAX_LEVELS + 1]; // chunks per level (index 0 = level 1)
  uint32_t K1 = 0, G = 0;
  int gbits = 0;
  int pf = 2;               // prefetch stages of the accumulation
  // affine tree levels before the chunk accumulation (zkb_msm_tree.cuh): level l's output count
  // is at most tQ[l]; tthr[l] threads of tB output slots each
  int tree = 0;
  uint32_t tB = 32;
  uint64_t tQ[MAX_TREE];
  uint32_t tthr[MAX_TREE];
  uint64_t acc_total = 0;   // entries of the chunk accumulation (a bound when tree > 0)
  // byte offsets into one arena block
  size_t o_std, o_cnt, o_off, o_cur, o_bs, o_ent, o_keyA, o_ptA, o_keyB, o_ptB, o_bsum, o_T, o_R, o_U, bytes;
  bool use_dig = false;   // digits and ranks stored at o_dig, o_rank (nwin x n words each)
  size_t o_dig = 0, o_rank = 0;
  size_t o_toff[2], o_tpts[2], o_tpre, o_ttt, o_tscr;
};

template <class C>
static zkg_status make_plan(int n, int nlimbs, int mont, MsmPlan& P, int c_force = 0) {
  using F = typename C::Fp;
  constexpr size_t XB = 16 * F::N;   // bytes of one XYZZ point
  P.n = n;
  const int scalar_bits = mont ? C::SCALAR_BITS : 64 * nlimbs;
  P.c = c_force > 0 ? c_force : pick_window(C::ID, n, scalar_bits);
  if (P.c < 2 || P.c > 24) return set_status(ZKG_ERR_ARG, "msm", "window width out of range [2, 24]");
  P.nwin = (scalar_bits + 1 + P.c - 1) / P.c;
  P.nw = mont ? 8 : 2 * nlimbs;
  P.B = 1u << (P.c - 1);
  P.nseg = (uint32_t)P.nwin * P.B;
  P.total_max = (uint64_t)P.nwin * (uint64_t)n;
  if (P.total_max >= (1ull << 31)) return set_status(ZKG_ERR_ARG, "msm", "too many (window, point) entries for one launch");
  const MsmTune& T = msm_tune(C::ID, round_log2((uint64_t)n));
  P.tree = pick_tree<C>(P.total_max, P.nseg, T.tree);
  P.acc_total = P.total_max;
  if (P.tree > 0) {
    P.tB = pick_tree_slots(P.total_max, P.nseg);
    for (int l = 0; l < P.tree; l++) {   // sum_s ceil(m_s / 2^(l+1)) <= total / 2^(l+1) + nseg
      P.tQ[l] = std::min<uint64_t>(P.acc_total, (P.total_max >> (l + 1)) + P.nseg);
      P.tthr[l] = (uint32_t)((P.tQ[l] + P.tB - 1) / P.tB);
      P.acc_total = P.tQ[l];
    }
  }
  P.L1 = (int)chunk_len(P.acc_total, accum_wave<C>(), T.L1);
  P.pf = g_msm_pf_env || T.pf < 0 ? g_msm_pf : T.pf;
  P.nch[0] = (uint32_t)((P.acc_total + P.L1 - 1) / P.L1);
  if (P.nch[0] == 0) P.nch[0] = 1;
  // later levels: slot arrays of 2 * previous chunks, folded in chunks of 16
  P.nlev = 0;
  uint64_t Y = 2ull * P.nch[0];
  uint32_t prev_chunks = P.nch[0];
  while (prev_chunks > 1) {
    if (P.nlev >= MAX_LEVELS - 1) return set_status(ZKG_ERR_ARG, "msm", "level overflow");
    const uint32_t L = 16;
    P.Llev[P.nlev] = L;
    P.Ylev[P.nlev] = Y;
    const uint32_t ch = (uint32_t)((Y + L - 1) / L);
    P.nch[P.nlev + 1] = ch;
    P.nlev++;
    Y = 2ull * ch;
    prev_chunks = ch;
  }
  P.K1 = pick_k1((uint32_t)P.nwin, P.B, T.K1);
  P.G = P.B / P.K1;
  P.gbits = ilog2_floor(P.G);

  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o = (o + bytes + 255) & ~size_t(255); return r; };
  const bool dig_path = g_msm_digits && g_msm_wmajor;   // P.use_dig below
  P.o_std = take(mont && !dig_path ? (size_t)n * 32 : 0);
  P.o_cnt = take((size_t)P.nseg * 4 + 4);
  P.o_off = take((size_t)P.nseg * 4 + 4);
  P.o_cur = take((size_t)P.nseg * 4 + 4);
  const uint32_t nb = (P.nseg + SCAN_T * SCAN_E - 1) / (SCAN_T * SCAN_E);
  if (nb > (uint32_t)SCAN_T * SCAN_E) return set_status(ZKG_ERR_ARG, "msm", "too many buckets");
  P.o_bs = take((size_t)nb * 4 + 4);
  P.o_ent = take((size_t)P.total_max * 4 + 4);
  P.use_dig = dig_path;
  P.o_dig = take(P.use_dig ? (size_t)P.total_max * 4 + 4 : 0);
  P.o_rank = take(P.use_dig ? (size_t)P.total_max * 4 + 4 : 0);
  uint64_t slotsA = 2ull * P.nch[0], slotsB = 0;
  for (int k = 1; k <= P.nlev; k++) {
    if (k % 2 == 1) slotsB = std::max<uint64_t>(slotsB, 2ull * P.nch[k]);
    else slotsA = std::max<uint64_t>(slotsA, 2ull * P.nch[k]);
  }
  P.o_keyA = take(slotsA * 4);
  P.o_ptA = take(slotsA * XB);
  P.o_keyB = take(slotsB * 4 + 4);
  P.o_ptB = take(slotsB * XB + 4);
  P.o_bsum = take((size_t)P.nseg * XB);
  P.o_T = take((size_t)P.nwin * P.G * XB);
  P.o_R = take((size_t)P.nwin * P.G * XB);
  P.o_U = take((size_t)P.nwin * (P.gbits + 1) * XB);
  P.o_toff[0] = P.o_toff[1] = P.o_tpts[0] = P.o_tpts[1] = P.o_tpre = P.o_ttt = P.o_tscr = 0;
  if (P.tree > 0) {
    constexpr size_t AB = 8 * F::N, FB = 4 * F::N;   // bytes of an affine point, of a field element
    P.o_toff[0] = take((size_t)P.nseg * 4 + 4);
    P.o_toff[1] = take((size_t)P.nseg * 4 + 4);
    P.o_tpts[0] = take(P.tQ[0] * AB);
    P.o_tpts[1] = take(P.tree > 1 ? P.tQ[1] * AB : 0);
    P.o_tpre = take(P.tQ[0] * FB);
    P.o_ttt = take((size_t)P.tthr[0] * FB);
    P.o_tscr = take((size_t)P.tthr[0] * FB);
  }
  P.bytes = o;
  return ZKG_OK;
}

// per-window sums U of a finished FP64-product pipeline back to radix R (before the host tail)
template <class CP>
static zkg_status msm_u_to_radix(const MsmPlan& P, char* ws, cudaStream_t st) {
  if constexpr (radix_conv_v<typename CP::Fp>) {
    Fe<typename CP::Fp> kin, kout;
    dpf_consts_for<CP>(kin, kout);
    const uint32_t npts = (uint32_t)P.nwin * (P.gbits + 1);
    ZKB_TRY(launch("msm_xyzz_from_dpf", k_msm_xyzz_from_dpf<CP>, dim3((4 * npts + 255) / 256), dim3(256), 0, st,
                   npts, reinterpret_cast<uint32_t*>(ws + P.o_U), kout));
  }
  return ZKG_OK;
}

// Dynamic shared memory above the default 48 KB needs the kernel's attribute set, once per kernel
// (the statics are per instantiation: FWD, C, L0, NT and PF name the tree kernel).
template <bool FWD, class C, bool L0, int NT, int PF, class K>
static zkg_status tree_smem_limit(K kernel, size_t bytes) {
  static const cudaError_t e = bytes > 48 * 1024
                                   ? cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes)
                                   : cudaSuccess;
  if (e != cudaSuccess) return set_status(ZKG_ERR_CUDA, "msm", cudaGetErrorString(e));
  return ZKG_OK;
}

// prefetch stages of the tree's backward pass (ZKB_MSM_TREE_PF = 2 or 3); the forward pass has 3
static int g_tree_pf = env_int("ZKB_MSM_TREE_PF", 2);

template <class C, bool L0, int NT, int PF>
static zkg_status launch_tree_bwd(const MsmPlan& P, uint32_t nthr, cudaStream_t st, const uint32_t* ent,
                                  const uint32_t* in_pts, const uint32_t* in_off, const uint32_t* out_off,
                                  const uint32_t* pre, const uint32_t* tinv, uint32_t* out_pts, uint32_t* chk,
                                  uint32_t npts) {
  const size_t smem = (size_t)PF * tree_bwd_pieces<typename C::Fp>() * NT * 16;
  ZKB_TRY((tree_smem_limit<false, C, L0, NT, PF>(k_tree_bwd<C, L0, NT, PF>, smem)));
  return launch("msm_tree_bwd", k_tree_bwd<C, L0, NT, PF>, dim3((nthr + NT - 1) / NT), dim3(NT), smem, st, ent,
                in_pts, in_off, out_off, P.nseg, P.tB, nthr, pre, tinv, out_pts, chk, npts);
}

template <class C, bool L0>
static zkg_status launch_tree_level(const MsmPlan& P, uint32_t nthr, cudaStream_t st, const uint32_t* ent,
                                    const uint32_t* in_pts, const uint32_t* in_off, const uint32_t* out_off,
                                    uint32_t* pre, uint32_t* tt, uint32_t* scr, uint32_t* out_pts, uint32_t* chk,
                                    uint32_t npts) {
  using F = typename C::Fp;
  constexpr int NTF = 256, PFF = 3;
  const size_t smf = (size_t)PFF * tree_fwd_pieces<F>() * NTF * 16;
  ZKB_TRY((tree_smem_limit<true, C, L0, NTF, PFF>(k_tree_fwd<C, L0, NTF, PFF>, smf)));
  ZKB_TRY(launch("msm_tree_fwd", k_tree_fwd<C, L0, NTF, PFF>, dim3((nthr + NTF - 1) / NTF), dim3(NTF), smf, st, ent,
                 in_pts, in_off, out_off, P.nseg, P.tB, nthr, pre, tt, chk, npts));
  // simultaneous inversion of the thread products: about 16 per thread
  const size_t T = std::min<size_t>(((size_t)nthr + 255) & ~size_t(255), std::max<size_t>(2048, (size_t)nthr / 16));
  ZKB_TRY(launch("msm_tree_inv", k_tree_inv<F>, dim3((unsigned)((T + 255) / 256)), dim3(256), 0, st, nthr, tt, scr));
  // backward pass: one block per SM, as the accumulation (BN254: 384 threads, 166 registers)
  constexpr int NTB = F::N == 8 ? 384 : 256;
  if (g_tree_pf >= 3)
    return launch_tree_bwd<C, L0, NTB, 3>(P, nthr, st, ent, in_pts, in_off, out_off, pre, tt, out_pts, chk, npts);
  return launch_tree_bwd<C, L0, NTB, 2>(P, nthr, st, ent, in_pts, in_off, out_off, pre, tt, out_pts, chk, npts);
}

// The affine tree levels of one point range (zkb_msm_tree.cuh): level l reads the sorted entries
// and bases (l = 0) or level l - 1's list, and writes its offsets to o_toff[l & 1] and its points
// to o_tpts[l & 1]. The sort's count, cursor and scan buffers are free by now and are reused.
template <class C>
static zkg_status msm_tree_launch(const MsmPlan& P, char* ws, const uint32_t* ent, const uint32_t* off,
                                  const uint32_t* bases, cudaStream_t st, uint32_t* chk) {
  auto U32 = [&](size_t o) { return reinterpret_cast<uint32_t*>(ws + o); };
  const uint32_t nb = (P.nseg + SCAN_T * SCAN_E - 1) / (SCAN_T * SCAN_E);
  const uint32_t* in_off = off;
  const uint32_t* in_pts = bases;
  for (int l = 0; l < P.tree; l++) {
    uint32_t* out_off = U32(P.o_toff[l & 1]);
    uint32_t* out_pts = U32(P.o_tpts[l & 1]);
    ZKB_TRY(launch("msm_tree_counts", k_tree_counts, dim3((P.nseg + 255) / 256), dim3(256), 0, st, in_off, P.nseg,
                   U32(P.o_cnt)));
    ZKB_TRY(launch("scan_blocks", k_scan_blocks, dim3(nb), dim3(SCAN_T), 0, st, (const uint32_t*)U32(P.o_cnt),
                   out_off, U32(P.o_bs), P.nseg));
    ZKB_TRY(launch("scan_top", k_scan_top, dim3(1), dim3(SCAN_T), 0, st, U32(P.o_bs), nb));
    ZKB_TRY(launch("scan_add", k_scan_add, dim3((P.nseg + 255) / 256), dim3(256), 0, st, out_off, U32(P.o_cur),
                   (const uint32_t*)U32(P.o_bs), P.nseg, nb));
    const uint32_t npts = l == 0 ? (uint32_t)P.n : (uint32_t)P.tQ[l - 1];
    if (l == 0)
      ZKB_TRY((launch_tree_level<C, true>(P, P.tthr[l], st, ent, in_pts, in_off, out_off, U32(P.o_tpre), U32(P.o_ttt),
                                          U32(P.o_tscr), out_pts, chk, npts)));
    else
      ZKB_TRY((launch_tree_level<C, false>(P, P.tthr[l], st, ent, in_pts, in_off, out_off, U32(P.o_tpre),
                                           U32(P.o_ttt), U32(P.o_tscr), out_pts, chk, npts)));
    in_off = out_off;
    in_pts = out_pts;
  }
  return ZKG_OK;
}

// Sort the scalars of one point range into (window, bucket) segments and accumulate its bucket
// sums (phases 1-6). bases_ready, if given, is waited for just before the accumulation.
template <class C>
static zkg_status msm_launch_part(Context& cx, const MsmPlan& P, char* ws, const uint64_t* d_scal, int mont,
                                  const uint64_t* d_bases, cudaStream_t st, cudaEvent_t bases_ready, bool first,
                                  bool last, const uint32_t* conv_src = nullptr, int fold_part = -1) {
  NvtxRange nvtx_sort("zkb.msm.sort");
  uint32_t* chk = dev_check_word(cx);
  const int n = P.n;
  auto U32 = [&](size_t o) { return reinterpret_cast<uint32_t*>(ws + o); };
  // phase events: 0 start, 1 sorted, 2 level-1 accumulated, 3 levels folded, 4 reduced
  if (first) ZKB_CUDA(cudaEventRecord(cx.ev_phase[0], st));
  const uint32_t* scal = reinterpret_cast<const uint32_t*>(d_scal);
  const bool hist_mont = mont && P.use_dig;   // conversion inside the histogram
  if (mont && !hist_mont) {
    ZKB_TRY(launch("msm_scalar_from_mont", k_msm_scalar_from_mont<C>, dim3((n + 255) / 256), dim3(256), 0, st,
                   n, d_scal, U32(P.o_std)));
    scal = U32(P.o_std);
  }
  ZKB_CUDA(cudaMemsetAsync(U32(P.o_cnt), 0, (size_t)P.nseg * 4, st));
  CarryTable ct;
  const bool wmajor = g_msm_wmajor && make_carry_table(P.nwin, P.nw, P.c, ct);
  // the histogram reads each scalar once and loops over its windows (the window-major histogram
  // re-reads the scalars per window and measured slower); the scatter is window-major, from the
  // digits the histogram stores (P.o_dig) or, without them, re-deriving each digit from its scalar
  uint32_t* dig = P.use_dig ? U32(P.o_dig) : nullptr;
  uint32_t* rank = P.use_dig ? U32(P.o_rank) : nullptr;
  if (hist_mont)
    ZKB_TRY(launch("msm_hist_mont", k_msm_hist_mont<C>, dim3((n + 255) / 256), dim3(256), 0, st, n, d_scal, P.c,
                   P.nwin, P.B, U32(P.o_cnt), chk, dig, rank));
  else if (wmajor && g_msm_hist_wmajor && !dig)
    ZKB_TRY(launch("msm_hist_w", k_msm_hist_w, dim3((n + 255) / 256, P.nwin), dim3(256), 0, st, n, scal, P.nw, P.c,
                   P.B, ct, U32(P.o_cnt), chk));
  else
    ZKB_TRY(launch("msm_hist", k_msm_hist, dim3((n + 255) / 256), dim3(256), 0, st, n, scal, P.nw, P.c, P.nwin,
                   P.B, U32(P.o_cnt), chk, dig, rank));
  const uint32_t nb = (P.nseg + SCAN_T * SCAN_E - 1) / (SCAN_T * SCAN_E);
  ZKB_TRY(launch("scan_blocks", k_scan_blocks, dim3(nb), dim3(SCAN_T), 0, st, (const uint32_t*)U32(P.o_cnt),
                 U32(P.o_off), U32(P.o_bs), P.nseg));
  ZKB_TRY(launch("scan_top", k_scan_top, dim3(1), dim3(SCAN_T), 0, st, U32(P.o_bs), nb));
  ZKB_TRY(launch("scan_add", k_scan_add, dim3((P.nseg + 255) / 256), dim3(256), 0, st, U32(P.o_off),
                 U32(P.o_cur), (const uint32_t*)U32(P.o_bs), P.nseg, nb));
  if (dig)
    ZKB_TRY(launch("msm_scatter_d", k_msm_scatter_d, dim3((n + 255) / 256, P.nwin), dim3(256), 0, st, n,
                   (const uint32_t*)dig, (const uint32_t*)rank, P.B, (const uint32_t*)U32(P.o_off), U32(P.o_ent),
                   chk, (uint32_t)P.total_max));
  else if (wmajor)
    ZKB_TRY(launch("msm_scatter_w", k_msm_scatter_w, dim3((n + 255) / 256, P.nwin), dim3(256), 0, st, n, scal, P.nw,
                   P.c, P.B, ct, U32(P.o_cur), U32(P.o_ent), chk, (uint32_t)P.total_max));
  else
    ZKB_TRY(launch("msm_scatter", k_msm_scatter, dim3((n + 255) / 256), dim3(256), 0, st, n, scal, P.nw, P.c,
                   P.nwin, P.B, U32(P.o_cur), U32(P.o_ent)));
  const uint32_t* bases = reinterpret_cast<const uint32_t*>(d_bases);
  if (first) ZKB_CUDA(cudaEventRecord(cx.ev_phase[1], st));
  if (bases_ready) ZKB_CUDA(cudaStreamWaitEvent(st, bases_ready, 0));
  const uint32_t* ent = U32(P.o_ent);
  const uint32_t* off = U32(P.o_off);
  if constexpr (radix_conv_v<typename C::Fp>) {
    if (conv_src) {   // FP64-product pipeline: bases into its radix first (d_bases is the output)
      Fe<typename C::Fp> kin, kout;
      dpf_consts_for<C>(kin, kout);
      ZKB_TRY(launch("msm_bases_to_dpf", k_msm_bases_to_dpf<C>, dim3((n + 255) / 256), dim3(256), 0, st,
                     (uint32_t)n, conv_src, kin, const_cast<uint32_t*>(bases)));
    }
  }
  nvtx_sort.end();
  NvtxRange nvtx_acc("zkb.msm.accumulate_fold");
  uint32_t acc_npts = (uint32_t)P.n;
  if constexpr (!radix_conv_v<typename C::Fp>) {
    if (P.tree > 0) {   // affine tree levels; the chunk accumulation takes the last level's list
      NvtxRange nvtx_tree("zkb.msm.affine_tree");
      ZKB_TRY(msm_tree_launch<C>(P, ws, ent, off, bases, st, chk));
      const int lt = (P.tree - 1) & 1;
      ent = nullptr;
      off = U32(P.o_toff[lt]);
      bases = U32(P.o_tpts[lt]);
      acc_npts = (uint32_t)P.tQ[P.tree - 1];
    }
  }
  ZKB_TRY(launch_accum<C>(P.nch[0], st, ent, off, P.nseg, (uint32_t)P.L1, bases, U32(P.o_bsum), U32(P.o_keyA),
                          U32(P.o_ptA), P.pf, chk, acc_npts));
  if (last) ZKB_CUDA(cudaEventRecord(cx.ev_phase[2], st));
  // fold_part >= 0: the fold levels run on the side stream (they are latency-bound and use few
  // SMs, so the next part's sort and accumulation fill the rest); ev_fold[fold_part] marks them done
  const cudaStream_t fst = fold_part >= 0 ? cx.side_stream : st;
  if (fold_part >= 0) {
    ZKB_CUDA(cudaEventRecord(cx.ev_acc[fold_part], st));
    ZKB_CUDA(cudaStreamWaitEvent(fst, cx.ev_acc[fold_part], 0));
  }
  ZKB_TRY(launch("msm_pair_merge", k_msm_pair_merge<C>, dim3((P.nch[0] + 255) / 256), dim3(256), 0, fst, off, P.nch[0], (uint32_t)P.L1,
                 U32(P.o_keyA), (const uint32_t*)U32(P.o_ptA), U32(P.o_bsum), chk, P.nseg));
  LevelHist hist;
  hist.n = 1;
  hist.L[0] = (uint32_t)P.L1;
  for (int k = 0; k < P.nlev; k++) {
    const bool fromA = (k % 2 == 0);
    const uint32_t* ik = U32(fromA ? P.o_keyA : P.o_keyB);
    const uint32_t* ip = U32(fromA ? P.o_ptA : P.o_ptB);
    uint32_t* ok = U32(fromA ? P.o_keyB : P.o_keyA);
    uint32_t* op = U32(fromA ? P.o_ptB : P.o_ptA);
    const uint32_t ch = P.nch[k + 1];
    ZKB_TRY(launch("msm_seg_level", k_msm_seg_level<C>, dim3((ch + 255) / 256), dim3(256), 0, fst, ik, ip,
                   (uint32_t)P.Ylev[k], P.Llev[k], ch, hist, off, U32(P.o_bsum), ok, op));
    hist.L[hist.n++] = P.Llev[k];
  }
  if (last) ZKB_CUDA(cudaEventRecord(cx.ev_phase[3], fst));
  if (fold_part >= 0) ZKB_CUDA(cudaEventRecord(cx.ev_fold[fold_part], fst));
  return ZKG_OK;
}

// Bucket reduction over the parts' bucket arrays (phase 7) into U of workspace ws0 / plan P0.
template <class C>
static zkg_status msm_launch_reduce(Context& cx, const MsmPlan& P0, char* ws0, const PartSet& parts,
                                    cudaStream_t st, bool record_phase = true) {
  NvtxRange nvtx("zkb.msm.bucket_reduce");
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  auto U32 = [&](size_t o) { return reinterpret_cast<uint32_t*>(ws0 + o); };
  const uint32_t nthr = (uint32_t)P0.nwin * P0.G;
  PartSet rs = parts;
  if (parts.n > 1) {   // one parallel merge into part 0's bucket array, then running sums over it
    uint32_t* merged = U32(P0.o_bsum);
    ZKB_TRY(launch("msm_merge_parts", k_msm_merge_parts<C>, dim3((P0.nseg + 255) / 256), dim3(256), 0, st, parts,
                   P0.nseg, merged));
    rs.n = 1;
    rs.bsum[0] = merged;
    rs.off[0] = nullptr;   // merged sums are present for every segment (the identity where all parts were empty)
  }
  ZKB_TRY(launch("msm_bucket_rs", k_msm_bucket_rs<C>, dim3((nthr + 127) / 128), dim3(128), 0, st, rs, P0.B,
                 (uint32_t)P0.nwin, P0.K1, P0.G, U32(P0.o_T), U32(P0.o_R)));
  const size_t smem = 256 * XW * 4;
  ZKB_TRY(launch("msm_bucket_bits", k_msm_bucket_bits<C>, dim3(P0.nwin, P0.gbits + 1), dim3(256), smem, st,
                 (const uint32_t*)U32(P0.o_T), (const uint32_t*)U32(P0.o_R), P0.G, P0.gbits, U32(P0.o_U)));
  if (record_phase) ZKB_CUDA(cudaEventRecord(cx.ev_phase[4], st));
  return ZKG_OK;
}

// Host tail: Horner over bits and windows on the per-window sums.
template <int NL>
static host::Xyzz<NL> msm_host_combine(const host::Field<NL>& F, const MsmPlan& P, const uint64_t* U) {
  auto ld = [&](int w, int k) {
    host::Xyzz<NL> r;
    const uint64_t* p = U + ((size_t)w * (P.gbits + 1) + k) * 4 * NL;
    std::memcpy(r.X.v, p, 8 * NL);
    std::memcpy(r.Y.v, p + NL, 8 * NL);
    std::memcpy(r.ZZ.v, p + 2 * NL, 8 * NL);
    std::memcpy(r.ZZZ.v, p + 3 * NL, 8 * NL);
    return r;
  };
  int k1bits = 0;
  while ((1u << k1bits) < P.K1) k1bits++;
  host::Xyzz<NL> res = host::xyzz_inf<NL>();
  for (int w = P.nwin - 1; w >= 0; w--) {
    if (w != P.nwin - 1)
      for (int i = 0; i < P.c; i++) res = host::xyzz_dbl(F, res);
    host::Xyzz<NL> V = host::xyzz_inf<NL>();
    for (int k = P.gbits - 1; k >= 0; k--) {
      V = host::xyzz_dbl(F, V);
      V = host::xyzz_add(F, V, ld(w, k));
    }
    for (int i = 0; i < k1bits; i++) V = host::xyzz_dbl(F, V);
    V = host::xyzz_add(F, V, ld(w, P.gbits));
    res = host::xyzz_add(F, res, V);
  }
  return res;
}

// Reads back U and the addition counts, runs the host tail and writes the output encoding.
template <class C, int NL>
static zkg_status msm_finish(Context& cx, const host::Field<NL>& F, const MsmPlan& P0, char* ws0,
                             char* const* ws, const MsmPlan* P, int nparts, int kind, uint64_t* tgt,
                             cudaStream_t st) {
  const size_t ubytes = (size_t)P0.nwin * (P0.gbits + 1) * 4 * NL * 8;
  ZKB_TRY(pinned_reserve(cx, ubytes + 64));
  char* pin = static_cast<char*>(cx.pinned);
  ZKB_CUDA(cudaMemcpyAsync(pin, ws0 + P0.o_U, ubytes, cudaMemcpyDeviceToHost, st));
  // number of (window, point) entries with a non-zero digit = mixed additions performed
  for (int q = 0; q < nparts; q++)
    ZKB_CUDA(cudaMemcpyAsync(pin + ubytes + 4 * q, ws[q] + P[q].o_off + (size_t)P[q].nseg * 4, 4,
                             cudaMemcpyDeviceToHost, st));
  ZKB_CUDA(cudaStreamSynchronize(st));
  cx.last_msm_entries = 0;
  for (int q = 0; q < nparts; q++) {
    uint32_t e;
    std::memcpy(&e, pin + ubytes + 4 * q, 4);
    cx.last_msm_entries += e;
  }
  cx.last_msm_c = P0.c;
  cx.last_msm_nwin = P0.nwin;
  ZKB_CUDA(cudaEventElapsedTime(&cx.last_kernel_ms, cx.ev_phase[0], cx.ev_phase[4]));
  cx.nphase = 4;
  for (int i = 0; i < 4; i++) ZKB_CUDA(cudaEventElapsedTime(&cx.last_phase_ms[i], cx.ev_phase[i], cx.ev_phase[i + 1]));
  const host::Xyzz<NL> r = msm_host_combine<NL>(F, P0, reinterpret_cast<const uint64_t*>(pin));
  host::xyzz_write<NL>(F, r, kind, tgt);
  return ZKG_OK;
}

// ------------------------------------------------------------------------------ entry

static zkg_status check_msm_args(int n, const void* expos, int nlimbs, int mont, const void* grps, const void* tgt) {
  if (n < 0) return set_status(ZKG_ERR_ARG, "msm", "npoints < 0");
  if (!tgt) return set_status(ZKG_ERR_ARG, "msm", "null tgt");
  if (n > 0 && (!expos || !grps)) return set_status(ZKG_ERR_ARG, "msm", "null input");
  if (nlimbs < 1 || nlimbs > 64) return set_status(ZKG_ERR_ARG, "msm", "expo_nlimbs out of range [1, 64]");
  if (mont && nlimbs != 4)
    return set_status(ZKG_ERR_UNSUPPORTED, "msm", "Montgomery coefficients need expo_nlimbs == 4");
  return ZKG_OK;
}

static int g_tune_parts = env_int("ZKB_MSM_PARTS", 0);
// ZKB_MSM_TRACE=1: the host-buffer MSM prints to stderr when each part's copies and launches
// finished on the device, in ms from the call's start (a timeline for tuning the part layout)
static int g_msm_trace = env_int("ZKB_MSM_TRACE", 0);
// Size ratio of consecutive parts of a pipelined host-buffer MSM (ZKB_MSM_PART_RATIO, in tenths).
// Part q + 1's copy should end when part q's compute does; pinned host->device copies run about
// 1.8-2.2x faster than the MSM consumes points. Default: 3 parts growing 2.2x from 2^20 points,
// 4 parts growing 1.8x from 2^21 (measured at 2^22 with ZKB_MSM_TRACE: 16.25 against 17.2 ms end
// to end; the smaller first part exposes less copy time, the parts' bucket arrays merge in one
// parallel pass).
static int g_part_ratio_env = env_int("ZKB_MSM_PART_RATIO", 0);

// Host buffers. Large MSMs are split into point-range parts: part q's scalars and bases are
// copied on the copy stream while part q-1 sorts and accumulates on the compute stream; one
// bucket reduction then merges the parts' bucket arrays.
// CP is the pipeline's curve type: C itself, or its FP64-product twin (MsmCurve<C>::type).
template <class CP, class C, int NL>
static zkg_status msm_host_run(const host::Field<NL>& F, int n, const uint64_t* expos, int nlimbs, int mont,
                               const uint64_t* grps, int kind, uint64_t* tgt) {
  NvtxRange nvtx("zkb.msm.host_buffers");
  constexpr bool dpf = radix_conv_v<typename CP::Fp>;   // bases converted into the pipeline's radix
  ZKB_TRY(check_msm_args(n, expos, nlimbs, mont, grps, tgt));
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  if (n == 0) {
    host::xyzz_write<NL>(F, host::xyzz_inf<NL>(), kind, tgt);
    return set_status(ZKG_OK, nullptr, nullptr);
  }
  int nparts = g_tune_parts > 0 ? g_tune_parts : (n >= (1 << 21) ? 4 : n >= (1 << 20) ? 3 : n >= (1 << 19) ? 2 : 1);
  nparts = std::max(1, std::min(4, std::min(nparts, n)));
  const double part_ratio = g_part_ratio_env > 0 ? g_part_ratio_env / 10.0 : (nparts == 4 ? 1.8 : 2.2);
  // part boundaries: sizes in geometric progression (the first part's copy is the only one that
  // nothing overlaps, and each later copy hides behind the previous part's compute)
  int pstart[5];
  pstart[0] = 0;
  {
    double w[4], sum = 0.0, acc = 0.0;
    for (int q = 0; q < nparts; q++) sum += (w[q] = q == 0 ? 1.0 : w[q - 1] * part_ratio);
    for (int q = 1; q < nparts; q++) {
      acc += w[q - 1];
      pstart[q] = std::max(pstart[q - 1] + 1, std::min(n - (nparts - q), (int)((double)n * (acc / sum))));
    }
  }
  pstart[nparts] = n;
  const int scalar_bits = mont ? C::SCALAR_BITS : 64 * nlimbs;
  const int c = pick_window(C::ID, n, scalar_bits);
  MsmPlan P[4];
  size_t total = 0, off_s[4], off_b[4], off_w[4], off_c[4];
  auto rup = [](size_t x) { return (x + 255) & ~size_t(255); };
  for (int q = 0; q < nparts; q++) {
    const int nq = pstart[q + 1] - pstart[q];
    ZKB_TRY(make_plan<CP>(nq, nlimbs, mont, P[q], c));
    off_s[q] = total;
    total += rup((size_t)nq * nlimbs * 8);
    off_b[q] = total;
    total += rup((size_t)nq * 2 * NL * 8);
    off_c[q] = total;   // bases in the FP64 pipeline's radix
    if (dpf) total += rup((size_t)nq * 2 * NL * 8);
    off_w[q] = total;
    total += rup(P[q].bytes);
  }
  ZKB_TRY(cx.arena.reserve(total));
  cx.arena.reset();
  char* base = static_cast<char*>(cx.arena.take(total));
  if (!base) return set_status(ZKG_ERR_NOMEM, "msm", "arena");
  const cudaStream_t st = cx.compute();
  // the copy stream must not overwrite the arena before earlier work on the compute stream is done
  ZKB_CUDA(cudaEventRecord(cx.ev_copy, st));
  ZKB_CUDA(cudaStreamWaitEvent(cx.copy_stream, cx.ev_copy, 0));
  char* ws[4];
  PartSet parts;
  parts.n = nparts;
  // trace events: 0 start, then per part scalars copied, bases copied, part's launches done; then
  // the reduction done
  cudaEvent_t tev[3 + 3 * 4] = {nullptr};
  const int ntev = g_msm_trace ? 2 + 3 * nparts : 0;
  for (int k = 0; k < ntev; k++) ZKB_CUDA(cudaEventCreate(&tev[k]));
  if (ntev) ZKB_CUDA(cudaEventRecord(tev[0], st));
  // per part: scalars, then bases, then the part's launches; a part's sort waits only for its
  // scalars, its accumulation for its bases, so the sort runs while the bases are still in
  // flight, and staging the next part's pageable host data overlaps this part's compute
  for (int q = 0; q < nparts; q++) {
    const size_t first = (size_t)pstart[q], nq = P[q].n;
    ZKB_TRY(copy_h2d(cx, base + off_s[q], expos + first * nlimbs, nq * nlimbs * 8, cx.copy_stream));
    ZKB_CUDA(cudaEventRecord(cx.ev_scal[q], cx.copy_stream));
    if (ntev) ZKB_CUDA(cudaEventRecord(tev[1 + 3 * q], cx.copy_stream));
    ZKB_TRY(copy_h2d(cx, base + off_b[q], grps + first * 2 * NL, nq * 2 * NL * 8, cx.copy_stream));
    ZKB_CUDA(cudaEventRecord(cx.ev_part[q], cx.copy_stream));
    if (ntev) ZKB_CUDA(cudaEventRecord(tev[2 + 3 * q], cx.copy_stream));
    ws[q] = base + off_w[q];
    ZKB_CUDA(cudaStreamWaitEvent(st, cx.ev_scal[q], 0));
    ZKB_TRY(msm_launch_part<CP>(cx, P[q], ws[q], reinterpret_cast<const uint64_t*>(base + off_s[q]), mont,
                                reinterpret_cast<const uint64_t*>(base + (dpf ? off_c[q] : off_b[q])), st,
                                cx.ev_part[q], q == 0, q == nparts - 1,
                                dpf ? reinterpret_cast<const uint32_t*>(base + off_b[q]) : nullptr,
                                nparts > 1 ? q : -1));
    parts.bsum[q] = reinterpret_cast<const uint32_t*>(ws[q] + P[q].o_bsum);
    parts.off[q] = reinterpret_cast<const uint32_t*>(ws[q] + P[q].o_off);
    if (ntev) ZKB_CUDA(cudaEventRecord(tev[3 + 3 * q], st));
  }
  if (nparts > 1)   // the bucket reduction reads every part's folded bucket array
    for (int q = 0; q < nparts; q++) ZKB_CUDA(cudaStreamWaitEvent(st, cx.ev_fold[q], 0));
  ZKB_TRY(msm_launch_reduce<CP>(cx, P[0], ws[0], parts, st));
  if (ntev) ZKB_CUDA(cudaEventRecord(tev[ntev - 1], st));
  ZKB_TRY(msm_u_to_radix<CP>(P[0], ws[0], st));
  ZKB_TRY((msm_finish<C, NL>(cx, F, P[0], ws[0], ws, P, nparts, kind, tgt, st)));
  if (ntev) {
    ZKB_CUDA(cudaEventSynchronize(tev[ntev - 1]));
    auto at = [&](int k) { float ms = 0.f; cudaEventElapsedTime(&ms, tev[0], tev[k]); return ms; };
    std::fprintf(stderr, "zkb msm trace n=%d parts=%d:", n, nparts);
    for (int q = 0; q < nparts; q++)
      std::fprintf(stderr, " [part %d: %d points, scalars %.3f bases %.3f launches %.3f]", q,
                   pstart[q + 1] - pstart[q], at(1 + 3 * q), at(2 + 3 * q), at(3 + 3 * q));
    std::fprintf(stderr, " reduced %.3f ms\n", at(ntev - 1));
    for (int k = 0; k < ntev; k++) cudaEventDestroy(tev[k]);
  }
  ZKB_TRY(dev_check_report(cx, "msm"));
  return set_status(ZKG_OK, nullptr, nullptr);
}

template <class C, int NL>
static zkg_status msm_host_entry(const host::Field<NL>& F, int n, const uint64_t* expos, int nlimbs, int mont,
                                 const uint64_t* grps, int kind, uint64_t* tgt) {
  if (g_msm_dpf) return msm_host_run<typename MsmCurve<C>::type, C, NL>(F, n, expos, nlimbs, mont, grps, kind, tgt);
  return msm_host_run<C, C, NL>(F, n, expos, nlimbs, mont, grps, kind, tgt);
}

// Device-resident inputs: one part. pre_converted: d_grps already holds the bases in the
// pipeline's radix (a resident base set), so no conversion runs. h_expos (optional): the scalars
// are in host memory and are copied into the workspace first (d_expos is then ignored).
template <class CP, class C, int NL>
static zkg_status msm_dev_run(const host::Field<NL>& F, int n, const uint64_t* d_expos, int nlimbs, int mont,
                              const uint64_t* d_grps, int kind, uint64_t* tgt, bool pre_converted = false,
                              const uint64_t* h_expos = nullptr) {
  NvtxRange nvtx("zkb.msm.device");
  constexpr bool dpf = radix_conv_v<typename CP::Fp>;   // bases converted into the pipeline's radix
  ZKB_TRY(check_msm_args(n, h_expos ? h_expos : d_expos, nlimbs, mont, d_grps, tgt));
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  if (n == 0) {
    host::xyzz_write<NL>(F, host::xyzz_inf<NL>(), kind, tgt);
    return set_status(ZKG_OK, nullptr, nullptr);
  }
  if (!cx.user_stream) ZKB_CUDA(cudaDeviceSynchronize());   // inputs may come from any stream
  MsmPlan P;
  ZKB_TRY(make_plan<CP>(n, nlimbs, mont, P));
  const bool convert = dpf && !pre_converted;
  const size_t cb = convert ? (((size_t)n * 2 * NL * 8 + 255) & ~size_t(255)) : 0;   // converted bases
  const size_t sb = h_expos ? (((size_t)n * nlimbs * 8 + 255) & ~size_t(255)) : 0;   // copied scalars
  ZKB_TRY(cx.arena.reserve(P.bytes + cb + sb + 512));
  cx.arena.reset();
  char* ws = static_cast<char*>(cx.arena.take(P.bytes));
  char* conv = convert ? static_cast<char*>(cx.arena.take(cb)) : nullptr;
  char* sbuf = h_expos ? static_cast<char*>(cx.arena.take(sb)) : nullptr;
  if (!ws || (convert && !conv) || (h_expos && !sbuf)) return set_status(ZKG_ERR_NOMEM, "msm", "arena");
  const cudaStream_t st = cx.compute();
  if (h_expos) {
    ZKB_TRY(copy_h2d(cx, sbuf, h_expos, (size_t)n * nlimbs * 8, st));
    d_expos = reinterpret_cast<const uint64_t*>(sbuf);
  }
  ZKB_TRY(msm_launch_part<CP>(cx, P, ws, d_expos, mont, convert ? reinterpret_cast<const uint64_t*>(conv) : d_grps,
                              st, nullptr, true, true, convert ? reinterpret_cast<const uint32_t*>(d_grps) : nullptr));
  PartSet parts;
  parts.n = 1;
  parts.bsum[0] = reinterpret_cast<const uint32_t*>(ws + P.o_bsum);
  parts.off[0] = reinterpret_cast<const uint32_t*>(ws + P.o_off);
  ZKB_TRY(msm_launch_reduce<CP>(cx, P, ws, parts, st));
  ZKB_TRY(msm_u_to_radix<CP>(P, ws, st));
  ZKB_TRY((msm_finish<C, NL>(cx, F, P, ws, &ws, &P, 1, kind, tgt, st)));
  ZKB_TRY(dev_check_report(cx, "msm"));
  return set_status(ZKG_OK, nullptr, nullptr);
}

template <class C, int NL>
static zkg_status msm_dev_entry(const host::Field<NL>& F, int n, const uint64_t* d_expos, int nlimbs, int mont,
                                const uint64_t* d_grps, int kind, uint64_t* tgt) {
  if (g_msm_dpf) return msm_dev_run<typename MsmCurve<C>::type, C, NL>(F, n, d_expos, nlimbs, mont, d_grps, kind, tgt);
  return msm_dev_run<C, C, NL>(F, n, d_expos, nlimbs, mont, d_grps, kind, tgt);
}


// =================================================================== batched MSMs (many sizes)
//
// A batch of MSMs against one resident base set (request r uses bases[0, n_r), the KZG pattern of
// committing polynomials of different degrees) runs as ONE segmented pipeline: segments are
// keyed by (request, window, bucket), each request with its own window width. Conversion,
// digits, histogram and scatter find their request by a binary search over the descriptor table;
// the scan, the chunked accumulation and the folding levels run unchanged over all requests'
// segments at once, so small requests share the GPU instead of each under-filling it.

struct MReq {
  const uint64_t* scal_in;   // the request's Montgomery scalars (device), 4 limbs each
  uint32_t pt_off;           // first point in the batch's concatenated standard scalars
  uint32_t n, c, nwin, B;    // points, window width, windows, buckets per window
  uint32_t seg_base;         // first segment
  uint32_t K1, G, gbits;     // running-sum group size, groups per window, log2 G
  uint32_t thr_off;          // first running-sum thread (= first T/R entry)
  uint32_t blk_off;          // first (window, k) reduction block (= first U entry)
  uint32_t rank_base;        // first rank word (window-major per request: base + win n + point)
};

template <int FIELD>
__device__ __forceinline__ uint32_t mreq_key(const MReq& r) {
  return FIELD == 0 ? r.pt_off : (FIELD == 1 ? r.thr_off : r.blk_off);
}
// largest r with key(r) <= x (keys ascending, key(0) = 0)
template <int FIELD>
__device__ __forceinline__ int mreq_find(const MReq* __restrict__ reqs, int nreq, uint32_t x) {
  int lo = 0, hi = nreq;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (mreq_key<FIELD>(reqs[mid]) <= x) lo = mid; else hi = mid;
  }
  return lo;
}

template <class C>
__global__ void k_mmsm_from_mont(const MReq* __restrict__ reqs, int nreq, uint32_t npts, uint32_t* __restrict__ out) {
  using Fr = typename C::Fr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const MReq& q = reqs[mreq_find<0>(reqs, nreq, i)];
  const Fe<Fr> a = fe_load_nc<Fr>(reinterpret_cast<const uint32_t*>(q.scal_in) + 8 * (size_t)(i - q.pt_off));
  fe_store<Fr>(out + 8 * (size_t)i, fe_from_mont(a));
}

// The histogram keeps each entry's rank in its segment (the value its count increment returned),
// so the scatter places entries at offset + rank without atomics.
__global__ void k_mmsm_hist(const MReq* __restrict__ reqs, int nreq, uint32_t npts, const uint32_t* __restrict__ scal,
                            uint32_t* __restrict__ cnt, uint32_t* __restrict__ rank) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const MReq q = reqs[mreq_find<0>(reqs, nreq, i)];
  const uint32_t* w = scal + 8 * (size_t)i;
  uint32_t carry = 0, neg;
  for (int win = 0; win < (int)q.nwin; win++) {
    const uint32_t b = next_digit(w, 8, win, (int)q.c, carry, neg);
    if (b)
      rank[q.rank_base + (size_t)win * q.n + (i - q.pt_off)] =
          atomicAdd(cnt + q.seg_base + (size_t)win * q.B + (b - 1), 1u);
  }
}

__global__ void k_mmsm_scatter(const MReq* __restrict__ reqs, int nreq, uint32_t npts,
                               const uint32_t* __restrict__ scal, const uint32_t* __restrict__ off,
                               const uint32_t* __restrict__ rank, uint32_t* __restrict__ entries) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const MReq q = reqs[mreq_find<0>(reqs, nreq, i)];
  const uint32_t* w = scal + 8 * (size_t)i;
  uint32_t carry = 0, neg;
  for (int win = 0; win < (int)q.nwin; win++) {
    const uint32_t b = next_digit(w, 8, win, (int)q.c, carry, neg);
    if (b) {
      const uint32_t pos = __ldg(off + q.seg_base + (size_t)win * q.B + (b - 1)) +
                           __ldg(rank + q.rank_base + (size_t)win * q.n + (i - q.pt_off));
      entries[pos] = (i - q.pt_off) | (neg << 31);
    }
  }
}

template <class C>
__global__ void __launch_bounds__(128) k_mmsm_bucket_rs(const MReq* __restrict__ reqs, int nreq, uint32_t nthr,
                                                        const uint32_t* __restrict__ bsum,
                                                        const uint32_t* __restrict__ off,
                                                        uint32_t* __restrict__ Tout, uint32_t* __restrict__ Rout) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nthr) return;
  const MReq q = reqs[mreq_find<1>(reqs, nreq, t)];
  const uint32_t tl = t - q.thr_off, w = tl / q.G, g = tl % q.G;
  Xyzz<F> T = xyzz_inf<F>(), R = xyzz_inf<F>();
  for (int l = (int)q.K1 - 1; l >= 0; l--) {
    const size_t s = q.seg_base + (size_t)w * q.B + (size_t)g * q.K1 + l;
    if (__ldg(off + s) != __ldg(off + s + 1)) xyzz_add_paired(T, xyzz_load<F>(bsum + s * XW));
    xyzz_add_paired(R, T);
  }
  xyzz_store<F>(Tout + (size_t)t * XW, T);
  xyzz_store<F>(Rout + (size_t)t * XW, R);
}

template <class C>
__global__ void __launch_bounds__(256) k_mmsm_bucket_bits(const MReq* __restrict__ reqs, int nreq,
                                                          const uint32_t* __restrict__ Tin,
                                                          const uint32_t* __restrict__ Rin, uint32_t* __restrict__ U) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  extern __shared__ uint4 smem_u4[];
  uint32_t* sm = reinterpret_cast<uint32_t*>(smem_u4);
  const uint32_t b = blockIdx.x;
  const MReq q = reqs[mreq_find<2>(reqs, nreq, b)];
  const uint32_t bl = b - q.blk_off, w = bl / (q.gbits + 1), k = bl % (q.gbits + 1);
  Xyzz<F> acc = xyzz_inf<F>();
  for (uint32_t g = threadIdx.x; g < q.G; g += blockDim.x) {
    const size_t idx = (size_t)q.thr_off + (size_t)w * q.G + g;
    if (k < q.gbits) {
      if ((g >> k) & 1u) xyzz_add_paired(acc, xyzz_load<F>(Tin + idx * XW));
    } else {
      xyzz_add_paired(acc, xyzz_load<F>(Rin + idx * XW));
    }
  }
  xyzz_store<F>(sm + threadIdx.x * XW, acc);
  __syncthreads();
  for (uint32_t half = blockDim.x >> 1; half > 0; half >>= 1) {
    if (threadIdx.x < half) {
      Xyzz<F> a = xyzz_load<F>(sm + threadIdx.x * XW);
      xyzz_add_paired(a, xyzz_load<F>(sm + (threadIdx.x + half) * XW));
      xyzz_store<F>(sm + threadIdx.x * XW, a);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) xyzz_store<F>(U + (size_t)b * XW, xyzz_canon(xyzz_load<F>(sm)));
}

// ------------------------------------------------------------------------- batch plan

struct MultiPlan {
  std::vector<MReq> reqs;     // descriptors of the non-empty requests
  std::vector<int> owner;     // batch MSM index of each descriptor
  uint32_t npts = 0, nseg = 0, nthr = 0, nblk = 0;
  uint64_t total_max = 0;
  int L1 = 128, nlev = 0;
  uint32_t Llev[MAX_LEVELS];
  uint64_t Ylev[MAX_LEVELS];
  uint32_t nch[MAX_LEVELS + 1];
  size_t o_std, o_cnt, o_off, o_cur, o_bs, o_ent, o_keyA, o_ptA, o_keyB, o_ptB, o_bsum, o_T, o_R, o_U, o_reqs, bytes;
  size_t o_rank = 0;          // entry ranks (total_max words)
};

template <class C>
static zkg_status make_multi_plan(const std::vector<int>& ns, const std::vector<const uint64_t*>& scal, MultiPlan& M) {
  using F = typename C::Fp;
  constexpr size_t XB = 16 * F::N;
  M = MultiPlan();
  for (size_t i = 0; i < ns.size(); i++) {
    if (ns[i] <= 0) continue;
    MReq q;
    q.scal_in = scal[i];
    q.n = (uint32_t)ns[i];
    q.c = (uint32_t)pick_window(C::ID, ns[i], C::SCALAR_BITS);
    q.nwin = (C::SCALAR_BITS + 1 + q.c - 1) / q.c;
    q.B = 1u << (q.c - 1);
    // the batch as a whole fills the GPU: work-efficient groups of 32 for every request
    q.K1 = std::min<uint32_t>(q.B, g_tune_K1 > 0 ? (uint32_t)g_tune_K1 : 32u);
    q.G = q.B / q.K1;
    q.gbits = (uint32_t)ilog2_floor(q.G);
    q.pt_off = M.npts;
    q.seg_base = M.nseg;
    q.thr_off = M.nthr;
    q.blk_off = M.nblk;
    q.rank_base = (uint32_t)M.total_max;   // < 2^31, checked below for the running total
    const uint64_t np = (uint64_t)M.npts + q.n, ns_ = (uint64_t)M.nseg + (uint64_t)q.nwin * q.B;
    if (np >= (1ull << 31) || ns_ >= (1ull << 30)) return set_status(ZKG_ERR_ARG, "batch", "batch too large");
    M.npts = (uint32_t)np;
    M.nseg = (uint32_t)ns_;
    M.nthr += q.nwin * q.G;
    M.nblk += q.nwin * (q.gbits + 1);
    M.total_max += (uint64_t)q.nwin * q.n;
    M.reqs.push_back(q);
    M.owner.push_back((int)i);
  }
  if (M.reqs.empty()) return ZKG_OK;
  if (M.total_max >= (1ull << 31)) return set_status(ZKG_ERR_ARG, "batch", "too many (window, point) entries");
  M.L1 = (int)chunk_len(M.total_max, accum_wave<C>());
  M.nch[0] = (uint32_t)std::max<uint64_t>(1, (M.total_max + M.L1 - 1) / M.L1);
  uint64_t Y = 2ull * M.nch[0];
  uint32_t prev = M.nch[0];
  while (prev > 1) {
    if (M.nlev >= MAX_LEVELS - 1) return set_status(ZKG_ERR_ARG, "batch", "level overflow");
    M.Llev[M.nlev] = 16;
    M.Ylev[M.nlev] = Y;
    const uint32_t ch = (uint32_t)((Y + 15) / 16);
    M.nch[++M.nlev] = ch;
    Y = 2ull * ch;
    prev = ch;
  }
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o = (o + bytes + 255) & ~size_t(255); return r; };
  M.o_std = take((size_t)M.npts * 32);
  M.o_cnt = take((size_t)M.nseg * 4 + 4);
  M.o_off = take((size_t)M.nseg * 4 + 4);
  M.o_cur = take((size_t)M.nseg * 4 + 4);
  const uint32_t nb = (M.nseg + SCAN_T * SCAN_E - 1) / (SCAN_T * SCAN_E);
  if (nb > (uint32_t)SCAN_T * SCAN_E) return set_status(ZKG_ERR_ARG, "batch", "too many buckets");
  M.o_bs = take((size_t)nb * 4 + 4);
  M.o_ent = take((size_t)M.total_max * 4 + 4);
  M.o_rank = take((size_t)M.total_max * 4 + 4);
  uint64_t slotsA = 2ull * M.nch[0], slotsB = 0;
  for (int k = 1; k <= M.nlev; k++) {
    if (k % 2 == 1) slotsB = std::max<uint64_t>(slotsB, 2ull * M.nch[k]);
    else slotsA = std::max<uint64_t>(slotsA, 2ull * M.nch[k]);
  }
  M.o_keyA = take(slotsA * 4);
  M.o_ptA = take(slotsA * XB);
  M.o_keyB = take(slotsB * 4 + 4);
  M.o_ptB = take(slotsB * XB + 4);
  M.o_bsum = take((size_t)M.nseg * XB);
  M.o_T = take((size_t)M.nthr * XB);
  M.o_R = take((size_t)M.nthr * XB);
  M.o_U = take((size_t)M.nblk * XB);
  M.o_reqs = take(M.reqs.size() * sizeof(MReq));
  M.bytes = o;
  return ZKG_OK;
}

// Enqueue the whole batch pipeline on st (capturable: no host synchronisation); the descriptor
// table must already be in ws + o_reqs. phase: 0 all, 1 up to the sorted entries (the
// accumulation then runs elsewhere: the batch's persistent kernel), 2 from the merge on.
template <class C>
static zkg_status multi_msm_launch(const MultiPlan& M, char* ws, const uint64_t* d_bases, cudaStream_t st,
                                   int phase = 0) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  auto U32 = [&](size_t o) { return reinterpret_cast<uint32_t*>(ws + o); };
  const MReq* reqs = reinterpret_cast<const MReq*>(ws + M.o_reqs);
  const int nreq = (int)M.reqs.size();
  const dim3 gp((M.npts + 255) / 256);
  const uint32_t* bases = reinterpret_cast<const uint32_t*>(d_bases);
  const uint32_t* ent = U32(M.o_ent);
  const uint32_t* off = U32(M.o_off);
  if (phase != 2) {
  ZKB_TRY(launch("mmsm_from_mont", k_mmsm_from_mont<C>, gp, dim3(256), 0, st, reqs, nreq, M.npts, U32(M.o_std)));
  ZKB_CUDA(cudaMemsetAsync(U32(M.o_cnt), 0, (size_t)M.nseg * 4, st));
  ZKB_TRY(launch("mmsm_hist", k_mmsm_hist, gp, dim3(256), 0, st, reqs, nreq, M.npts, (const uint32_t*)U32(M.o_std),
                 U32(M.o_cnt), U32(M.o_rank)));
  const uint32_t nb = (M.nseg + SCAN_T * SCAN_E - 1) / (SCAN_T * SCAN_E);
  ZKB_TRY(launch("scan_blocks", k_scan_blocks, dim3(nb), dim3(SCAN_T), 0, st, (const uint32_t*)U32(M.o_cnt),
                 U32(M.o_off), U32(M.o_bs), M.nseg));
  ZKB_TRY(launch("scan_top", k_scan_top, dim3(1), dim3(SCAN_T), 0, st, U32(M.o_bs), nb));
  ZKB_TRY(launch("scan_add", k_scan_add, dim3((M.nseg + 255) / 256), dim3(256), 0, st, U32(M.o_off),
                 U32(M.o_cur), (const uint32_t*)U32(M.o_bs), M.nseg, nb));
  ZKB_TRY(launch("mmsm_scatter", k_mmsm_scatter, gp, dim3(256), 0, st, reqs, nreq, M.npts,
                 (const uint32_t*)U32(M.o_std), (const uint32_t*)U32(M.o_off), (const uint32_t*)U32(M.o_rank),
                 U32(M.o_ent)));
  if (phase == 1) return ZKG_OK;
  ZKB_TRY(launch_accum<C>(M.nch[0], st, ent, off, M.nseg, (uint32_t)M.L1, bases, U32(M.o_bsum), U32(M.o_keyA),
                          U32(M.o_ptA)));
  }
  ZKB_TRY(launch("mmsm_pair_merge", k_msm_pair_merge<C>, dim3((M.nch[0] + 255) / 256), dim3(256), 0, st, off, M.nch[0], (uint32_t)M.L1,
                 U32(M.o_keyA), (const uint32_t*)U32(M.o_ptA), U32(M.o_bsum), (uint32_t*)nullptr, M.nseg));
  LevelHist hist;
  hist.n = 1;
  hist.L[0] = (uint32_t)M.L1;
  for (int k = 0; k < M.nlev; k++) {
    const bool fromA = (k % 2 == 0);
    const uint32_t ch = M.nch[k + 1];
    ZKB_TRY(launch("mmsm_seg_level", k_msm_seg_level<C>, dim3((ch + 255) / 256), dim3(256), 0, st,
                   (const uint32_t*)U32(fromA ? M.o_keyA : M.o_keyB), (const uint32_t*)U32(fromA ? M.o_ptA : M.o_ptB),
                   (uint32_t)M.Ylev[k], M.Llev[k], ch, hist, off, U32(M.o_bsum), U32(fromA ? M.o_keyB : M.o_keyA),
                   U32(fromA ? M.o_ptB : M.o_ptA)));
    hist.L[hist.n++] = M.Llev[k];
  }
  ZKB_TRY(launch("mmsm_bucket_rs", k_mmsm_bucket_rs<C>, dim3((M.nthr + 127) / 128), dim3(128), 0, st, reqs, nreq,
                 M.nthr, (const uint32_t*)U32(M.o_bsum), off, U32(M.o_T), U32(M.o_R)));
  ZKB_TRY(launch("mmsm_bucket_bits", k_mmsm_bucket_bits<C>, dim3(M.nblk), dim3(256), (size_t)256 * XW * 4, st, reqs,
                 nreq, (const uint32_t*)U32(M.o_T), (const uint32_t*)U32(M.o_R), U32(M.o_U)));
  return ZKG_OK;
}

// Host tails of a finished batch (U copied to host), spread over CPU threads.
template <int NL>
static void multi_msm_tails(const host::Field<NL>& F, const MultiPlan& M, const uint64_t* U,
                            const std::vector<uint64_t*>& outs, const std::vector<int>& kinds) {
  const int nreq = (int)M.reqs.size();
  auto work = [&](int lo, int hi) {
    for (int r = lo; r < hi; r++) {
      const MReq& q = M.reqs[r];
      MsmPlan P;
      P.c = (int)q.c;
      P.nwin = (int)q.nwin;
      P.gbits = (int)q.gbits;
      P.K1 = q.K1;
      const host::Xyzz<NL> res = msm_host_combine<NL>(F, P, U + (size_t)q.blk_off * 4 * NL);
      host::xyzz_write<NL>(F, res, kinds[M.owner[r]], outs[M.owner[r]]);
    }
  };
  const int hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const int nt = std::min(hw, nreq);
  if (nt <= 1) { work(0, nreq); return; }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++) th.emplace_back(work, nreq * t / nt, nreq * (t + 1) / nt);
  for (auto& x : th) x.join();
}

// The batch's persistent kernel (k_batch_work) and its work-queue types: zkb_batch_work.cu / .h.
// ZKB_BATCH_PERSISTENT=1 makes it the default form of a batch. The default is graph branches: on
// B200 the separate launches measured faster for the mixed batch of 64 MSMs (2^10-2^20 points)
// and 64 NTTs (2^12-2^22), 48.3 against 53.4 ms, because the bucket accumulation runs best as
// one 384-thread block per SM (168 registers) while the kernel that also runs NTT tiles needs
// 256-thread blocks, whose accumulation spills and issues 7% more instructions per addition.
static int g_batch_persistent = env_int("ZKB_BATCH_PERSISTENT", 0);

}  // namespace zkb

// ------------------------------------------------------------------ resident base set

// A base set uploaded once and kept on the device in the form the bucket pipeline reads (the
// reference's own layout and radix for the FP64 pipeline of exact-radix products; converted once
// here when a pipeline keeps another radix). The handle owns its device memory.
struct zkg_bases {
  int curve = 0;
  int n = 0;
  int dev = 0;
  bool converted = false;      // d_pts is in the FP64 pipeline's form (runs on that pipeline)
  uint64_t* d_pts = nullptr;   // n affine points, 2 * NLIMBS_P limbs each
  ~zkg_bases() {
    if (d_pts) cudaFree(d_pts);
  }
};

// ----------------------------------------------------------------------- batch object

struct zkg_batch {
  int curve = 0;
  const uint64_t* d_bases = nullptr;
  int n_bases = 0;
  bool bases_converted = false;   // d_bases already in the FP64 pipeline's radix (resident base set)
  struct Msm { int n; const uint64_t* d_scal; uint64_t* out; int kind; };
  struct Ntt { int m; uint64_t gen[4]; const uint64_t* d_src; uint64_t* d_tgt; int inverse; };
  std::vector<Msm> msms;
  std::vector<Ntt> ntts;
  bool built = false;
  zkb::MultiPlan mp;
  std::vector<zkb::NttPlan*> plans;
  void* ws = nullptr;           // device workspace (MSM pipeline + NTT scratch)
  size_t conv_off = 0;          // bases in the FP64 pipeline's radix (inside ws), 0 = integer pipeline
  uint32_t conv_n = 0;          // bases converted per run (largest request)
  void* pin = nullptr;          // pinned copy of U
  size_t ubytes = 0;
  std::vector<size_t> ntt_scratch_off;
  cudaStream_t s_main = nullptr;
  std::vector<cudaStream_t> s_ntt;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> ev_fork;
  float last_ms = 0.f;
  // persistent mode: the accumulation and every NTT pass in one launch (k_batch_work)
  bool persistent = false;
  uint32_t wait_limit = 1u << 24;   // polls of a pass-dependency wait (~2 s) before ZKG_ERR_TIMEOUT
  bool inject_stall = false;        // testing: one pass waits for a tile that never comes
  bool persistent_wanted = true;    // build the persistent form (ZKB_BATCH_PERSISTENT / zkg_batch_set_mode)
  size_t err_pin_off = 0;           // error word's copy inside pin
  int work_grid = 0;
  uint32_t work_tasks = 0;
  ~zkg_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto p : plans) delete p;
    if (ws) cudaFree(ws);
    if (pin) cudaFreeHost(pin);
    for (auto s : s_ntt) cudaStreamDestroy(s);
    if (s_main) cudaStreamDestroy(s_main);
    for (auto e : ev_fork) cudaEventDestroy(e);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

namespace zkb {

// Persistent-kernel form of a batch (FP64 pipelines): one graph of the MSM sort launches, one
// k_batch_work launch (accumulation + all NTT passes), then the MSM merge / fold / reduction.
template <class C, int NL>
static zkg_status batch_build_persistent(zkg_batch* b, const host::Field<NL>& F) {
  using CD = typename MsmCurve<C>::type;
  std::vector<int> ns;
  std::vector<const uint64_t*> sc;
  for (auto& m : b->msms) { ns.push_back(m.n); sc.push_back(m.d_scal); }
  ZKB_TRY(make_multi_plan<CD>(ns, sc, b->mp));
  ZKB_CUDA(cudaStreamCreateWithFlags(&b->s_main, cudaStreamNonBlocking));
  for (size_t i = 0; i < b->ntts.size(); i++) {
    NttPlan* pl = nullptr;
    ZKB_TRY(ntt_plan_new(b->curve, b->ntts[i].m, b->ntts[i].gen, b->ntts[i].inverse, 0, b->s_main, &pl));
    b->plans.push_back(pl);
    if (!pl->dpf) return set_status(ZKG_ERR_UNSUPPORTED, "batch", "persistent mode needs FP64 NTT plans");
  }
  auto rup = [](size_t x) { return (x + 255) & ~size_t(255); };
  size_t total = rup(b->mp.bytes);
  std::vector<size_t> scr(b->ntts.size(), 0);   // one scratch vector per NTT (they all run at once)
  for (size_t i = 0; i < b->ntts.size(); i++)
    if (b->plans[i]->passes.size() >= 2) { scr[i] = total; total += rup((size_t)32 << b->ntts[i].m); }
  if (radix_conv_v<typename CD::Fp> && !b->mp.reqs.empty() && !b->bases_converted) {   // converted every run
    for (auto& m : b->msms) b->conv_n = std::max<uint32_t>(b->conv_n, (uint32_t)m.n);
    b->conv_off = total;
    total += rup((size_t)b->conv_n * 2 * NL * 8);
  }
  // pass descriptors and the task queue
  std::vector<NttPassDesc> descs;
  std::vector<std::vector<int>> by_step;   // descriptor indices by pass step (0 = first pass)
  char* ws = nullptr;
  const size_t ws_descs_placeholder = 0;
  (void)ws_descs_placeholder;
  for (size_t i = 0; i < b->ntts.size(); i++) {
    const NttPlan& pl = *b->plans[i];
    const int np = (int)pl.passes.size();
    int prev = -1;
    for (int e = 0; e < np; e++) {
      const NttPass& q = pl.inverse ? pl.passes[np - 1 - e] : pl.passes[e];
      NttPassDesc d;
      d.m = pl.m;
      d.K = q.k;
      d.Mp = q.Mp;
      d.s = q.s;
      d.W = NTT_THREADS * std::min(8, 1 << q.k) >> q.k;
      d.ntiles = (uint32_t)((((size_t)1 << (pl.m - q.k)) + d.W - 1) / d.W);
      d.inverse = pl.inverse;
      d.om = pl.d_om[q.k];
      d.tw = q.Mp > 0 ? pl.d_tw : nullptr;
      d.scale = nullptr;
      if (pl.inverse && e == np - 1) {
        if (d.tw && pl.d_tw_last) d.tw = pl.d_tw_last;
        else d.scale = pl.d_scale;
      }
      // pointers into ws are filled in below (offsets for now: in = previous output)
      d.in = nullptr;
      d.out = nullptr;
      d.dep = prev;
      d.dep_count = prev >= 0 ? descs[prev].ntiles : 0;
      if ((int)by_step.size() <= e) by_step.resize(e + 1);
      by_step[e].push_back((int)descs.size());
      prev = (int)descs.size();
      descs.push_back(d);
    }
  }
  if (b->inject_stall) {   // testing: the first dependent pass waits for one tile too many
    for (auto& d : descs)
      if (d.dep >= 0) { d.dep_count += 1; break; }
  }
  const uint32_t bt = (uint32_t)batch_work_threads(b->curve);   // chunks per accumulation task
  const uint32_t nacc = b->mp.reqs.empty() ? 0u : (b->mp.nch[0] + bt - 1) / bt;
  // queue: the tiles of pass step e, then a share of the accumulation blocks, for every step; the
  // accumulation between two steps covers the time the earlier step's tiles take to finish, so a
  // later step's tiles rarely wait, and the queue ends with accumulation work that fills every SM
  std::vector<uint2> tasks;
  const size_t nsteps = std::max<size_t>(1, by_step.size());
  uint32_t acc_next = 0;
  for (size_t e = 0; e < nsteps; e++) {
    if (e < by_step.size())
      for (int di : by_step[e])
        for (uint32_t t = 0; t < descs[di].ntiles; t++) tasks.push_back(make_uint2((uint32_t)di + 1, t));
    const uint32_t acc_end = (uint32_t)(((uint64_t)nacc * (e + 1)) / nsteps);
    for (; acc_next < acc_end; acc_next++) tasks.push_back(make_uint2(0u, acc_next));
  }
  b->work_tasks = (uint32_t)tasks.size();
  const size_t o_tasks = total;
  total += rup(std::max<size_t>(1, tasks.size()) * sizeof(uint2));
  const size_t o_descs = total;
  total += rup(std::max<size_t>(1, descs.size()) * sizeof(NttPassDesc));
  const size_t o_done = total;
  total += rup((descs.size() + 2) * 4);   // done[ndesc], next, error
  ZKB_CUDA(cudaMalloc(&b->ws, total));
  ws = static_cast<char*>(b->ws);
  // buffer pointers: pass e of NTT i reads its input (first pass) or the previous pass's output,
  // and writes tgt when (np - 1 - e) is even, the NTT's scratch otherwise
  {
    size_t di = 0;
    for (size_t i = 0; i < b->ntts.size(); i++) {
      const int np = (int)b->plans[i]->passes.size();
      const uint32_t* in = reinterpret_cast<const uint32_t*>(b->ntts[i].d_src);
      for (int e = 0; e < np; e++, di++) {
        uint32_t* out = ((np - 1 - e) % 2 == 0) ? reinterpret_cast<uint32_t*>(b->ntts[i].d_tgt)
                                                : reinterpret_cast<uint32_t*>(ws + scr[i]);
        descs[di].in = in;
        descs[di].out = out;
        in = out;
      }
    }
  }
  if (!tasks.empty())
    ZKB_CUDA(cudaMemcpy(ws + o_tasks, tasks.data(), tasks.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  if (!descs.empty())
    ZKB_CUDA(cudaMemcpy(ws + o_descs, descs.data(), descs.size() * sizeof(NttPassDesc), cudaMemcpyHostToDevice));
  if (!b->mp.reqs.empty())
    ZKB_CUDA(cudaMemcpy(ws + b->mp.o_reqs, b->mp.reqs.data(), b->mp.reqs.size() * sizeof(MReq), cudaMemcpyHostToDevice));
  b->ubytes = (size_t)b->mp.nblk * 4 * NL * 8;
  b->err_pin_off = rup(b->ubytes);
  ZKB_CUDA(cudaMallocHost(&b->pin, b->err_pin_off + 64));
  ZKB_CUDA(cudaEventCreate(&b->ev0));
  ZKB_CUDA(cudaEventCreate(&b->ev1));
  // launch shape: every CTA that fits the GPU at once (the kernel loops over the queue)
  int per_sm = 1;
  ZKB_TRY(batch_work_prepare(b->curve, &per_sm));
  b->work_grid = std::max(1, per_sm) * std::max(1, device_sm_count());
  if ((uint32_t)b->work_grid > b->work_tasks) b->work_grid = (int)std::max<uint32_t>(1, b->work_tasks);
  BatchWork W;
  W.tasks = reinterpret_cast<const uint2*>(ws + o_tasks);
  W.ntasks = b->work_tasks;
  W.done = reinterpret_cast<uint32_t*>(ws + o_done);
  W.next = W.done + descs.size();
  W.error = W.next + 1;
  W.descs = reinterpret_cast<const NttPassDesc*>(ws + o_descs);
  W.wait_limit = b->wait_limit;
  const uint64_t* msm_bases = b->d_bases;
  if (!b->mp.reqs.empty()) {
    W.ent = reinterpret_cast<const uint32_t*>(ws + b->mp.o_ent);
    W.off = reinterpret_cast<const uint32_t*>(ws + b->mp.o_off);
    W.nseg = b->mp.nseg;
    W.nch = b->mp.nch[0];
    W.L = (uint32_t)b->mp.L1;
    if (b->conv_off) msm_bases = reinterpret_cast<const uint64_t*>(ws + b->conv_off);
    W.bases = reinterpret_cast<const uint32_t*>(msm_bases);
    W.bsum = reinterpret_cast<uint32_t*>(ws + b->mp.o_bsum);
    W.key = reinterpret_cast<uint32_t*>(ws + b->mp.o_keyA);
    W.pt = reinterpret_cast<uint32_t*>(ws + b->mp.o_ptA);
  } else {
    W.ent = W.off = W.bases = nullptr;
    W.nseg = W.nch = W.L = 0;
    W.bsum = W.key = W.pt = nullptr;
  }
  auto enqueue = [&]() -> zkg_status {
    const cudaStream_t st = b->s_main;
    ZKB_CUDA(cudaMemsetAsync(W.done, 0, (descs.size() + 2) * 4, st));
    for (size_t i = 0; i < b->ntts.size(); i++)   // m = 0: a copy (bn128_poly_mont.c:420-423)
      if (b->plans[i]->passes.empty())
        ZKB_CUDA(cudaMemcpyAsync(b->ntts[i].d_tgt, b->ntts[i].d_src, 32, cudaMemcpyDeviceToDevice, st));
    if (!b->mp.reqs.empty()) {
      if (b->conv_off)
        ZKB_TRY(launch("msm_bases_to_dpf", k_msm_bases_to_dpf<CD>, dim3((b->conv_n + 255) / 256), dim3(256), 0, st,
                       b->conv_n, reinterpret_cast<const uint32_t*>(b->d_bases), dpf_kin<CD>(),
                       reinterpret_cast<uint32_t*>(ws + b->conv_off)));
      ZKB_TRY(multi_msm_launch<CD>(b->mp, ws, msm_bases, st, 1));
    }
    // level-1 slot keys start as "unused": if a run stops early (a wait ran out), the merge and
    // fold kernels after it then find no slot of an accumulation block that never ran
    if (!b->mp.reqs.empty()) ZKB_CUDA(cudaMemsetAsync(W.key, 0xff, (size_t)2 * W.nch * 4, st));
    if (b->work_tasks)
      ZKB_TRY(batch_work_launch(b->curve, W, b->work_grid, st));
    if (!b->mp.reqs.empty()) {
      ZKB_TRY(multi_msm_launch<CD>(b->mp, ws, msm_bases, st, 2));
      if constexpr (radix_conv_v<typename CD::Fp>)
        ZKB_TRY(launch("msm_xyzz_from_dpf", k_msm_xyzz_from_dpf<CD>, dim3((4 * b->mp.nblk + 255) / 256), dim3(256),
                       0, st, (uint32_t)b->mp.nblk, reinterpret_cast<uint32_t*>(ws + b->mp.o_U), dpf_kout<CD>()));
      ZKB_CUDA(cudaMemcpyAsync(b->pin, ws + b->mp.o_U, b->ubytes, cudaMemcpyDeviceToHost, st));
    }
    ZKB_CUDA(cudaMemcpyAsync(static_cast<char*>(b->pin) + b->err_pin_off, W.error, 4, cudaMemcpyDeviceToHost, st));
    return ZKG_OK;
  };
  ZKB_TRY(enqueue());   // an uncaptured run first (module loading, kernel attributes)
  ZKB_CUDA(cudaStreamSynchronize(b->s_main));
  ZKB_CUDA(cudaStreamBeginCapture(b->s_main, cudaStreamCaptureModeRelaxed));
  zkg_status st = enqueue();
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->s_main, &g);
  if (st != ZKG_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (e != cudaSuccess) return set_status(ZKG_ERR_CUDA, "cudaStreamEndCapture", cudaGetErrorString(e));
  b->graph = g;
  ZKB_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->persistent = true;
  b->built = true;
  return ZKG_OK;
}

template <class C, int NL>
static zkg_status batch_build(zkg_batch* b, const host::Field<NL>& F) {
  if (b->persistent_wanted && g_msm_dpf) return batch_build_persistent<C, NL>(b, F);
  std::vector<int> ns;
  std::vector<const uint64_t*> sc;
  for (auto& m : b->msms) { ns.push_back(m.n); sc.push_back(m.d_scal); }
  ZKB_TRY(make_multi_plan<C>(ns, sc, b->mp));
  // NTT plans owned by the batch, and one scratch region per NTT stream
  const int nstreams = (int)std::min<size_t>(8, std::max<size_t>(1, b->ntts.size()));
  ZKB_CUDA(cudaStreamCreateWithFlags(&b->s_main, cudaStreamNonBlocking));
  for (int i = 0; i < nstreams; i++) {
    cudaStream_t s;
    ZKB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b->s_ntt.push_back(s);
  }
  std::vector<size_t> maxN(nstreams, 0);
  for (size_t i = 0; i < b->ntts.size(); i++) {
    NttPlan* pl = nullptr;
    ZKB_TRY(ntt_plan_new(b->curve, b->ntts[i].m, b->ntts[i].gen, b->ntts[i].inverse, 0, b->s_main, &pl));
    b->plans.push_back(pl);
    maxN[i % nstreams] = std::max(maxN[i % nstreams], (size_t)1 << b->ntts[i].m);
  }
  size_t total = (b->mp.bytes + 255) & ~size_t(255);
  for (int i = 0; i < nstreams; i++) {
    b->ntt_scratch_off.push_back(total);
    total += (maxN[i] * 32 + 255) & ~size_t(255);
  }
  using CD = typename MsmCurve<C>::type;
  if (g_msm_dpf && radix_conv_v<typename CD::Fp> && !b->mp.reqs.empty() && !b->bases_converted) {
    // the bases, converted inside every run (their contents may change); a resident base set
    // was converted once when it was uploaded
    for (auto& m : b->msms) b->conv_n = std::max<uint32_t>(b->conv_n, (uint32_t)m.n);
    b->conv_off = total;
    total += ((size_t)b->conv_n * 2 * NL * 8 + 255) & ~size_t(255);
  }
  ZKB_CUDA(cudaMalloc(&b->ws, std::max<size_t>(total, 256)));
  char* ws = static_cast<char*>(b->ws);
  if (!b->mp.reqs.empty())
    ZKB_CUDA(cudaMemcpy(ws + b->mp.o_reqs, b->mp.reqs.data(), b->mp.reqs.size() * sizeof(MReq), cudaMemcpyHostToDevice));
  b->ubytes = (size_t)b->mp.nblk * 4 * NL * 8;
  ZKB_CUDA(cudaMallocHost(&b->pin, std::max<size_t>(b->ubytes, 64)));
  ZKB_CUDA(cudaEventCreate(&b->ev0));
  ZKB_CUDA(cudaEventCreate(&b->ev1));
  for (int i = 0; i <= nstreams; i++) {
    cudaEvent_t e;
    ZKB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev_fork.push_back(e);
  }
  // set kernel attributes (shared memory limits) outside capture by running once uncaptured
  auto enqueue = [&](bool) -> zkg_status {
    ZKB_CUDA(cudaEventRecord(b->ev_fork[nstreams], b->s_main));
    for (int i = 0; i < nstreams; i++) ZKB_CUDA(cudaStreamWaitEvent(b->s_ntt[i], b->ev_fork[nstreams], 0));
    for (size_t i = 0; i < b->ntts.size(); i++) {
      const int si = (int)(i % nstreams);
      ZKB_TRY(ntt_plan_execute(*b->plans[i], reinterpret_cast<const uint32_t*>(b->ntts[i].d_src),
                               reinterpret_cast<uint32_t*>(b->ntts[i].d_tgt),
                               reinterpret_cast<uint32_t*>(ws + b->ntt_scratch_off[si]), b->s_ntt[si]));
    }
    if (!b->mp.reqs.empty()) {
      if (b->conv_off) {
        Fe<typename CD::Fp> kin, kout;
        dpf_consts_for<CD>(kin, kout);
        uint32_t* conv = reinterpret_cast<uint32_t*>(ws + b->conv_off);
        ZKB_TRY(launch("msm_bases_to_dpf", k_msm_bases_to_dpf<CD>, dim3((b->conv_n + 255) / 256), dim3(256), 0,
                       b->s_main, b->conv_n, reinterpret_cast<const uint32_t*>(b->d_bases), kin, conv));
        ZKB_TRY(multi_msm_launch<CD>(b->mp, ws, reinterpret_cast<const uint64_t*>(conv), b->s_main));
        ZKB_TRY(launch("msm_xyzz_from_dpf", k_msm_xyzz_from_dpf<CD>, dim3((4 * b->mp.nblk + 255) / 256), dim3(256), 0,
                       b->s_main, (uint32_t)b->mp.nblk, reinterpret_cast<uint32_t*>(ws + b->mp.o_U), kout));
      } else if (g_msm_dpf) {   // bases already in the pipeline's form
        ZKB_TRY(multi_msm_launch<CD>(b->mp, ws, b->d_bases, b->s_main));
        if constexpr (radix_conv_v<typename CD::Fp>)
          ZKB_TRY(launch("msm_xyzz_from_dpf", k_msm_xyzz_from_dpf<CD>, dim3((4 * b->mp.nblk + 255) / 256), dim3(256),
                         0, b->s_main, (uint32_t)b->mp.nblk, reinterpret_cast<uint32_t*>(ws + b->mp.o_U),
                         dpf_kout<CD>()));
      } else {
        ZKB_TRY(multi_msm_launch<C>(b->mp, ws, b->d_bases, b->s_main));
      }
      ZKB_CUDA(cudaMemcpyAsync(b->pin, ws + b->mp.o_U, b->ubytes, cudaMemcpyDeviceToHost, b->s_main));
    }
    for (int i = 0; i < nstreams; i++) {
      ZKB_CUDA(cudaEventRecord(b->ev_fork[i], b->s_ntt[i]));
      ZKB_CUDA(cudaStreamWaitEvent(b->s_main, b->ev_fork[i], 0));
    }
    return ZKG_OK;
  };
  ZKB_TRY(enqueue(false));
  ZKB_CUDA(cudaStreamSynchronize(b->s_main));
  ZKB_CUDA(cudaStreamBeginCapture(b->s_main, cudaStreamCaptureModeRelaxed));
  zkg_status st = enqueue(true);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->s_main, &g);
  if (st != ZKG_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (e != cudaSuccess) return set_status(ZKG_ERR_CUDA, "cudaStreamEndCapture", cudaGetErrorString(e));
  b->graph = g;
  ZKB_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->built = true;
  return ZKG_OK;
}

template <class C, int NL>
static zkg_status batch_run(zkg_batch* b, const host::Field<NL>& F) {
  NvtxRange nvtx("zkb.batch.run");
  if (!b->built) ZKB_TRY((batch_build<C, NL>(b, F)));
  ZKB_CUDA(cudaDeviceSynchronize());   // inputs may come from any stream
  ZKB_CUDA(cudaEventRecord(b->ev0, b->s_main));
  ZKB_CUDA(cudaGraphLaunch(b->exec, b->s_main));
  g_launches.fetch_add(1, std::memory_order_relaxed);
  ZKB_CUDA(cudaEventRecord(b->ev1, b->s_main));
  ZKB_CUDA(cudaStreamSynchronize(b->s_main));
  ZKB_CUDA(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
  if (b->persistent) {
    uint32_t err = 0;
    std::memcpy(&err, static_cast<const char*>(b->pin) + b->err_pin_off, 4);
    if (err) return set_status(ZKG_ERR_TIMEOUT, "zkg_batch_run", "an NTT pass waited too long for its input");
  }
  std::vector<uint64_t*> outs;
  std::vector<int> kinds;
  for (auto& m : b->msms) { outs.push_back(m.out); kinds.push_back(m.kind); }
  for (auto& m : b->msms)
    if (m.n == 0) host::xyzz_write<NL>(F, host::xyzz_inf<NL>(), m.kind, m.out);
  if (!b->mp.reqs.empty()) multi_msm_tails<NL>(F, b->mp, static_cast<const uint64_t*>(b->pin), outs, kinds);
  return ZKG_OK;
}


// ====================================================================== served commits
//
// A commit request is the KZG `commitInterpolate` of the reference's example
// (examples/KZG.hs:91-97): coefficients = inverse NTT of 2^k values on the size-2^k subgroup,
// commitment = MSM of the coefficients (Montgomery form) against bases[0, 2^k) of a resident set.
// The server keeps the bases and the inverse-NTT plans resident, admits requests whenever a slot
// (stream) is free and the request's device memory fits in the HBM budget, and finishes
// requests as their slots' streams complete, so requests that arrive while others run are
// admitted as soon as capacity frees up and their work overlaps on the device.
//
// Admission takes the oldest pending request that fits; a request that does not fit may be
// overtaken by younger ones at most SRV_MAX_OVERTAKE times, after which nothing younger is
// admitted until it fits (no starvation of large requests). The host tail of a finished request
// (Horner over the window sums, output encoding) runs outside the server lock, so submitters and
// waiters are not held up by it. After a failure (a launch that fails on the host, or a device
// error reported by a slot's event) every pending and failed ticket is completed with an error
// status, requests already running on healthy slots finish normally, and new submissions are
// refused with the error.

struct SrvReq {
  uint64_t ticket;
  int k;
  const uint64_t* values;   // host, 2^k Montgomery Fr elements (pinned memory copies asynchronously)
  uint64_t* out;            // host, affine result
  std::chrono::steady_clock::time_point t0;
  int overtaken = 0;        // younger requests admitted before this one
};

static constexpr int SRV_MAX_OVERTAKE = 16;

struct SrvSlot {
  bool busy = false;
  bool finishing = false;   // its host tail is running outside the lock
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  void* pin = nullptr;
  size_t pin_cap = 0;
  SrvReq req;
  MsmPlan P;
  size_t off = 0, bytes = 0;
};

struct Srv {
  int curve = 0, dev = 0, kmin = 1, kmax = 1;
  const uint64_t* d_bases = nullptr;
  uint32_t* d_bases_dpf = nullptr;   // bases[0, 2^kmax) in the FP64 pipeline's radix, or null
  bool owns_bases_dpf = true;        // false: borrowed from a resident base set
  int n_bases = 0;
  size_t budget = 0, used = 0, peak = 0;
  char* pool = nullptr;
  std::map<size_t, size_t> free_list;   // offset -> size
  std::vector<NttPlan*> plans;          // index k
  std::vector<SrvSlot> slots;
  std::deque<SrvReq> pending;
  std::map<uint64_t, std::pair<bool, double>> results;   // ticket -> (done, latency ms)
  uint64_t next_ticket = 1, completed = 0;
  int inflight = 0, max_inflight = 0;
  zkg_status error = ZKG_OK;
  std::vector<size_t> req_bytes;   // device bytes of one request, by k
  std::vector<MsmPlan> req_plan;   // its MSM plan, by k
  long inject_fail_at = -1;        // host-side failure injection: admission number that fails
  long admissions = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::thread worker;
};

static size_t srv_alloc(Srv& S, size_t bytes) {
  for (auto it = S.free_list.begin(); it != S.free_list.end(); ++it) {
    if (it->second >= bytes) {
      const size_t off = it->first, rest = it->second - bytes;
      S.free_list.erase(it);
      if (rest) S.free_list[off + bytes] = rest;
      S.used += bytes;
      S.peak = std::max(S.peak, S.used);
      return off;
    }
  }
  return (size_t)-1;
}

static void srv_free(Srv& S, size_t off, size_t bytes) {
  S.used -= bytes;
  auto it = S.free_list.emplace(off, bytes).first;
  auto nx = std::next(it);
  if (nx != S.free_list.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    S.free_list.erase(nx);
  }
  if (it != S.free_list.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      S.free_list.erase(it);
    }
  }
}

static inline size_t rup256(size_t x) { return (x + 255) & ~size_t(255); }

template <class C>
static size_t srv_bytes(int k, MsmPlan& P) {
  if (make_plan<C>(1 << k, 4, 1, P) != ZKG_OK) return (size_t)-1;
  return 3 * rup256(((size_t)32) << k) + rup256(P.bytes);
}

template <class C, int NL>
static zkg_status srv_launch(Srv& S, SrvSlot& sl) {
  NvtxRange nvtx("zkb.server.launch");
  if (S.inject_fail_at >= 0 && S.admissions == S.inject_fail_at)
    return set_status(ZKG_ERR_CUDA, "server", "injected launch failure (zkg_server_inject_failure)");
  Context* cx = nullptr;
  ZKB_TRY(get_context(&cx));
  const int k = sl.req.k;
  const size_t N = (size_t)1 << k, vb = rup256(N * 32);
  char* base = S.pool + sl.off;
  uint32_t* d_vals = reinterpret_cast<uint32_t*>(base);
  uint32_t* d_coef = reinterpret_cast<uint32_t*>(base + vb);
  uint32_t* d_scr = reinterpret_cast<uint32_t*>(base + 2 * vb);
  char* ws = base + 3 * vb;
  ZKB_CUDA(cudaMemcpyAsync(d_vals, sl.req.values, N * 32, cudaMemcpyHostToDevice, sl.st));
  ZKB_TRY(ntt_plan_execute(*S.plans[k], d_vals, d_coef, d_scr, sl.st));
  PartSet parts;
  parts.n = 1;
  parts.bsum[0] = reinterpret_cast<const uint32_t*>(ws + sl.P.o_bsum);
  parts.off[0] = reinterpret_cast<const uint32_t*>(ws + sl.P.o_off);
  if (g_msm_dpf) {   // the pipeline's bases: converted once (S.d_bases_dpf) or as given
    using CD = typename MsmCurve<C>::type;
    const uint64_t* pb = S.d_bases_dpf ? reinterpret_cast<const uint64_t*>(S.d_bases_dpf) : S.d_bases;
    ZKB_TRY(msm_launch_part<CD>(*cx, sl.P, ws, reinterpret_cast<const uint64_t*>(d_coef), 1, pb, sl.st, nullptr,
                                false, false));
    ZKB_TRY(msm_launch_reduce<CD>(*cx, sl.P, ws, parts, sl.st, false));
    ZKB_TRY(msm_u_to_radix<CD>(sl.P, ws, sl.st));
  } else {
    ZKB_TRY(msm_launch_part<C>(*cx, sl.P, ws, reinterpret_cast<const uint64_t*>(d_coef), 1, S.d_bases, sl.st,
                               nullptr, false, false));
    ZKB_TRY(msm_launch_reduce<C>(*cx, sl.P, ws, parts, sl.st, false));
  }
  const size_t ubytes = (size_t)sl.P.nwin * (sl.P.gbits + 1) * 4 * NL * 8;
  if (sl.pin_cap < ubytes) return set_status(ZKG_ERR_ARG, "server", "slot staging smaller than a request's sums");
  ZKB_CUDA(cudaMemcpyAsync(sl.pin, ws + sl.P.o_U, ubytes, cudaMemcpyDeviceToHost, sl.st));
  ZKB_CUDA(cudaEventRecord(sl.done, sl.st));
  return ZKG_OK;
}

// Completes every pending request with an error status (after a failure); caller holds S.mu.
static void srv_fail_pending(Srv& S) {
  if (S.pending.empty()) return;
  for (auto& r : S.pending) S.results[r.ticket] = {true, -1.0};
  S.pending.clear();
  S.cv_done.notify_all();
}

template <class C, int NL>
static void srv_loop(Srv* S, const host::Field<NL>* F) {
  cudaSetDevice(S->dev);
  std::unique_lock<std::mutex> lk(S->mu);
  std::vector<SrvSlot*> done;
  while (true) {
    bool progress = false;
    // finished slots: collect under the lock, run the host tails without it
    done.clear();
    for (auto& sl : S->slots) {
      if (!sl.busy || sl.finishing) continue;
      const cudaError_t q = cudaEventQuery(sl.done);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) {   // the device reported an error for this request's work
        (void)cudaGetLastError();
        if (S->error == ZKG_OK) S->error = set_status(ZKG_ERR_CUDA, "server", cudaGetErrorString(q));
        S->results[sl.req.ticket] = {true, -1.0};
        srv_free(*S, sl.off, sl.bytes);
        sl.busy = false;
        S->inflight--;
        progress = true;
        continue;
      }
      sl.finishing = true;
      done.push_back(&sl);
    }
    if (!done.empty()) {
      lk.unlock();
      for (SrvSlot* sl : done) {
        const host::Xyzz<NL> r = msm_host_combine<NL>(*F, sl->P, static_cast<const uint64_t*>(sl->pin));
        host::xyzz_write<NL>(*F, r, ZKG_OUT_AFFINE, sl->req.out);
      }
      lk.lock();
      const auto now = std::chrono::steady_clock::now();
      for (SrvSlot* sl : done) {
        S->results[sl->req.ticket] = {true, std::chrono::duration<double, std::milli>(now - sl->req.t0).count()};
        srv_free(*S, sl->off, sl->bytes);
        sl->busy = false;
        sl->finishing = false;
        S->inflight--;
        S->completed++;
      }
      progress = true;
    }
    if (progress) S->cv_done.notify_all();
    if (S->error != ZKG_OK) srv_fail_pending(*S);
    // admission: the oldest pending request that fits, within the overtaking bound
    while (!S->pending.empty() && S->error == ZKG_OK) {
      SrvSlot* free_slot = nullptr;
      for (auto& sl : S->slots)
        if (!sl.busy) { free_slot = &sl; break; }
      if (!free_slot) break;
      const bool head_only = S->pending.front().overtaken >= SRV_MAX_OVERTAKE;
      size_t pick = (size_t)-1, off = (size_t)-1;
      for (size_t q = 0; q < S->pending.size() && (q == 0 || !head_only); q++) {
        off = srv_alloc(*S, S->req_bytes[S->pending[q].k]);
        if (off != (size_t)-1) { pick = q; break; }
      }
      if (pick == (size_t)-1) break;
      for (size_t q = 0; q < pick; q++) S->pending[q].overtaken++;
      const int k = S->pending[pick].k;
      free_slot->req = S->pending[pick];
      S->pending.erase(S->pending.begin() + (long)pick);
      free_slot->P = S->req_plan[k];
      free_slot->off = off;
      free_slot->bytes = S->req_bytes[k];
      free_slot->busy = true;
      S->inflight++;
      S->max_inflight = std::max(S->max_inflight, S->inflight);
      const zkg_status st = srv_launch<C, NL>(*S, *free_slot);
      S->admissions++;
      if (st != ZKG_OK) {
        // work already enqueued on the slot's stream may still touch its memory: wait for it
        // before the memory can be reused (nothing else is admitted after an error anyway)
        cudaStreamSynchronize(free_slot->st);
        (void)cudaGetLastError();
        S->error = st;
        S->results[free_slot->req.ticket] = {true, -1.0};
        srv_free(*S, off, free_slot->bytes);
        free_slot->busy = false;
        S->inflight--;
        srv_fail_pending(*S);
        S->cv_done.notify_all();
      }
      progress = true;
    }
    if (S->stop && S->inflight == 0 && S->pending.empty()) break;
    if (!progress) {
      if (S->inflight > 0) S->cv_work.wait_for(lk, std::chrono::microseconds(50));
      else S->cv_work.wait(lk, [&] { return S->stop || !S->pending.empty(); });
    }
  }
}

template <class C, int NL>
static zkg_status srv_start(Srv* S, const host::Field<NL>* F, const host::Field<4>& FR, int log_max,
                            const uint64_t* gmax_std, int kmin, int kmax, int nslots) {
  ZKB_CUDA(cudaGetDevice(&S->dev));
  cudaStream_t st0;
  ZKB_CUDA(cudaStreamCreateWithFlags(&st0, cudaStreamNonBlocking));
  S->plans.assign(kmax + 1, nullptr);
  host::El<4> g;
  std::memcpy(g.v, gmax_std, 32);
  g = host::from_std(FR, g);
  for (int k = kmin; k <= kmax; k++) {
    host::El<4> gk = g;
    for (int i = 0; i < log_max - k; i++) gk = host::mul(FR, gk, gk);
    zkg_status st = ntt_plan_new(S->curve, k, gk.v, 1, 0, st0, &S->plans[k]);
    if (st != ZKG_OK) { cudaStreamDestroy(st0); return st; }
  }
  // bases of the largest request, converted once into the FP64 pipeline's radix (unless they
  // come from a resident base set that already holds them so)
  if (g_msm_dpf && radix_conv_v<typename MsmCurve<C>::type::Fp> && !S->d_bases_dpf) {
    using CD = typename MsmCurve<C>::type;
    const uint32_t nb = (uint32_t)std::min<int64_t>(S->n_bases, (int64_t)1 << kmax);
    if (cudaMalloc(&S->d_bases_dpf, (size_t)nb * 2 * NL * 8) != cudaSuccess) {
      (void)cudaGetLastError();
      S->d_bases_dpf = nullptr;
      cudaStreamDestroy(st0);
      return set_status(ZKG_ERR_NOMEM, "zkg_server_create", "converted bases");
    }
    Fe<typename CD::Fp> kin, kout;
    dpf_consts_for<CD>(kin, kout);
    zkg_status st = launch("msm_bases_to_dpf", k_msm_bases_to_dpf<CD>, dim3((nb + 255) / 256), dim3(256), 0, st0, nb,
                           reinterpret_cast<const uint32_t*>(S->d_bases), kin, S->d_bases_dpf);
    if (st == ZKG_OK && cudaStreamSynchronize(st0) != cudaSuccess) st = set_status(ZKG_ERR_CUDA, "zkg_server_create", "sync");
    if (st != ZKG_OK) { cudaStreamDestroy(st0); return st; }
  }
  cudaStreamDestroy(st0);
  // plans and device bytes of every request size, once; every admissible request must fit in
  // the budget on its own
  S->req_bytes.assign(kmax + 1, (size_t)-1);
  S->req_plan.assign(kmax + 1, MsmPlan());
  size_t ubytes_max = 64;
  using CP = typename MsmCurve<C>::type;
  for (int k = kmin; k <= kmax; k++) {
    MsmPlan P;
    const size_t b = g_msm_dpf ? srv_bytes<CP>(k, P) : srv_bytes<C>(k, P);
    if (b == (size_t)-1 || b > S->budget)
      return set_status(ZKG_ERR_ARG, "zkg_server_create", "HBM budget smaller than one request of the largest size");
    S->req_bytes[k] = b;
    S->req_plan[k] = P;
    ubytes_max = std::max(ubytes_max, (size_t)P.nwin * (P.gbits + 1) * 4 * NL * 8);
  }
  ZKB_CUDA(cudaMalloc(&S->pool, S->budget));
  S->free_list[0] = S->budget;
  S->slots.resize(nslots);
  for (auto& sl : S->slots) {   // page-locked staging of each slot's window sums, sized once
    ZKB_CUDA(cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking));
    ZKB_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    ZKB_CUDA(cudaMallocHost(&sl.pin, ubytes_max));
    sl.pin_cap = ubytes_max;
  }
  S->worker = std::thread(srv_loop<C, NL>, S, F);
  return ZKG_OK;
}

// domain generators of Fr in standard form (codegen/src/Zikkurat/Generate.hs:143-144)
static const uint64_t BN_FFT_GEN[4] = {0x9bd61b6e725b19f0ULL, 0x402d111e41112ed4ULL, 0x00e0a7eb8ef62abcULL,
                                       0x2a3c09f0a58a7e85ULL};
static const uint64_t BLS_FFT_GEN[4] = {0x3829971f439f0d2bULL, 0xb63683508c2280b9ULL, 0xd09b681922c813b4ULL,
                                        0x16a2a19edfe81f20ULL};


// ============================================================================== autotuner

// splitmix64-style words below 2^252 (valid Montgomery scalars for both curves)
__global__ void k_rand_scalars(uint64_t* out, uint32_t n, uint64_t seed) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int l = 0; l < 4; l++) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (4ull * i + l + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    out[4 * (size_t)i + l] = l == 3 ? (z & 0x0fffffffffffffffull) : z;
  }
}

// Tunes the MSM for n = 2^L, L in [lmin, lmax], on device-resident bases and random scalars:
// window width first (around the cost model's choice, other settings at their defaults), then
// with that width the level-1 chunk length, the running-sum group size and the prefetch stages,
// one at a time (coordinate search). Each setting is timed as the best of two calls after a
// warm-up call. The winners become that size's settings (and are persisted when ZKG_TUNE_CACHE
// is set). Results never depend on them: only the order of exact operations changes.
template <class C, int NL>
static zkg_status autotune_msm(const host::Field<NL>& F, const uint64_t* d_bases, int n_bases, int lmin, int lmax,
                               int* chosen) {
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  uint64_t* d_s = nullptr;
  const uint32_t nmax = 1u << lmax;
  ZKB_CUDA(cudaMalloc(&d_s, (size_t)nmax * 32));
  zkg_status st = launch("rand_scalars", k_rand_scalars, dim3((nmax + 255) / 256), dim3(256), 0, cx.stream, d_s,
                         nmax, 0x5eed7u);
  if (st == ZKG_OK && cudaStreamSynchronize(cx.stream) != cudaSuccess)
    st = set_status(ZKG_ERR_CUDA, "autotune", "scalar generation");
  uint64_t out[3 * 6];
  const int sms = device_sm_count();
  for (int L = lmin; st == ZKG_OK && L <= lmax; L++) {
    const int n = 1 << L;
    MsmTune& T = msm_tune(C::ID, L);
    auto time_it = [&]() -> float {
      float t = 1e30f;
      for (int rep = 0; rep < 3 && st == ZKG_OK; rep++) {
        st = msm_dev_entry<C, NL>(F, n, d_s, 4, 1, d_bases, ZKG_OUT_PROJ, out);
        if (rep > 0) t = std::min(t, cx.last_kernel_ms);
      }
      return t;
    };
    T = MsmTune();
    const int c0 = auto_window(n, C::SCALAR_BITS, bucket_weight(C::ID));
    float best = 1e30f;
    MsmTune bestT;
    for (int c = std::max(2, c0 - 2); c <= std::min(20, c0 + 2) && st == ZKG_OK; c++) {
      T = MsmTune();
      T.c = c;
      const float t = time_it();
      if (t < best) { best = t; bestT = T; }
    }
    // affine tree levels (0-3; the exact-radix pipelines, where the rule by segment length may
    // not be the best for this size)
    for (int lv = 0; lv <= 3; lv++) {
      T = bestT;
      T.tree = lv + 1;
      const float t = time_it();
      if (st == ZKG_OK && t < best) { best = t; bestT = T; }
    }
    const int L1s[] = {64, 96, 160, 224};
    for (int v : L1s) {
      T = bestT;
      T.L1 = v;
      const float t = time_it();
      if (st == ZKG_OK && t < best) { best = t; bestT = T; }
    }
    const int K1s[] = {4, 8, 16, 64};
    for (int v : K1s) {
      T = bestT;
      T.K1 = v;
      const float t = time_it();
      if (st == ZKG_OK && t < best) { best = t; bestT = T; }
    }
    const int PFs[] = {0, 3};
    for (int v : PFs) {
      if (v == 3 && C::Fp::N != 8) continue;
      T = bestT;
      T.pf = v;
      const float t = time_it();
      if (st == ZKG_OK && t < best) { best = t; bestT = T; }
    }
    T = bestT;
    if (st == ZKG_OK) {
      const int v[5] = {T.c, T.L1, T.K1, T.pf, T.tree};
      tune_cache_put("msm", C::ID, L, sms, v, 5);
      if (chosen) chosen[L - lmin] = T.c;
    }
  }
  cudaFree(d_s);
  (void)n_bases;
  return st;
}

}  // namespace zkb

extern "C" {

zkg_status zkg_msm(zkg_curve curve, int npoints, const uint64_t* expos, int expo_nlimbs, int expos_mont,
                   const uint64_t* grps, zkg_out_kind kind, uint64_t* tgt) {
  if (kind < 0 || kind > 2) return zkb::set_status(ZKG_ERR_ARG, "zkg_msm", "bad output kind");
  if (curve == ZKG_BN254)
    return zkb::msm_host_entry<zkb::BN254, 4>(zkb::host::BN_FP, npoints, expos, expo_nlimbs, expos_mont, grps, kind, tgt);
  if (curve == ZKG_BLS12_381)
    return zkb::msm_host_entry<zkb::BLS12_381, 6>(zkb::host::BLS_FP, npoints, expos, expo_nlimbs, expos_mont, grps, kind, tgt);
  return zkb::set_status(ZKG_ERR_ARG, "zkg_msm", "unknown curve");
}

zkg_status zkg_msm_device(zkg_curve curve, int npoints, const uint64_t* d_expos, int expo_nlimbs, int expos_mont,
                          const uint64_t* d_grps, zkg_out_kind kind, uint64_t* tgt) {
  if (kind < 0 || kind > 2) return zkb::set_status(ZKG_ERR_ARG, "zkg_msm_device", "bad output kind");
  if (curve == ZKG_BN254)
    return zkb::msm_dev_entry<zkb::BN254, 4>(zkb::host::BN_FP, npoints, d_expos, expo_nlimbs, expos_mont, d_grps, kind, tgt);
  if (curve == ZKG_BLS12_381)
    return zkb::msm_dev_entry<zkb::BLS12_381, 6>(zkb::host::BLS_FP, npoints, d_expos, expo_nlimbs, expos_mont, d_grps, kind, tgt);
  return zkb::set_status(ZKG_ERR_ARG, "zkg_msm_device", "unknown curve");
}

zkg_status zkg_bases_upload(zkg_curve curve, const uint64_t* bases, int n, int on_device, zkg_bases** out) {
  if (!out || (curve != ZKG_BN254 && curve != ZKG_BLS12_381) || n <= 0 || !bases)
    return zkb::set_status(ZKG_ERR_ARG, "zkg_bases_upload", "bad arguments");
  *out = nullptr;
  const int nl = curve == ZKG_BN254 ? 4 : 6;
  const size_t bytes = (size_t)n * 2 * nl * 8;
  zkg_bases* h = new zkg_bases();
  h->curve = curve;
  h->n = n;
  auto fail = [&](zkg_status st) { delete h; return st; };
  if (cudaGetDevice(&h->dev) != cudaSuccess) return fail(zkb::set_status(ZKG_ERR_CUDA, "zkg_bases_upload", "no device"));
  const cudaError_t e = cudaMalloc(&h->d_pts, bytes);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    h->d_pts = nullptr;
    return fail(zkb::set_status(ZKG_ERR_NOMEM, "zkg_bases_upload", cudaGetErrorString(e)));
  }
  zkb::Context* cx = nullptr;
  zkg_status st = zkb::get_context(&cx);
  if (st != ZKG_OK) return fail(st);
  std::lock_guard<std::mutex> lk(cx->mu);
  const cudaStream_t s = cx->compute();
  if (on_device) {
    if (cudaMemcpyAsync(h->d_pts, bases, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return fail(zkb::set_status(ZKG_ERR_CUDA, "zkg_bases_upload", "device copy"));
  } else {
    st = zkb::copy_h2d(*cx, h->d_pts, bases, bytes, s);
    if (st != ZKG_OK) return fail(st);
  }
  if (zkb::g_msm_dpf) {
    using CB = zkb::MsmCurve<zkb::BN254>::type;
    using CL = zkb::MsmCurve<zkb::BLS12_381>::type;
    if constexpr (zkb::radix_conv_v<CB::Fp>) {   // into the pipeline's radix, in place (each thread
      const uint32_t* src = reinterpret_cast<const uint32_t*>(h->d_pts);   // reads its point first)
      uint32_t* dst = reinterpret_cast<uint32_t*>(h->d_pts);
      const dim3 g(((uint32_t)n + 255) / 256);
      st = curve == ZKG_BN254
               ? zkb::launch("msm_bases_to_dpf", zkb::k_msm_bases_to_dpf<CB>, g, dim3(256), 0, s, (uint32_t)n, src,
                             zkb::dpf_kin<CB>(), dst)
               : zkb::launch("msm_bases_to_dpf", zkb::k_msm_bases_to_dpf<CL>, g, dim3(256), 0, s, (uint32_t)n, src,
                             zkb::dpf_kin<CL>(), dst);
      if (st != ZKG_OK) return fail(st);
    }
    h->converted = true;   // held in the form the FP64 pipeline reads
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(zkb::set_status(ZKG_ERR_CUDA, "zkg_bases_upload", "sync"));
  *out = h;
  return zkb::set_status(ZKG_OK, nullptr, nullptr);
}

zkg_status zkg_bases_destroy(zkg_bases* h) {
  if (h) {
    cudaDeviceSynchronize();
    delete h;
  }
  return ZKG_OK;
}

int zkg_bases_count(const zkg_bases* h) { return h ? h->n : 0; }

static zkg_status msm_resident(const char* who, zkg_bases* h, int npoints, const uint64_t* d_expos,
                               const uint64_t* h_expos, int expo_nlimbs, int expos_mont, zkg_out_kind kind,
                               uint64_t* tgt) {
  if (!h || kind < 0 || kind > 2) return zkb::set_status(ZKG_ERR_ARG, who, "null handle or bad output kind");
  if (npoints < 0 || npoints > h->n) return zkb::set_status(ZKG_ERR_ARG, who, "npoints outside [0, bases in the set]");
  const uint64_t* g = h->d_pts;
  if (h->curve == ZKG_BN254)
    return h->converted
               ? zkb::msm_dev_run<zkb::MsmCurve<zkb::BN254>::type, zkb::BN254, 4>(zkb::host::BN_FP, npoints, d_expos, expo_nlimbs,
                                                              expos_mont, g, kind, tgt, true, h_expos)
               : zkb::msm_dev_run<zkb::BN254, zkb::BN254, 4>(zkb::host::BN_FP, npoints, d_expos, expo_nlimbs,
                                                             expos_mont, g, kind, tgt, true, h_expos);
  return h->converted
             ? zkb::msm_dev_run<zkb::MsmCurve<zkb::BLS12_381>::type, zkb::BLS12_381, 6>(zkb::host::BLS_FP, npoints, d_expos, expo_nlimbs,
                                                                    expos_mont, g, kind, tgt, true, h_expos)
             : zkb::msm_dev_run<zkb::BLS12_381, zkb::BLS12_381, 6>(zkb::host::BLS_FP, npoints, d_expos, expo_nlimbs,
                                                                   expos_mont, g, kind, tgt, true, h_expos);
}

zkg_status zkg_msm_resident(zkg_bases* h, int npoints, const uint64_t* d_expos, int expo_nlimbs, int expos_mont,
                            zkg_out_kind kind, uint64_t* tgt) {
  return msm_resident("zkg_msm_resident", h, npoints, d_expos, nullptr, expo_nlimbs, expos_mont, kind, tgt);
}

zkg_status zkg_msm_resident_host(zkg_bases* h, int npoints, const uint64_t* expos, int expo_nlimbs, int expos_mont,
                                 zkg_out_kind kind, uint64_t* tgt) {
  return msm_resident("zkg_msm_resident_host", h, npoints, nullptr, expos, expo_nlimbs, expos_mont, kind, tgt);
}

zkg_status zkg_batch_create_resident(zkg_bases* h, zkg_batch** out) {
  if (!h) return zkb::set_status(ZKG_ERR_ARG, "zkg_batch_create_resident", "null handle");
  zkg_status st = zkg_batch_create((zkg_curve)h->curve, h->d_pts, h->n, out);
  if (st == ZKG_OK) (*out)->bases_converted = h->converted;
  return st;
}

zkg_status zkg_batch_create(zkg_curve curve, const uint64_t* d_bases, int n_bases, zkg_batch** out) {
  if (!out || (curve != ZKG_BN254 && curve != ZKG_BLS12_381) || n_bases < 0 || (n_bases > 0 && !d_bases))
    return zkb::set_status(ZKG_ERR_ARG, "zkg_batch_create", "bad arguments");
  zkg_batch* b = new zkg_batch();
  b->persistent_wanted = zkb::g_batch_persistent != 0;
  b->curve = curve;
  b->d_bases = d_bases;
  b->n_bases = n_bases;
  *out = b;
  return zkb::set_status(ZKG_OK, nullptr, nullptr);
}

zkg_status zkg_batch_add_msm(zkg_batch* b, int n, const uint64_t* d_scalars_mont, uint64_t* out_affine) {
  if (!b || b->built) return zkb::set_status(ZKG_ERR_ARG, "zkg_batch_add_msm", "null or already run batch");
  if (n < 0 || n > b->n_bases || (n > 0 && !d_scalars_mont) || !out_affine)
    return zkb::set_status(ZKG_ERR_ARG, "zkg_batch_add_msm", "n must be in [0, n_bases]");
  b->msms.push_back({n, d_scalars_mont, out_affine, ZKG_OUT_AFFINE});
  return zkb::set_status(ZKG_OK, nullptr, nullptr);
}

zkg_status zkg_batch_add_ntt(zkg_batch* b, int m, const uint64_t* gen, const uint64_t* d_src, uint64_t* d_tgt,
                             int inverse) {
  if (!b || b->built) return zkb::set_status(ZKG_ERR_ARG, "zkg_batch_add_ntt", "null or already run batch");
  if (m < 0 || m > zkb::NTT_MMAX || !gen || !d_src || !d_tgt || d_src == d_tgt)
    return zkb::set_status(ZKG_ERR_ARG, "zkg_batch_add_ntt", "bad arguments");
  zkg_batch::Ntt t;
  t.m = m;
  std::memcpy(t.gen, gen, 32);
  t.d_src = d_src;
  t.d_tgt = d_tgt;
  t.inverse = inverse;
  b->ntts.push_back(t);
  return zkb::set_status(ZKG_OK, nullptr, nullptr);
}

zkg_status zkg_batch_run(zkg_batch* b) {
  if (!b) return zkb::set_status(ZKG_ERR_ARG, "zkg_batch_run", "null batch");
  zkb::Context* cx = nullptr;
  zkg_status s = zkb::get_context(&cx);
  if (s != ZKG_OK) return s;
  std::lock_guard<std::mutex> lk(cx->mu);
  s = b->curve == ZKG_BN254 ? zkb::batch_run<zkb::BN254, 4>(b, zkb::host::BN_FP)
                            : zkb::batch_run<zkb::BLS12_381, 6>(b, zkb::host::BLS_FP);
  return s == ZKG_OK ? zkb::set_status(ZKG_OK, nullptr, nullptr) : s;
}

float zkg_batch_last_ms(const zkg_batch* b) { return b ? b->last_ms : -1.f; }

zkg_status zkg_batch_set_wait_limit(zkg_batch* b, uint32_t polls, int inject_stall) {
  if (!b || b->built || polls == 0)
    return zkb::set_status(ZKG_ERR_ARG, "zkg_batch_set_wait_limit", "null or already run batch, or zero polls");
  b->wait_limit = polls;
  b->inject_stall = inject_stall != 0;
  return zkb::set_status(ZKG_OK, nullptr, nullptr);
}

zkg_status zkg_batch_set_mode(zkg_batch* b, int persistent) {
  if (!b || b->built) return zkb::set_status(ZKG_ERR_ARG, "zkg_batch_set_mode", "null or already run batch");
  b->persistent_wanted = persistent != 0;
  return zkb::set_status(ZKG_OK, nullptr, nullptr);
}

int zkg_batch_persistent(const zkg_batch* b, int* grid, uint32_t* tasks) {
  if (!b) return -1;
  if (grid) *grid = b->work_grid;
  if (tasks) *tasks = b->work_tasks;
  return b->persistent ? 1 : 0;
}

zkg_status zkg_batch_destroy(zkg_batch* b) {
  if (b) {
    cudaDeviceSynchronize();
    delete b;
  }
  return ZKG_OK;
}

struct zkg_server {
  zkb::Srv S;
};

static zkg_status server_create(zkg_curve curve, const uint64_t* d_bases, const zkg_bases* h, int n_bases, int k_min,
                                int k_max, size_t hbm_budget, int slots, zkg_server** out);

zkg_status zkg_server_create(zkg_curve curve, const uint64_t* d_bases, int n_bases, int k_min, int k_max,
                             size_t hbm_budget, int slots, zkg_server** out) {
  return server_create(curve, d_bases, nullptr, n_bases, k_min, k_max, hbm_budget, slots, out);
}

zkg_status zkg_server_create_resident(zkg_bases* h, int k_min, int k_max, size_t hbm_budget, int slots,
                                      zkg_server** out) {
  if (!h) return zkb::set_status(ZKG_ERR_ARG, "zkg_server_create_resident", "null handle");
  return server_create((zkg_curve)h->curve, h->d_pts, h, h->n, k_min, k_max, hbm_budget, slots, out);
}

static zkg_status server_create(zkg_curve curve, const uint64_t* d_bases, const zkg_bases* h, int n_bases, int k_min,
                                int k_max, size_t hbm_budget, int slots, zkg_server** out) {
  if (!out || (curve != ZKG_BN254 && curve != ZKG_BLS12_381) || !d_bases || n_bases <= 0 || k_min < 1 ||
      k_max < k_min || k_max > 26 || ((size_t)1 << k_max) > (size_t)n_bases || slots < 1 || slots > 64)
    return zkb::set_status(ZKG_ERR_ARG, "zkg_server_create",
                           "need 1 <= k_min <= k_max <= 26, 2^k_max <= n_bases, 1 <= slots <= 64");
  zkg_server* srv = new zkg_server();
  zkb::Srv& S = srv->S;
  S.curve = curve;
  S.d_bases = d_bases;
  S.n_bases = n_bases;
  S.budget = hbm_budget;
  if (h && h->converted) {   // borrowed: already in the FP64 pipeline's radix
    S.d_bases = nullptr;
    S.d_bases_dpf = reinterpret_cast<uint32_t*>(h->d_pts);
    S.owns_bases_dpf = false;
  }
  S.kmin = k_min;
  S.kmax = k_max;
  zkg_status st = curve == ZKG_BN254
      ? zkb::srv_start<zkb::BN254, 4>(&S, &zkb::host::BN_FP, zkb::host::BN_FR, 28, zkb::BN_FFT_GEN, k_min, k_max, slots)
      : zkb::srv_start<zkb::BLS12_381, 6>(&S, &zkb::host::BLS_FP, zkb::host::BLS_FR, 32, zkb::BLS_FFT_GEN, k_min, k_max,
                                          slots);
  if (st != ZKG_OK) {
    zkg_server_destroy(srv);
    return st;
  }
  *out = srv;
  return zkb::set_status(ZKG_OK, nullptr, nullptr);
}

zkg_status zkg_server_submit(zkg_server* srv, int k, const uint64_t* values, uint64_t* out_affine, uint64_t* ticket) {
  if (!srv || !values || !out_affine || !ticket) return zkb::set_status(ZKG_ERR_ARG, "zkg_server_submit", "null argument");
  zkb::Srv& S = srv->S;
  if (k < S.kmin || k > S.kmax) return zkb::set_status(ZKG_ERR_ARG, "zkg_server_submit", "k outside the server's range");
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.error != ZKG_OK) return S.error;
  zkb::SrvReq r;
  r.ticket = S.next_ticket++;
  r.k = k;
  r.values = values;
  r.out = out_affine;
  r.t0 = std::chrono::steady_clock::now();
  S.results[r.ticket] = {false, 0.0};
  S.pending.push_back(r);
  *ticket = r.ticket;
  S.cv_work.notify_one();
  return zkb::set_status(ZKG_OK, nullptr, nullptr);
}

zkg_status zkg_server_wait_for(zkg_server* srv, uint64_t ticket, double timeout_ms, double* latency_ms) {
  if (!srv) return zkb::set_status(ZKG_ERR_ARG, "zkg_server_wait", "null server");
  zkb::Srv& S = srv->S;
  std::unique_lock<std::mutex> lk(S.mu);
  auto it = S.results.find(ticket);
  if (it == S.results.end()) return zkb::set_status(ZKG_ERR_ARG, "zkg_server_wait", "unknown ticket");
  auto ready = [&] { return S.results[ticket].first; };
  if (timeout_ms < 0) {
    S.cv_done.wait(lk, ready);
  } else if (!S.cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) {
    return zkb::set_status(ZKG_ERR_TIMEOUT, "zkg_server_wait", "deadline passed; the ticket stays valid");
  }
  const double ms = S.results[ticket].second;
  S.results.erase(ticket);
  if (latency_ms) *latency_ms = ms;
  if (ms < 0) {
    const zkg_status e = S.error != ZKG_OK ? S.error : ZKG_ERR_CUDA;
    return zkb::set_status(e, "zkg_server_wait", "the request failed (server error)");
  }
  return zkb::set_status(ZKG_OK, nullptr, nullptr);
}

zkg_status zkg_server_wait(zkg_server* srv, uint64_t ticket, double* latency_ms) {
  return zkg_server_wait_for(srv, ticket, -1.0, latency_ms);
}

zkg_status zkg_server_inject_failure(zkg_server* srv, long admission) {
  if (!srv) return zkb::set_status(ZKG_ERR_ARG, "zkg_server_inject_failure", "null server");
  std::lock_guard<std::mutex> lk(srv->S.mu);
  srv->S.inject_fail_at = admission < 0 ? -1 : srv->S.admissions + admission;
  return ZKG_OK;
}

zkg_status zkg_server_stats(zkg_server* srv, uint64_t* completed, int* max_inflight, size_t* peak_bytes) {
  if (!srv) return zkb::set_status(ZKG_ERR_ARG, "zkg_server_stats", "null server");
  std::lock_guard<std::mutex> lk(srv->S.mu);
  if (completed) *completed = srv->S.completed;
  if (max_inflight) *max_inflight = srv->S.max_inflight;
  if (peak_bytes) *peak_bytes = srv->S.peak;
  return ZKG_OK;
}

zkg_status zkg_server_destroy(zkg_server* srv) {
  if (!srv) return ZKG_OK;
  zkb::Srv& S = srv->S;
  {
    std::lock_guard<std::mutex> lk(S.mu);
    S.stop = true;
  }
  S.cv_work.notify_all();
  if (S.worker.joinable()) S.worker.join();
  cudaDeviceSynchronize();
  for (auto& sl : S.slots) {
    if (sl.st) cudaStreamDestroy(sl.st);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.pin) cudaFreeHost(sl.pin);
  }
  for (auto p : S.plans) delete p;
  if (S.pool) cudaFree(S.pool);
  if (S.d_bases_dpf && S.owns_bases_dpf) cudaFree(S.d_bases_dpf);
  delete srv;
  return ZKG_OK;
}

zkg_status zkg_autotune_msm(zkg_curve curve, const uint64_t* d_bases, int n_bases, int log_min, int log_max,
                            int* chosen) {
  if ((curve != ZKG_BN254 && curve != ZKG_BLS12_381) || !d_bases || log_min < 1 || log_max < log_min ||
      log_max > 26 || (1 << log_max) > n_bases)
    return zkb::set_status(ZKG_ERR_ARG, "zkg_autotune_msm", "need 1 <= log_min <= log_max <= 26, 2^log_max <= n_bases");
  return curve == ZKG_BN254
             ? zkb::autotune_msm<zkb::BN254, 4>(zkb::host::BN_FP, d_bases, n_bases, log_min, log_max, chosen)
             : zkb::autotune_msm<zkb::BLS12_381, 6>(zkb::host::BLS_FP, d_bases, n_bases, log_min, log_max, chosen);
}

int zkg_msm_tuned_window(zkg_curve curve, int log_n) {
  if ((curve != ZKG_BN254 && curve != ZKG_BLS12_381) || log_n < 0 || log_n >= 32) return 0;
  return zkb::msm_tune(curve, log_n).c;
}

int zkg_msm_tuned_config(zkg_curve curve, int log_n, int* c, int* chunk_len, int* group, int* prefetch) {
  if ((curve != ZKG_BN254 && curve != ZKG_BLS12_381) || log_n < 0 || log_n >= 32) return -1;
  const zkb::MsmTune& T = zkb::msm_tune(curve, log_n);
  if (c) *c = T.c;
  if (chunk_len) *chunk_len = T.L1;
  if (group) *group = T.K1;
  if (prefetch) *prefetch = T.pf;
  return T.c > 0 ? 1 : 0;
}

int zkg_msm_last_info(int* c, int* nwin, uint64_t* additions) {
  zkb::Context* cx = nullptr;
  if (zkb::get_context(&cx) != ZKG_OK) return -1;
  if (c) *c = cx->last_msm_c;
  if (nwin) *nwin = cx->last_msm_nwin;
  if (additions) *additions = cx->last_msm_entries;
  return 0;
}

int zkg_set_msm_parts(int parts) {
  const int prev = zkb::g_tune_parts;
  zkb::g_tune_parts = parts < 0 ? 0 : (parts > 4 ? 4 : parts);
  return prev;
}

int zkg_set_msm_tree(int levels, int slots_per_thread) {
  const int prev = zkb::g_tree_env;
  zkb::g_tree_env = levels < 0 ? -1 : (levels > zkb::MAX_TREE ? zkb::MAX_TREE : levels);
  if (slots_per_thread > 0) zkb::g_tree_B = (uint32_t)std::max(4, slots_per_thread);
  else if (slots_per_thread < 0) zkb::g_tree_B = 0;   // back to the choice by entries per segment
  return prev;
}

int zkg_set_msm_window(int c) {
  const int prev = zkb::g_window_override;
  zkb::g_window_override = c < 0 ? 0 : c;
  return prev;
}

int zkg_msm_window_for(zkg_curve curve, int npoints) {
  if (zkb::g_window_override > 0) return zkb::g_window_override;
  return zkb::auto_window(npoints, curve == ZKG_BLS12_381 ? zkb::BLS12_381::SCALAR_BITS : zkb::BN254::SCALAR_BITS,
                          zkb::bucket_weight(curve));
}

}  // extern "C"
