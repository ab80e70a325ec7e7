// Pippenger MSM on G1 for BN254 and BLS12-381, B200 (sm_100a).
//
// Reference: lib/cbits/curves/g1/proj/bn128_G1_proj.c:506-586 (unsigned c-bit windows over all
// 64*expo_nlimbs scalar bits, one bucket array per window filled by mixed additions, running
// sum, c doublings per window) and the Montgomery / affine / Jacobian wrappers :597-673,
// lib/cbits/curves/g1/jac/bn128_G1_jac.c:646-720. The sum computed is the same group element;
// the schedule is the GPU's:
//
//   1. scalar prep   Montgomery -> standard form (only for *_mont_* entry points)
//   2. digits+hist   signed c-bit digits (buckets 1..2^(c-1), sign folded into the point),
//                    per-(window,bucket) counts by atomics
//   3. scan          exclusive prefix sum of the counts -> one segment per (window, bucket)
//   4. scatter       point indices (+ sign bit) placed into their segment
//   5. accumulate    equal-length chunks of the segmented array, one chunk per thread:
//                    mixed additions of affine bases into an XYZZ accumulator. Complete
//                    segments go straight to the bucket array; segments cut by a chunk
//                    boundary leave partial sums that later levels (6) fold, again in
//                    equal chunks, so any digit distribution is load balanced.
//   7. bucket reduce per (window, group of K buckets) running sums (T_g, R_g), then per
//                    window the plain sums U_R = sum R_g and U_k = sum_{g: bit k of g} T_g,
//                    so that sum_b b*S_b = U_R + K * sum_k 2^k U_k needs no doublings on
//                    the GPU
//   8. host tail     Horner over windows and bits, normalisation, output encoding.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "zkb_curve.cuh"
#include "zkb_host_ec.h"
#include "zkb_runtime.h"

namespace zkb {

static constexpr uint32_t INVALID = 0xffffffffu;
static constexpr int MAX_LEVELS = 12;

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

__global__ void k_msm_hist(int n, const uint32_t* __restrict__ scal, int nw, int c, int nwin,
                           uint32_t B, uint32_t* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* w = scal + (size_t)nw * i;
  uint32_t carry = 0, neg;
  for (int win = 0; win < nwin; win++) {
    const uint32_t b = next_digit(w, nw, win, c, carry, neg);
    if (b) atomicAdd(cnt + (size_t)win * B + (b - 1), 1u);
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

// largest s in [0, nseg) with off[s] <= pos (off[0] = 0 <= pos)
__device__ __forceinline__ uint32_t find_seg(const uint32_t* __restrict__ off, uint32_t nseg, uint32_t pos) {
  uint32_t lo = 0, hi = nseg;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= pos) lo = mid; else hi = mid;
  }
  return lo;
}

// Route a finished run of segment s inside chunk [start, start+L): the whole segment goes to
// the bucket array, a cut one to this chunk's slot A (segment began before the chunk) or
// slot B (segment continues after it).
template <class F>
__device__ __forceinline__ void route_run(uint32_t s, const Xyzz<F>& acc, uint64_t seg_lo, uint64_t seg_hi,
                                          uint64_t start, uint64_t L, uint32_t t, uint32_t* __restrict__ bsum,
                                          uint32_t* __restrict__ spt, uint32_t& keyA, uint32_t& keyB) {
  constexpr int XW = 4 * F::N;
  const bool before = seg_lo < start;
  const bool after = seg_hi > start + L;
  if (!before && !after) {
    xyzz_store<F>(bsum + (size_t)s * XW, acc);
  } else if (before) {
    keyA = s;
    xyzz_store<F>(spt + (size_t)(2 * t) * XW, acc);
  } else {
    keyB = s;
    xyzz_store<F>(spt + (size_t)(2 * t + 1) * XW, acc);
  }
}

template <class C, int L>
__global__ void __launch_bounds__(256) k_msm_accum(const uint32_t* __restrict__ entries,
                                                   const uint32_t* __restrict__ off, uint32_t nseg,
                                                   uint32_t nchunks, const uint32_t* __restrict__ bases,
                                                   uint32_t* __restrict__ bsum, uint32_t* __restrict__ skey,
                                                   uint32_t* __restrict__ spt) {
  using F = typename C::Fp;
  constexpr int AW = 2 * F::N;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nchunks) return;
  const uint32_t total = __ldg(off + nseg);
  const uint32_t start = t * (uint32_t)L;
  uint32_t keyA = INVALID, keyB = INVALID;
  if (start < total) {
    const uint32_t end = min(start + (uint32_t)L, total);
    uint32_t s = find_seg(off, nseg, start);
    uint32_t seg_lo = __ldg(off + s), seg_hi = __ldg(off + s + 1);
    Xyzz<F> acc = xyzz_inf<F>();
    bool have = false;
    uint32_t e = __ldg(entries + start);
    Affine<F> nxt = affine_load<F>(bases + (size_t)(e & 0x7fffffffu) * AW);
    for (uint32_t pos = start; pos < end; pos++) {
      while (pos >= seg_hi) {
        if (have) route_run<F>(s, acc, seg_lo, seg_hi, start, L, t, bsum, spt, keyA, keyB);
        have = false;
        acc = xyzz_inf<F>();
        s++;
        seg_lo = seg_hi;
        seg_hi = __ldg(off + s + 1);
      }
      Affine<F> a = nxt;
      const uint32_t neg = e >> 31;
      if (pos + 1 < end) {   // prefetch the next base while this addition runs
        e = __ldg(entries + pos + 1);
        nxt = affine_load<F>(bases + (size_t)(e & 0x7fffffffu) * AW);
      }
      if (!(fe_is_zero(a.x) && fe_is_zero(a.y))) {
        if (neg) a.y = fe_neg(a.y);
        xyzz_madd(acc, a);
      }
      have = true;
    }
    if (have) route_run<F>(s, acc, seg_lo, seg_hi, start, L, t, bsum, spt, keyA, keyB);
  }
  skey[2 * t] = keyA;
  skey[2 * t + 1] = keyB;
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
    xyzz_add(acc, xyzz_load<F>(ipt + y * XW));
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
  const uint32_t* off[4];
};

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
      if (__ldg(parts.off[q] + s) != __ldg(parts.off[q] + s + 1)) xyzz_add(T, xyzz_load<F>(parts.bsum[q] + s * XW));
    xyzz_add(R, T);
  }
  xyzz_store<F>(Tout + (size_t)t * XW, T);
  xyzz_store<F>(Rout + (size_t)t * XW, R);
}

// block (w, k): k < gbits -> U_k = sum over g with bit k set of T_g; k == gbits -> sum of R_g
template <class C>
__global__ void __launch_bounds__(256) k_msm_bucket_bits(const uint32_t* __restrict__ Tin,
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
      if ((g >> k) & 1u) xyzz_add(acc, xyzz_load<F>(Tin + ((size_t)w * G + g) * XW));
    } else {
      xyzz_add(acc, xyzz_load<F>(Rin + ((size_t)w * G + g) * XW));
    }
  }
  xyzz_store<F>(sm + threadIdx.x * XW, acc);
  __syncthreads();
  for (uint32_t half = blockDim.x >> 1; half > 0; half >>= 1) {
    if (threadIdx.x < half) {
      Xyzz<F> a = xyzz_load<F>(sm + threadIdx.x * XW);
      xyzz_add(a, xyzz_load<F>(sm + (threadIdx.x + half) * XW));
      xyzz_store<F>(sm + threadIdx.x * XW, a);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const Xyzz<F> r = xyzz_load<F>(sm);
    xyzz_store<F>(U + ((size_t)w * (gbits + 1) + k) * XW, r);
  }
}

// ---------------------------------------------------------------------------- planning

static int g_window_override = 0;
// tuning knobs (ZKB_MSM_L1: level-1 chunk length in {8,16,32,64,128,256}; ZKB_MSM_K1: buckets per
// running-sum group, a power of two); read once from the environment
static int env_int(const char* name, int dflt) {
  const char* v = std::getenv(name);
  return v ? std::atoi(v) : dflt;
}
static int g_tune_L1 = env_int("ZKB_MSM_L1", 0);
static int g_tune_K1 = env_int("ZKB_MSM_K1", 0);

static int ilog2_floor(uint64_t x) {
  int r = -1;
  while (x) { x >>= 1; r++; }
  return r;
}

// Cost model: nwin * (n madds + 2^(c-1) buckets * ~2.8 madd-equivalents) + per-window tail
static int auto_window(int n, int scalar_bits) {
  if (n <= 1) return 2;
  double best = 1e300;
  int bestc = 2;
  for (int c = 2; c <= 20; c++) {
    const int nwin = (scalar_bits + 1 + c - 1) / c;
    const double cost = (double)nwin * ((double)n + 2.8 * (double)(1u << (c - 1)) + 4000.0);
    if (cost < best) { best = cost; bestc = c; }
  }
  return bestc;
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
  // byte offsets into one arena block
  size_t o_std, o_cnt, o_off, o_cur, o_bs, o_ent, o_keyA, o_ptA, o_keyB, o_ptB, o_bsum, o_T, o_R, o_U, bytes;
};

template <class C>
static zkg_status make_plan(int n, int nlimbs, int mont, MsmPlan& P, int c_force = 0) {
  using F = typename C::Fp;
  constexpr size_t XB = 16 * F::N;   // bytes of one XYZZ point
  P.n = n;
  const int scalar_bits = mont ? C::SCALAR_BITS : 64 * nlimbs;
  P.c = c_force > 0 ? c_force : g_window_override > 0 ? g_window_override : auto_window(n, scalar_bits);
  if (P.c < 2 || P.c > 24) return set_status(ZKG_ERR_ARG, "msm", "window width out of range [2, 24]");
  P.nwin = (scalar_bits + 1 + P.c - 1) / P.c;
  P.nw = mont ? 8 : 2 * nlimbs;
  P.B = 1u << (P.c - 1);
  P.nseg = (uint32_t)P.nwin * P.B;
  P.total_max = (uint64_t)P.nwin * (uint64_t)n;
  if (P.total_max >= (1ull << 31)) return set_status(ZKG_ERR_ARG, "msm", "too many (window, point) entries for one launch");
  // chunk length: long chunks when there is plenty of parallelism, short ones otherwise
  const uint64_t want_threads = 148ull * 256ull;
  P.L1 = g_tune_L1 > 0 ? g_tune_L1 : 128;
  while (P.L1 > 8 && P.total_max / (uint64_t)P.L1 < want_threads) P.L1 >>= 1;
  P.nch[0] = (uint32_t)((P.total_max + P.L1 - 1) / P.L1);
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
  P.K1 = std::min<uint32_t>(P.B, g_tune_K1 > 0 ? (uint32_t)g_tune_K1 : 32u);
  P.G = P.B / P.K1;
  P.gbits = ilog2_floor(P.G);

  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o = (o + bytes + 255) & ~size_t(255); return r; };
  P.o_std = take(mont ? (size_t)n * 32 : 0);
  P.o_cnt = take((size_t)P.nseg * 4 + 4);
  P.o_off = take((size_t)P.nseg * 4 + 4);
  P.o_cur = take((size_t)P.nseg * 4 + 4);
  const uint32_t nb = (P.nseg + SCAN_T * SCAN_E - 1) / (SCAN_T * SCAN_E);
  if (nb > (uint32_t)SCAN_T * SCAN_E) return set_status(ZKG_ERR_ARG, "msm", "too many buckets");
  P.o_bs = take((size_t)nb * 4 + 4);
  P.o_ent = take((size_t)P.total_max * 4 + 4);
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
  P.bytes = o;
  return ZKG_OK;
}

// Sort the scalars of one point range into (window, bucket) segments and accumulate its bucket
// sums (phases 1-6). bases_ready, if given, is waited for just before the accumulation.
template <class C>
static zkg_status msm_launch_part(Context& cx, const MsmPlan& P, char* ws, const uint64_t* d_scal, int mont,
                                  const uint64_t* d_bases, cudaStream_t st, cudaEvent_t bases_ready, bool first,
                                  bool last) {
  const int n = P.n;
  auto U32 = [&](size_t o) { return reinterpret_cast<uint32_t*>(ws + o); };
  // phase events: 0 start, 1 sorted, 2 level-1 accumulated, 3 levels folded, 4 reduced
  if (first) ZKB_CUDA(cudaEventRecord(cx.ev_phase[0], st));
  const uint32_t* scal = reinterpret_cast<const uint32_t*>(d_scal);
  if (mont) {
    ZKB_TRY(launch("msm_scalar_from_mont", k_msm_scalar_from_mont<C>, dim3((n + 255) / 256), dim3(256), 0, st,
                   n, d_scal, U32(P.o_std)));
    scal = U32(P.o_std);
  }
  ZKB_CUDA(cudaMemsetAsync(U32(P.o_cnt), 0, (size_t)P.nseg * 4, st));
  ZKB_TRY(launch("msm_hist", k_msm_hist, dim3((n + 255) / 256), dim3(256), 0, st, n, scal, P.nw, P.c, P.nwin,
                 P.B, U32(P.o_cnt)));
  const uint32_t nb = (P.nseg + SCAN_T * SCAN_E - 1) / (SCAN_T * SCAN_E);
  ZKB_TRY(launch("scan_blocks", k_scan_blocks, dim3(nb), dim3(SCAN_T), 0, st, (const uint32_t*)U32(P.o_cnt),
                 U32(P.o_off), U32(P.o_bs), P.nseg));
  ZKB_TRY(launch("scan_top", k_scan_top, dim3(1), dim3(SCAN_T), 0, st, U32(P.o_bs), nb));
  ZKB_TRY(launch("scan_add", k_scan_add, dim3((P.nseg + 255) / 256), dim3(256), 0, st, U32(P.o_off),
                 U32(P.o_cur), (const uint32_t*)U32(P.o_bs), P.nseg, nb));
  ZKB_TRY(launch("msm_scatter", k_msm_scatter, dim3((n + 255) / 256), dim3(256), 0, st, n, scal, P.nw, P.c,
                 P.nwin, P.B, U32(P.o_cur), U32(P.o_ent)));
  const uint32_t* bases = reinterpret_cast<const uint32_t*>(d_bases);
  if (first) ZKB_CUDA(cudaEventRecord(cx.ev_phase[1], st));
  if (bases_ready) ZKB_CUDA(cudaStreamWaitEvent(st, bases_ready, 0));
  const dim3 g1((P.nch[0] + 255) / 256);
  const uint32_t* ent = U32(P.o_ent);
  const uint32_t* off = U32(P.o_off);
  switch (P.L1) {
    case 256: ZKB_TRY(launch("msm_accum", k_msm_accum<C, 256>, g1, dim3(256), 0, st, ent, off, P.nseg, P.nch[0], bases, U32(P.o_bsum), U32(P.o_keyA), U32(P.o_ptA))); break;
    case 128: ZKB_TRY(launch("msm_accum", k_msm_accum<C, 128>, g1, dim3(256), 0, st, ent, off, P.nseg, P.nch[0], bases, U32(P.o_bsum), U32(P.o_keyA), U32(P.o_ptA))); break;
    case 64: ZKB_TRY(launch("msm_accum", k_msm_accum<C, 64>, g1, dim3(256), 0, st, ent, off, P.nseg, P.nch[0], bases, U32(P.o_bsum), U32(P.o_keyA), U32(P.o_ptA))); break;
    case 32: ZKB_TRY(launch("msm_accum", k_msm_accum<C, 32>, g1, dim3(256), 0, st, ent, off, P.nseg, P.nch[0], bases, U32(P.o_bsum), U32(P.o_keyA), U32(P.o_ptA))); break;
    case 16: ZKB_TRY(launch("msm_accum", k_msm_accum<C, 16>, g1, dim3(256), 0, st, ent, off, P.nseg, P.nch[0], bases, U32(P.o_bsum), U32(P.o_keyA), U32(P.o_ptA))); break;
    default: ZKB_TRY(launch("msm_accum", k_msm_accum<C, 8>, g1, dim3(256), 0, st, ent, off, P.nseg, P.nch[0], bases, U32(P.o_bsum), U32(P.o_keyA), U32(P.o_ptA))); break;
  }
  if (last) ZKB_CUDA(cudaEventRecord(cx.ev_phase[2], st));
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
    ZKB_TRY(launch("msm_seg_level", k_msm_seg_level<C>, dim3((ch + 255) / 256), dim3(256), 0, st, ik, ip,
                   (uint32_t)P.Ylev[k], P.Llev[k], ch, hist, off, U32(P.o_bsum), ok, op));
    hist.L[hist.n++] = P.Llev[k];
  }
  if (last) ZKB_CUDA(cudaEventRecord(cx.ev_phase[3], st));
  return ZKG_OK;
}

// Bucket reduction over the parts' bucket arrays (phase 7) into U of workspace ws0 / plan P0.
template <class C>
static zkg_status msm_launch_reduce(Context& cx, const MsmPlan& P0, char* ws0, const PartSet& parts,
                                    cudaStream_t st) {
  using F = typename C::Fp;
  constexpr int XW = 4 * F::N;
  auto U32 = [&](size_t o) { return reinterpret_cast<uint32_t*>(ws0 + o); };
  const uint32_t nthr = (uint32_t)P0.nwin * P0.G;
  ZKB_TRY(launch("msm_bucket_rs", k_msm_bucket_rs<C>, dim3((nthr + 127) / 128), dim3(128), 0, st, parts, P0.B,
                 (uint32_t)P0.nwin, P0.K1, P0.G, U32(P0.o_T), U32(P0.o_R)));
  const size_t smem = 256 * XW * 4;
  ZKB_TRY(launch("msm_bucket_bits", k_msm_bucket_bits<C>, dim3(P0.nwin, P0.gbits + 1), dim3(256), smem, st,
                 (const uint32_t*)U32(P0.o_T), (const uint32_t*)U32(P0.o_R), P0.G, P0.gbits, U32(P0.o_U)));
  ZKB_CUDA(cudaEventRecord(cx.ev_phase[4], st));
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

// Host buffers. Large MSMs are split into point-range parts: part q's scalars and bases are
// copied on the copy stream while part q-1 sorts and accumulates on the compute stream; one
// bucket reduction then merges the parts' bucket arrays.
template <class C, int NL>
static zkg_status msm_host_entry(const host::Field<NL>& F, int n, const uint64_t* expos, int nlimbs, int mont,
                                 const uint64_t* grps, int kind, uint64_t* tgt) {
  ZKB_TRY(check_msm_args(n, expos, nlimbs, mont, grps, tgt));
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  if (n == 0) {
    host::xyzz_write<NL>(F, host::xyzz_inf<NL>(), kind, tgt);
    return set_status(ZKG_OK, nullptr, nullptr);
  }
  int nparts = g_tune_parts > 0 ? g_tune_parts : (n >= (1 << 19) ? 2 : 1);
  nparts = std::max(1, std::min(4, std::min(nparts, n)));
  const int per = (n + nparts - 1) / nparts;
  nparts = (n + per - 1) / per;
  const int scalar_bits = mont ? C::SCALAR_BITS : 64 * nlimbs;
  const int c = g_window_override > 0 ? g_window_override : auto_window(n, scalar_bits);
  MsmPlan P[4];
  size_t total = 0, off_s[4], off_b[4], off_w[4];
  auto rup = [](size_t x) { return (x + 255) & ~size_t(255); };
  for (int q = 0; q < nparts; q++) {
    const int nq = std::min(per, n - q * per);
    ZKB_TRY(make_plan<C>(nq, nlimbs, mont, P[q], c));
    off_s[q] = total;
    total += rup((size_t)nq * nlimbs * 8);
    off_b[q] = total;
    total += rup((size_t)nq * 2 * NL * 8);
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
  for (int q = 0; q < nparts; q++) {
    const size_t first = (size_t)q * per, nq = P[q].n;
    ZKB_CUDA(cudaMemcpyAsync(base + off_s[q], expos + first * nlimbs, nq * nlimbs * 8, cudaMemcpyHostToDevice,
                             cx.copy_stream));
    ZKB_CUDA(cudaMemcpyAsync(base + off_b[q], grps + first * 2 * NL, nq * 2 * NL * 8, cudaMemcpyHostToDevice,
                             cx.copy_stream));
    ZKB_CUDA(cudaEventRecord(cx.ev_part[q], cx.copy_stream));
    ws[q] = base + off_w[q];
  }
  PartSet parts;
  parts.n = nparts;
  for (int q = 0; q < nparts; q++) {
    ZKB_CUDA(cudaStreamWaitEvent(st, cx.ev_part[q], 0));
    ZKB_TRY(msm_launch_part<C>(cx, P[q], ws[q], reinterpret_cast<const uint64_t*>(base + off_s[q]), mont,
                               reinterpret_cast<const uint64_t*>(base + off_b[q]), st, nullptr, q == 0,
                               q == nparts - 1));
    parts.bsum[q] = reinterpret_cast<const uint32_t*>(ws[q] + P[q].o_bsum);
    parts.off[q] = reinterpret_cast<const uint32_t*>(ws[q] + P[q].o_off);
  }
  ZKB_TRY(msm_launch_reduce<C>(cx, P[0], ws[0], parts, st));
  ZKB_TRY((msm_finish<C, NL>(cx, F, P[0], ws[0], ws, P, nparts, kind, tgt, st)));
  return set_status(ZKG_OK, nullptr, nullptr);
}

// Device-resident inputs: one part.
template <class C, int NL>
static zkg_status msm_dev_entry(const host::Field<NL>& F, int n, const uint64_t* d_expos, int nlimbs, int mont,
                                const uint64_t* d_grps, int kind, uint64_t* tgt) {
  ZKB_TRY(check_msm_args(n, d_expos, nlimbs, mont, d_grps, tgt));
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
  ZKB_TRY(make_plan<C>(n, nlimbs, mont, P));
  ZKB_TRY(cx.arena.reserve(P.bytes));
  cx.arena.reset();
  char* ws = static_cast<char*>(cx.arena.take(P.bytes));
  if (!ws) return set_status(ZKG_ERR_NOMEM, "msm", "arena");
  const cudaStream_t st = cx.compute();
  ZKB_TRY(msm_launch_part<C>(cx, P, ws, d_expos, mont, d_grps, st, nullptr, true, true));
  PartSet parts;
  parts.n = 1;
  parts.bsum[0] = reinterpret_cast<const uint32_t*>(ws + P.o_bsum);
  parts.off[0] = reinterpret_cast<const uint32_t*>(ws + P.o_off);
  ZKB_TRY(msm_launch_reduce<C>(cx, P, ws, parts, st));
  ZKB_TRY((msm_finish<C, NL>(cx, F, P, ws, &ws, &P, 1, kind, tgt, st)));
  return set_status(ZKG_OK, nullptr, nullptr);
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

int zkg_set_msm_window(int c) {
  const int prev = zkb::g_window_override;
  zkb::g_window_override = c < 0 ? 0 : c;
  return prev;
}

int zkg_msm_window_for(zkg_curve curve, int npoints) {
  if (zkb::g_window_override > 0) return zkb::g_window_override;
  return zkb::auto_window(npoints, curve == ZKG_BLS12_381 ? zkb::BLS12_381::SCALAR_BITS : zkb::BN254::SCALAR_BITS);
}

}  // extern "C"
