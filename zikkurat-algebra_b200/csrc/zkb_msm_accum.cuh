// The MSM bucket accumulation's per-block body, shared by the accumulation kernel (zkb_msm.cu)
// and the batch's persistent kernel (zkb_batch_work.cu).
#pragma once
#include "zkb_async.cuh"
#include "zkb_curve.cuh"
#include "zkb_dpf.cuh"
#include "zkb_runtime.h"

namespace zkb {

static constexpr uint32_t INVALID = 0xffffffffu;


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

// BN254: two resident 256-thread blocks per SM (at most 128 registers; measured 20% faster than
// one block with more registers); BLS12-381 needs more registers per thread.

// One block's share of the accumulation (NT chunks: chunk t = blk * NT + threadIdx.x), with the
// base-prefetch stages in `pf` (PF * Q * NT 16-byte pieces of shared memory). The kernel below
// runs it for blockIdx.x; the batch's persistent kernel runs it for the blocks it takes from its
// work queue. entries == nullptr: entry i is point i, positive (the list left by the affine tree
// levels).
template <class C, int PF, int NT = 256>
__device__ __forceinline__ void accum_block(uint32_t blk, const uint32_t* __restrict__ entries,
                                            const uint32_t* __restrict__ off, uint32_t nseg, uint32_t nchunks,
                                            uint32_t L, const uint32_t* __restrict__ bases,
                                            uint32_t* __restrict__ bsum, uint32_t* __restrict__ skey,
                                            uint32_t* __restrict__ spt, uint4* __restrict__ pf,
                                            uint32_t* chk = nullptr, uint32_t npts = 0) {
  using F = typename C::Fp;
  constexpr int AW = 2 * F::N;
  constexpr int Q = AW / 4;   // 16-byte pieces of one affine base
  const uint32_t t = blk * NT + threadIdx.x;
  if (t >= nchunks) return;
  const uint32_t total = __ldg(off + nseg);
  const uint32_t start = t * L;
  uint32_t keyA = INVALID, keyB = INVALID;
  auto ent_at = [&](uint32_t pos) -> uint32_t { return entries ? __ldg(entries + pos) : pos; };
  // point index of an entry; with device checks on, an index outside the base set is recorded and
  // replaced by 0, so no gather leaves the base array
  auto pidx = [&](uint32_t ent) -> uint32_t {
    const uint32_t i = ent & 0x7fffffffu;
    if (chk && i >= npts) {
      atomicOr(chk, CHK_POINT);
      return 0u;
    }
    return i;
  };
  auto issue = [&](uint32_t ent, uint32_t stage) {
    const uint4* src = reinterpret_cast<const uint4*>(bases + (size_t)pidx(ent) * AW);
#pragma unroll
    for (int q = 0; q < Q; q++) cp_async16(&pf[(stage * Q + q) * NT + threadIdx.x], src + q);
    cp_async_commit();
  };
  if (start < total) {
    const uint32_t end = min(start + L, total);
    uint32_t s = find_seg(off, nseg, start);
    uint32_t seg_lo = __ldg(off + s), seg_hi = __ldg(off + s + 1);
    Xyzz<F> acc = xyzz_inf<F>();
    bool have = false;
    uint32_t e = ent_at(start);
    Affine<F> nxt;
    if constexpr (PF > 0) {
#pragma unroll
      for (int k = 0; k < PF - 1; k++)
        if (start + k < end) issue(ent_at(start + k), k);
    } else {
      nxt = affine_load<F>(bases + (size_t)pidx(e) * AW);
    }
    for (uint32_t pos = start; pos < end; pos++) {
      while (pos >= seg_hi) {
        if (have) route_run<F>(s, acc, seg_lo, seg_hi, start, L, t, bsum, spt, keyA, keyB);
        have = false;
        acc = xyzz_inf<F>();
        s++;
        seg_lo = seg_hi;
        seg_hi = __ldg(off + s + 1);
      }
      Affine<F> a;
      uint32_t neg;
      if constexpr (PF > 0) {
        const uint32_t i = pos - start;
        if (i > 0) e = ent_at(pos);
        neg = e >> 31;
        // start the copy PF - 1 bases ahead, then wait for this base's copy (groups issued after
        // it may stay in flight)
        if (pos + PF - 1 < end) issue(ent_at(pos + PF - 1), (i + PF - 1) % PF);
        const uint32_t later = min((uint32_t)(PF - 1), end - 1 - pos);
        if (PF > 2 && later >= 2) cp_async_wait<(PF > 2 ? 2 : 0)>();
        else if (later >= 1) cp_async_wait<1>();
        else cp_async_wait<0>();
        const uint32_t stage = i % PF;
        uint32_t w[AW];
#pragma unroll
        for (int q = 0; q < Q; q++) {
          const uint4 x = pf[(stage * Q + q) * NT + threadIdx.x];
          w[4 * q + 0] = x.x; w[4 * q + 1] = x.y; w[4 * q + 2] = x.z; w[4 * q + 3] = x.w;
        }
#pragma unroll
        for (int k = 0; k < F::N; k++) { a.x.v[k] = w[k]; a.y.v[k] = w[F::N + k]; }
      } else {
        a = nxt;
        neg = e >> 31;
        if (pos + 1 < end) {   // prefetch the next base while this addition runs
          e = ent_at(pos + 1);
          nxt = affine_load<F>(bases + (size_t)pidx(e) * AW);
        }
      }
      // the identity input is (0, 0) exactly (the reference's affine test, bn128_G1_affine.c:57-60;
      // the bases are the caller's canonical coordinates)
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


}  // namespace zkb
