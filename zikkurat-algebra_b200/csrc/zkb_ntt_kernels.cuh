// NTT kernels: radix-2 NTT over Fr (BN254, BLS12-381) for B200 (sm_100a).
//
// Reference: lib/cbits/curves/poly/mont/bn128_poly_mont.c:418-473 (forward: recursive radix-2
// decimation in time, twiddles g^j, natural order in and out) and :565-622 (inverse: recursive
// decimation in frequency, each stage halves, twiddles g^-j / 2).
//
// Factorisation used here. Write the reference's forward network with generator g on
// N = 2^m points as F_g. For N = N1*N2 (N1 = 2^k) it satisfies, for every g,
//     F_g(x)[k1 + N1*k2] = F_{g^N1}( r -> g^(r*k1) * F_{g^N2}( t -> x[r + N2*t] )[k1] )[k2]
// with r < N2, t, k1 < N1 and the literal power g^(r*k1) (exponent < N, never reduced), which
// follows from unrolling the recursion; for a generator of order N it is the four-step DFT.
// Applying it recursively gives passes of 2^k-point networks with a twiddle multiply between
// passes. The reference's inverse network is the transpose of F_{g^-1} times (1/2)^m, so the
// inverse runs the transposed passes in reverse order: twiddle first, then a 2^k-point
// decimation-in-frequency network. Every butterfly and twiddle is an exact field operation on
// the same powers of g as the reference, so results are bit-identical, for any `gen`.
//
// Pass p (forward order) has k bits, s bits already done and M' = m - s - k bits after it.
// Column c in [0, 2^(m-k)), row t / output k1 in [0, 2^k):
//     forward reads  x[in(c,t)],  in(c,t)  = (c mod 2^M') + ((c >> M') << (M'+k)) + (t << M')
//     forward writes y[out(c,k1)], out(c,k1) = c + (k1 << (m-k)), times g^(((c mod 2^M')*k1) << s)
// A CTA owns a tile of consecutive columns, so every global access is a run of consecutive
// 32-byte elements. The tile lives in shared memory; each thread runs 2 butterfly stages at a
// time on 4 elements held in registers (NTT_RS).
#pragma once
#include "zkb_field.cuh"
#include "zkb_ntt.h"

namespace zkb {

static constexpr int FRW = 8;            // 32-bit words per Fr element
// Butterfly stages per register round: each thread holds 2^NTT_RS elements between shared-memory
// exchanges. Two stages (4 elements) keep the pass kernels free of register spills at two CTAs per
// SM; three stages (8 elements) spilled up to 176 bytes and measured slower (2^24 forward 5.41 ->
// 5.08 ms, inverse 5.63 -> 5.10 ms with two). A spill-free three-CTA shape does not exist: at 80
// registers the out-of-line product spills.
static constexpr int NTT_RS = 2;

__device__ __forceinline__ uint32_t bitrev_k(uint32_t x, int k) { return __brev(x) >> (32 - k); }

// Shared-memory tile: element idx is two 16-byte chunks 2 idx, 2 idx + 1, stored at chunk
// c ^ ((c >> 4) & 7). The XOR spreads accesses whose element indices differ by multiples of 8
// (the stride of the first butterfly round, and of transposed reads) over all eight 16-byte bank
// groups; both halves of an element stay in one 128-byte row.
__device__ __forceinline__ uint32_t sm_chunk(uint32_t c) { return c ^ ((c >> 4) & 7u); }
template <class P>
__device__ __forceinline__ Fe<P> sm_ld(const uint32_t* sm, uint32_t idx) {
  static_assert(P::N == 8, "tile elements are 32 bytes");
  const uint4* q = reinterpret_cast<const uint4*>(sm);
  const uint4 x = q[sm_chunk(2 * idx)], y = q[sm_chunk(2 * idx + 1)];
  Fe<P> r;
  r.v[0] = x.x; r.v[1] = x.y; r.v[2] = x.z; r.v[3] = x.w;
  r.v[4] = y.x; r.v[5] = y.y; r.v[6] = y.z; r.v[7] = y.w;
  return r;
}
template <class P>
__device__ __forceinline__ void sm_st(uint32_t* sm, uint32_t idx, const Fe<P>& a) {
  uint4* q = reinterpret_cast<uint4*>(sm);
  q[sm_chunk(2 * idx)] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
  q[sm_chunk(2 * idx + 1)] = make_uint4(a.v[4], a.v[5], a.v[6], a.v[7]);
}

// Run network stages [s0, s0+r) on every group of the tile. A group is 2^r positions
// base + i*2^(s0-1) within one column. DIT processes stages upward, DIF downward.
template <class P, int K, bool DIT, int r>
__device__ __forceinline__ void ntt_round(uint32_t* sm, int W, int s0, const uint32_t* __restrict__ om) {
  constexpr int gsize = 1 << r;
  const uint32_t ngroups_col = 1u << (K - r);
  const uint32_t ngroups = (uint32_t)W * ngroups_col;
  const uint32_t d = 1u << (s0 - 1);
  for (uint32_t gi = threadIdx.x; gi < ngroups; gi += blockDim.x) {
    const uint32_t col = gi >> (K - r);
    const uint32_t gl = gi & (ngroups_col - 1);
    // base: insert r zero bits at position s0-1 into gl
    const uint32_t lowmask = d - 1;
    const uint32_t base = (gl & lowmask) | ((gl & ~lowmask) << r);
    const uint32_t cbase = col << K;
    Fe<P> a[8];
#pragma unroll
    for (int i = 0; i < 8; i++)
      if (i < gsize) a[i] = sm_ld<P>(sm, cbase + base + i * d);
    const uint32_t jlow = base & lowmask;   // common low bits of j
#pragma unroll
    for (int q = 0; q < r; q++) {
      const int st = DIT ? q : (r - 1 - q);         // local stage index
      const int s = s0 + st;                         // network stage, pair distance 2^(s-1)
      const int hd = 1 << st;                        // distance in group slots
#pragma unroll
      for (int i = 0; i < 8; i++) {
        if (i >= gsize || (i & hd)) continue;
        // j = position mod 2^(s-1) = jlow + (i mod hd) * d
        const uint32_t j = jlow + (uint32_t)(i & (hd - 1)) * d;
        const uint32_t e = j << (K - s);
        // twiddle om[0] = 1: skipped where j = 0 is known at compile time (stage 1, and every
        // stage of the round that starts at stage 1, where jlow = 0 and d = 1); the product
        // by one would return the same element
        const bool unit = (s == 1) || (s0 == 1 && (i & (hd - 1)) == 0);
        Fe<P>& u = a[i];
        Fe<P>& v = a[i + hd];
        if (DIT) {
          const Fe<P> tv = unit ? v : fe_mul(v, fe_load_nc<P>(om + e * FRW));
          const Fe<P> nu = fe_add(u, tv);
          v = fe_sub(u, tv);
          u = nu;
        } else {
          const Fe<P> sum = fe_add(u, v);
          const Fe<P> dif = fe_sub(u, v);
          u = sum;
          v = unit ? dif : fe_mul(dif, fe_load_nc<P>(om + e * FRW));
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
      if (i < gsize) sm_st<P>(sm, cbase + base + i * d, a[i]);
  }
}

// Forward pass: gather columns (bit-reversed into shared memory), DIT network, twiddle, scatter.
// ntt_fwd_tile runs tile blk (W consecutive columns) with the tile in sm; CG = true reads the
// input through L2 only (input written earlier by other CTAs of the same persistent kernel).
template <class P, int K, bool CG>
__device__ __forceinline__ void ntt_fwd_tile(uint32_t blk, const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                             int m, int Mp, int s, const uint32_t* __restrict__ om,
                                             const uint32_t* __restrict__ tw, int W, uint32_t* sm) {
  const uint32_t ncols = 1u << (m - K);
  const uint32_t c0 = blk * (uint32_t)W;
  const uint32_t wcols = min((uint32_t)W, ncols - c0);
  const uint32_t mM = (1u << Mp) - 1;
  const uint32_t nel = wcols << K;
  for (uint32_t idx = threadIdx.x; idx < nel; idx += blockDim.x) {
    uint32_t ci, t;
    if (Mp == 0) { ci = idx >> K; t = idx & ((1u << K) - 1); }
    else { ci = idx % wcols; t = idx / wcols; }
    const uint32_t c = c0 + ci;
    const size_t src = (size_t)(c & mM) + ((size_t)(c >> Mp) << (Mp + K)) + ((size_t)t << Mp);
    sm_st<P>(sm, (ci << K) + bitrev_k(t, K), CG ? fe_load_cg<P>(in + src * FRW) : fe_load_nc<P>(in + src * FRW));
  }
  __syncthreads();
#pragma unroll
  for (int s0 = 1; s0 <= K; s0 += NTT_RS) {
    const int r = K - s0 + 1;
    if (r >= 3 && NTT_RS >= 3) ntt_round<P, K, true, (K >= 3 ? 3 : 1)>(sm, (int)wcols, s0, om);
    else if (r >= 2) ntt_round<P, K, true, (K >= 2 ? 2 : 1)>(sm, (int)wcols, s0, om);
    else ntt_round<P, K, true, 1>(sm, (int)wcols, s0, om);
    __syncthreads();
  }
  for (uint32_t idx = threadIdx.x; idx < nel; idx += blockDim.x) {
    const uint32_t ci = idx % wcols, k1 = idx / wcols;
    const uint32_t c = c0 + ci;
    Fe<P> v = sm_ld<P>(sm, (ci << K) + k1);
    if (tw) v = fe_mul(v, fe_load_nc<P>(tw + (size_t)((((c & mM) * k1) << s)) * FRW));
    fe_store<P>(out + ((size_t)c + ((size_t)k1 << (m - K))) * FRW, v);
  }
}

template <class P, int K>
__global__ void __launch_bounds__(NTT_THREADS, 2) k_ntt_fwd(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                         int m, int Mp, int s, const uint32_t* __restrict__ om,
                                                         const uint32_t* __restrict__ tw, int W) {
  extern __shared__ uint4 smem_u4[];
  ntt_fwd_tile<P, K, false>(blockIdx.x, in, out, m, Mp, s, om, tw, W, reinterpret_cast<uint32_t*>(smem_u4));
}

// Inverse (transposed) pass: gather the forward pass's outputs, twiddle, DIF network,
// scatter to the forward pass's input positions (bit-reversed read-out), optional scale.
template <class P, int K, bool CG>
__device__ __forceinline__ void ntt_inv_tile(uint32_t blk, const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                             int m, int Mp, int s, const uint32_t* __restrict__ om,
                                             const uint32_t* __restrict__ tw, const uint32_t* __restrict__ scale,
                                             int W, uint32_t* sm) {
  const uint32_t ncols = 1u << (m - K);
  const uint32_t c0 = blk * (uint32_t)W;
  const uint32_t wcols = min((uint32_t)W, ncols - c0);
  const uint32_t mM = (1u << Mp) - 1;
  const uint32_t nel = wcols << K;
  for (uint32_t idx = threadIdx.x; idx < nel; idx += blockDim.x) {
    const uint32_t ci = idx % wcols, k1 = idx / wcols;
    const uint32_t c = c0 + ci;
    const uint32_t* src = in + ((size_t)c + ((size_t)k1 << (m - K))) * FRW;
    Fe<P> v = CG ? fe_load_cg<P>(src) : fe_load_nc<P>(src);
    if (tw) v = fe_mul(v, fe_load_nc<P>(tw + (size_t)((((c & mM) * k1) << s)) * FRW));
    sm_st<P>(sm, (ci << K) + k1, v);
  }
  __syncthreads();
  // DIF: stages K..1 in the forward pass's groups of NTT_RS (1-2, 3-4, ...), last group first, so
  // the final round starts at stage 1 and skips its unit twiddles
#pragma unroll
  for (int s0 = 1 + NTT_RS * ((K - 1) / NTT_RS); s0 >= 1; s0 -= NTT_RS) {
    const int r = K - s0 + 1;
    if (r >= 3 && NTT_RS >= 3) ntt_round<P, K, false, (K >= 3 ? 3 : 1)>(sm, (int)wcols, s0, om);
    else if (r >= 2) ntt_round<P, K, false, (K >= 2 ? 2 : 1)>(sm, (int)wcols, s0, om);
    else ntt_round<P, K, false, 1>(sm, (int)wcols, s0, om);
    __syncthreads();
  }
  Fe<P> sc;
  if (scale) sc = fe_load<P>(scale);
  for (uint32_t idx = threadIdx.x; idx < nel; idx += blockDim.x) {
    uint32_t ci, t;
    if (Mp == 0) { ci = idx >> K; t = idx & ((1u << K) - 1); }
    else { ci = idx % wcols; t = idx / wcols; }
    const uint32_t c = c0 + ci;
    Fe<P> v = sm_ld<P>(sm, (ci << K) + bitrev_k(t, K));
    if (scale) v = fe_mul(v, sc);
    const size_t dst = (size_t)(c & mM) + ((size_t)(c >> Mp) << (Mp + K)) + ((size_t)t << Mp);
    fe_store<P>(out + dst * FRW, v);
  }
}

template <class P, int K>
__global__ void __launch_bounds__(NTT_THREADS, 2) k_ntt_inv(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                         int m, int Mp, int s, const uint32_t* __restrict__ om,
                                                         const uint32_t* __restrict__ tw,
                                                         const uint32_t* __restrict__ scale, int W) {
  extern __shared__ uint4 smem_u4[];
  ntt_inv_tile<P, K, false>(blockIdx.x, in, out, m, Mp, s, om, tw, scale, W, reinterpret_cast<uint32_t*>(smem_u4));
}

// T[e] = A[e mod 2^a] * Bt[e >> a]  (A[j] = h^j, Bt[i] = h^(i*2^a))
template <class P>
__global__ void k_ntt_twiddle_table(uint32_t* __restrict__ T, const uint32_t* __restrict__ A,
                                    const uint32_t* __restrict__ Bt, int a, uint32_t N) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N) return;
  const Fe<P> x = fe_load_nc<P>(A + (size_t)(e & ((1u << a) - 1)) * FRW);
  const Fe<P> y = fe_load_nc<P>(Bt + (size_t)(e >> a) * FRW);
  fe_store<P>(T + (size_t)e * FRW, fe_mul(x, y));
}

template <class P, int K>
static zkg_status launch_pass(const NttPlan& pl, const NttPass& q, const uint32_t* in, uint32_t* out,
                              bool last_inverse, cudaStream_t st) {
  const int E = std::min(8, 1 << K);
  const int W = NTT_THREADS * E >> K;
  const uint32_t ncols = 1u << (pl.m - K);
  const uint32_t grid = (ncols + W - 1) / W;
  const size_t smem = (size_t)W * ((size_t)1 << K) * 32;
  const uint32_t* om = pl.d_om[K];
  const uint32_t* tw = q.Mp > 0 ? pl.d_tw : nullptr;
  if (!pl.inverse) {
    ZKB_CUDA(cudaFuncSetAttribute(k_ntt_fwd<P, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    return launch("ntt_fwd", k_ntt_fwd<P, K>, dim3(grid), dim3(NTT_THREADS), smem, st, in, out, pl.m, q.Mp, q.s, om,
                  tw, W);
  }
  ZKB_CUDA(cudaFuncSetAttribute(k_ntt_inv<P, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
  // the last pass: the (1/2)^m scale rides on the pre-scaled twiddle table when the pass has
  // twiddles, and is a separate product at the end otherwise
  const uint32_t* scale = nullptr;
  if (last_inverse) {
    if (tw && pl.d_tw_last) tw = pl.d_tw_last;
    else scale = pl.d_scale;
  }
  return launch("ntt_inv", k_ntt_inv<P, K>, dim3(grid), dim3(NTT_THREADS), smem, st, in, out, pl.m, q.Mp, q.s, om,
                tw, scale, W);
}

template <class P>
zkg_status ntt_launch_pass(const NttPlan& pl, const NttPass& q, const uint32_t* in, uint32_t* out,
                                bool last_inverse, cudaStream_t st) {
  switch (q.k) {
    case 1: return launch_pass<P, 1>(pl, q, in, out, last_inverse, st);
    case 2: return launch_pass<P, 2>(pl, q, in, out, last_inverse, st);
    case 3: return launch_pass<P, 3>(pl, q, in, out, last_inverse, st);
    case 4: return launch_pass<P, 4>(pl, q, in, out, last_inverse, st);
    case 5: return launch_pass<P, 5>(pl, q, in, out, last_inverse, st);
    case 6: return launch_pass<P, 6>(pl, q, in, out, last_inverse, st);
    case 7: return launch_pass<P, 7>(pl, q, in, out, last_inverse, st);
    case 8: return launch_pass<P, 8>(pl, q, in, out, last_inverse, st);
    case 9: return launch_pass<P, 9>(pl, q, in, out, last_inverse, st);
    case 10: return launch_pass<P, 10>(pl, q, in, out, last_inverse, st);
    case 11: return launch_pass<P, 11>(pl, q, in, out, last_inverse, st);
  }
  return set_status(ZKG_ERR_ARG, "ntt", "pass size");
}


template <class P>
zkg_status ntt_launch_table(uint32_t* T, const uint32_t* A, const uint32_t* Bt, int a, uint32_t N, cudaStream_t st) {
  return launch("ntt_twiddle_table", k_ntt_twiddle_table<P>, dim3((N + 255) / 256), dim3(256), 0, st, T, A, Bt, a, N);
}

}  // namespace zkb
