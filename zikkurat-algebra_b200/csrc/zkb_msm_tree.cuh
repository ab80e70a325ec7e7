// The first levels of the MSM bucket accumulation as a tree of affine additions.
//
// Level l turns each bucket segment's m elements into ceil(m / 2): elements 2j and 2j + 1 are
// added, an odd last element is carried. An affine sum P0 + P1 needs one field inversion
// (lambda = (y1 - y0) / (x1 - x0), or 3 x0^2 / (2 y0) when P0 = P1); a whole level shares its
// inversions by Montgomery's simultaneous-inversion trick, so one addition costs six field
// products (one running product, two in the backward pass, lambda, lambda^2 and y3) against ten
// for the mixed XYZZ addition of the chunk accumulation (madd-2008-s). One level:
//   1. output offsets: exclusive scan of ceil(m_s / 2) over the segments (the sort's scan kernels);
//   2. k_tree_fwd: each thread takes B consecutive output slots, forms their denominators and
//      stores the running product before each one; the thread's whole product goes to tt;
//   3. k_tree_inv: tt is inverted in place (simultaneous inversion again, one binary-Euclid
//      inversion per block);
//   4. k_tree_bwd: each thread walks its slots backwards, peeling one denominator inverse per slot
//      off the inverse of its product, and writes each slot's sum as canonical affine coordinates.
// The short segments left after the last level go through the XYZZ chunk accumulation, whose
// entries are then the identity map onto the last level's list. The identity point is (0, 0)
// everywhere, as in the reference's affine test (bn128_G1_affine.c:57-60), and a sum P + (-P)
// becomes (0, 0). The bases must be canonical (coordinates below p), as the reference's field
// operations assume: the equality tests compare words.
#pragma once
#include "zkb_batch_inv.cuh"
#include "zkb_msm_accum.cuh"

namespace zkb {

enum : uint32_t { TREE_COPY0 = 0, TREE_COPY1 = 1, TREE_INF = 2, TREE_ADD = 3, TREE_DBL = 4 };

// input element i of a level: level 0 gathers a base through the sorted entries (point index,
// negation in bit 31); later levels read the previous level's list
template <class F, bool L0>
__device__ __forceinline__ const uint32_t* tree_elem(const uint32_t* __restrict__ ent,
                                                     const uint32_t* __restrict__ pts, uint32_t i, uint32_t npts,
                                                     uint32_t* chk, bool& neg) {
  constexpr int AW = 2 * F::N;
  if constexpr (L0) {
    const uint32_t e = __ldg(ent + i);
    neg = (e >> 31) != 0;
    uint32_t k = e & 0x7fffffffu;
    if (chk && k >= npts) {
      atomicOr(chk, CHK_POINT);
      k = 0;
    }
    return pts + (size_t)k * AW;
  } else {
    neg = false;
    return pts + (size_t)i * AW;
  }
}

// y of an input, negated for a negative digit (canonically: p - y, and 0 stays 0)
template <class F>
__device__ __forceinline__ Fe<F> tree_y(const uint32_t* p, bool neg) {
  const Fe<F> y = fe_load_nc<F>(p + F::N);
  return neg ? fe_canon(fe_neg(y)) : y;
}

// what the slot's sum is: a copy of one input (the other is the identity), the identity
// (both are, or P + (-P)), an addition or a doubling
template <class F>
__device__ __forceinline__ uint32_t tree_kind(const Fe<F>& x0, const Fe<F>& y0, const Fe<F>& x1, const Fe<F>& y1) {
  const bool inf0 = fe_is_zero(x0) && fe_is_zero(y0);
  const bool inf1 = fe_is_zero(x1) && fe_is_zero(y1);
  if (inf0) return inf1 ? TREE_INF : TREE_COPY1;
  if (inf1) return TREE_COPY0;
  if (!fe_eq(x0, x1)) return TREE_ADD;
  return fe_eq(y0, y1) ? TREE_DBL : TREE_INF;
}

// ceil(m_s / 2) per segment (the next level's element counts)
__global__ void k_tree_counts(const uint32_t* __restrict__ in_off, uint32_t nseg, uint32_t* __restrict__ cnt) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nseg) cnt[s] = (__ldg(in_off + s + 1) - __ldg(in_off + s) + 1) >> 1;
}

// Position of output slot q of a level: its segment s, the segment's output slots [o_lo, o_hi) and
// input elements [i_lo, i_hi); the slot adds inputs i0 and i0 + 1, or carries i0 alone.
struct TreeSlot {
  uint32_t q, s, o_lo, o_hi, i_lo, i_hi;
  __device__ __forceinline__ uint32_t i0() const { return i_lo + 2 * (q - o_lo); }
  __device__ __forceinline__ bool pair() const { return i0() + 1 < i_hi; }
};

__device__ __forceinline__ TreeSlot tree_slot_at(const uint32_t* __restrict__ out_off,
                                                 const uint32_t* __restrict__ in_off, uint32_t nseg, uint32_t q) {
  TreeSlot it;
  it.q = q;
  it.s = find_seg(out_off, nseg, q);
  it.o_lo = __ldg(out_off + it.s);
  it.o_hi = __ldg(out_off + it.s + 1);
  it.i_lo = __ldg(in_off + it.s);
  it.i_hi = __ldg(in_off + it.s + 1);
  return it;
}

// the next slot (the caller knows one exists, so the segment walk stays below nseg)
__device__ __forceinline__ void tree_next(TreeSlot& it, const uint32_t* __restrict__ out_off,
                                          const uint32_t* __restrict__ in_off) {
  it.q++;
  while (it.q >= it.o_hi) {
    it.s++;
    it.o_lo = it.o_hi;
    it.o_hi = __ldg(out_off + it.s + 1);
    it.i_lo = it.i_hi;
    it.i_hi = __ldg(in_off + it.s + 1);
  }
}

// the previous slot (the caller knows q > 0, so the walk stays at or above segment 0)
__device__ __forceinline__ void tree_prev(TreeSlot& it, const uint32_t* __restrict__ out_off,
                                          const uint32_t* __restrict__ in_off) {
  it.q--;
  while (it.q < it.o_lo) {
    it.s--;
    it.o_hi = it.o_lo;
    it.o_lo = __ldg(out_off + it.s);
    it.i_hi = it.i_lo;
    it.i_lo = __ldg(in_off + it.s);
  }
}

// negation flag of input element i (level 0: bit 31 of its entry)
template <bool L0>
__device__ __forceinline__ bool tree_neg(const uint32_t* __restrict__ ent, uint32_t i) {
  if constexpr (L0) return (__ldg(ent + i) >> 31) != 0;
  else return false;
}

template <class F>
__device__ __forceinline__ Fe<F> fe_from_smem(const uint4* __restrict__ sm, int stride) {
  Fe<F> r;
#pragma unroll
  for (int k = 0; k < F::N / 4; k++) {
    const uint4 x = sm[k * stride];
    r.v[4 * k + 0] = x.x; r.v[4 * k + 1] = x.y; r.v[4 * k + 2] = x.z; r.v[4 * k + 3] = x.w;
  }
  return r;
}

// Shared memory of the tree passes: per thread and prefetch stage, the x coordinates of a slot's
// two inputs (forward pass), or both inputs and the slot's running product (backward pass), as
// 16-byte pieces; piece k of stage g of thread i at [(g * pieces + k) * NT + i].
template <class F>
constexpr int tree_fwd_pieces() { return 2 * (F::N / 4); }
template <class F>
constexpr int tree_bwd_pieces() { return 4 * (F::N / 4) + F::N / 4; }

// Forward pass: thread t owns output slots [t B, t B + B). pre[q] = product of the denominators
// of the thread's addition slots before q (stored for addition slots after the first slot);
// tt[t] = product of all of them (1 when none). The inputs' x coordinates arrive through PF
// cp.async stages, PF - 1 slots ahead.
template <class C, bool L0, int NT, int PF>
__global__ void __launch_bounds__(NT) k_tree_fwd(const uint32_t* __restrict__ ent, const uint32_t* __restrict__ pts,
                                                 const uint32_t* __restrict__ in_off,
                                                 const uint32_t* __restrict__ out_off, uint32_t nseg, uint32_t B,
                                                 uint32_t nthr, uint32_t* __restrict__ pre,
                                                 uint32_t* __restrict__ tt, uint32_t* chk, uint32_t npts) {
  using F = typename C::Fp;
  constexpr int FW = F::N, QF = F::N / 4, QS = tree_fwd_pieces<F>();
  extern __shared__ uint4 tsm[];
  const uint32_t t = blockIdx.x * NT + threadIdx.x;
  if (t >= nthr) return;
  const uint32_t Q = __ldg(out_off + nseg);
  const uint64_t q0l = (uint64_t)t * B;
  Fe<F> acc = fe_one<F>();
  if (q0l < Q) {
    const uint32_t q0 = (uint32_t)q0l;
    const uint32_t q1 = (uint32_t)min(q0l + (uint64_t)B, (uint64_t)Q);
    TreeSlot ci = tree_slot_at(out_off, in_off, nseg, q0);
    TreeSlot ii = ci;
    bool more = true;
    auto issue = [&](int stage) {
      if (more) {
        if (ii.pair()) {
          bool ng;
          const uint4* p0 = reinterpret_cast<const uint4*>(tree_elem<F, L0>(ent, pts, ii.i0(), npts, chk, ng));
          const uint4* p1 = reinterpret_cast<const uint4*>(tree_elem<F, L0>(ent, pts, ii.i0() + 1, npts, chk, ng));
#pragma unroll
          for (int k = 0; k < QF; k++) {
            cp_async16(&tsm[(stage * QS + k) * NT + threadIdx.x], p0 + k);
            cp_async16(&tsm[(stage * QS + QF + k) * NT + threadIdx.x], p1 + k);
          }
        }
        if (ii.q + 1 < q1) tree_next(ii, out_off, in_off);
        else more = false;
      }
      cp_async_commit();   // possibly empty: one group per slot keeps the wait count fixed
    };
#pragma unroll
    for (int k = 0; k < PF - 1; k++) issue(k);
    for (uint32_t idx = 0;; idx++) {
      issue((int)((idx + PF - 1) % PF));
      cp_async_wait<PF - 1>();   // this slot's group has landed
      if (ci.pair()) {
        const int stage = (int)(idx % PF);
        const Fe<F> x0 = fe_from_smem<F>(&tsm[(stage * QS) * NT + threadIdx.x], NT);
        const Fe<F> x1 = fe_from_smem<F>(&tsm[(stage * QS + QF) * NT + threadIdx.x], NT);
        Fe<F> den;
        bool add = true;
        if (!fe_eq(x0, x1) && !fe_is_zero(x0) && !fe_is_zero(x1)) {   // the common case needs no y
          den = fe_sub(x1, x0);
        } else {
          bool n0, n1;
          const uint32_t* p0 = tree_elem<F, L0>(ent, pts, ci.i0(), npts, chk, n0);
          const uint32_t* p1 = tree_elem<F, L0>(ent, pts, ci.i0() + 1, npts, chk, n1);
          const Fe<F> y0 = tree_y<F>(p0, n0), y1 = tree_y<F>(p1, n1);
          const uint32_t kind = tree_kind(x0, y0, x1, y1);
          if (kind == TREE_ADD) den = fe_sub(x1, x0);
          else if (kind == TREE_DBL) den = fe_add(y0, y0);
          else add = false;
        }
        if (add) {
          if (ci.q > q0) fe_store<F>(pre + (size_t)ci.q * FW, acc);
          acc = fe_mul(acc, den);
        }
      }
      if (ci.q + 1 >= q1) break;
      tree_next(ci, out_off, in_off);
    }
    cp_async_wait<0>();
  }
  fe_store<F>(tt + (size_t)t * FW, acc);
}

// tt[0, n) <- their inverses (all non-zero mod p), by simultaneous inversion over each thread's
// strided subset (running products in scr) with one inversion per block of 256 threads
template <class F>
__global__ void __launch_bounds__(256) k_tree_inv(uint32_t n, uint32_t* __restrict__ tt, uint32_t* __restrict__ scr) {
  constexpr int FW = F::N;
  __shared__ Fe<F> sw[9];
  __shared__ Fe<F> s_inv;
  const size_t T = (size_t)gridDim.x * blockDim.x;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  Fe<F> acc = fe_one<F>();
  size_t last = t;
  for (size_t i = t; i < (size_t)n; i += T) {
    acc = fe_mul(acc, fe_load<F>(tt + i * FW));
    fe_store<F>(scr + i * FW, acc);
    last = i;
  }
  Fe<F> total, total2;
  const Fe<F> before = block_mul_excl_scan<F, false>(acc, sw, total);
  const Fe<F> after = block_mul_excl_scan<F, true>(acc, sw, total2);
  if (threadIdx.x == 0) s_inv = fe_inv_binary(fe_canon(total));
  __syncthreads();
  if (t >= (size_t)n) return;
  Fe<F> inv = fe_mul(fe_mul(s_inv, before), after);   // inverse of this thread's product
  for (size_t i = last;; i -= T) {
    const Fe<F> x = fe_load<F>(tt + i * FW);
    fe_store<F>(tt + i * FW, i >= t + T ? fe_mul(inv, fe_load<F>(scr + (i - T) * FW)) : inv);
    inv = fe_mul(inv, x);
    if (i < t + T) break;
  }
}

// Backward pass: thread t walks its slots from the last; acc is the inverse of the product of
// the denominators not yet peeled off, so a slot's inverse is acc * pre[q] and the next acc is
// acc * den. Every slot's sum is written, canonical, to out. A slot's inputs and running product
// arrive through PF cp.async stages, PF - 1 slots ahead.
template <class C, bool L0, int NT, int PF>
__global__ void __launch_bounds__(NT, 1) k_tree_bwd(const uint32_t* __restrict__ ent, const uint32_t* __restrict__ pts,
                                                    const uint32_t* __restrict__ in_off,
                                                    const uint32_t* __restrict__ out_off, uint32_t nseg, uint32_t B,
                                                    uint32_t nthr, const uint32_t* __restrict__ pre,
                                                    const uint32_t* __restrict__ tinv, uint32_t* __restrict__ out,
                                                    uint32_t* chk, uint32_t npts) {
  using F = typename C::Fp;
  constexpr int FW = F::N, AW = 2 * F::N, QF = F::N / 4, QA = 2 * QF, QS = tree_bwd_pieces<F>();
  extern __shared__ uint4 tsm[];
  const uint32_t t = blockIdx.x * NT + threadIdx.x;
  if (t >= nthr) return;
  const uint32_t Q = __ldg(out_off + nseg);
  const uint64_t q0l = (uint64_t)t * B;
  if (q0l >= Q) return;
  const uint32_t q0 = (uint32_t)q0l;
  const uint32_t q1 = (uint32_t)min(q0l + (uint64_t)B, (uint64_t)Q);
  Fe<F> acc = fe_load_nc<F>(tinv + (size_t)t * FW);
  TreeSlot ci = tree_slot_at(out_off, in_off, nseg, q1 - 1);
  TreeSlot ii = ci;
  bool more = true;
  auto issue = [&](int stage) {
    if (more) {
      bool ng;
      const uint4* p0 = reinterpret_cast<const uint4*>(tree_elem<F, L0>(ent, pts, ii.i0(), npts, chk, ng));
#pragma unroll
      for (int k = 0; k < QA; k++) cp_async16(&tsm[(stage * QS + k) * NT + threadIdx.x], p0 + k);
      if (ii.pair()) {
        const uint4* p1 = reinterpret_cast<const uint4*>(tree_elem<F, L0>(ent, pts, ii.i0() + 1, npts, chk, ng));
#pragma unroll
        for (int k = 0; k < QA; k++) cp_async16(&tsm[(stage * QS + QA + k) * NT + threadIdx.x], p1 + k);
        if (ii.q > q0) {
          const uint4* pp = reinterpret_cast<const uint4*>(pre + (size_t)ii.q * FW);
#pragma unroll
          for (int k = 0; k < QF; k++) cp_async16(&tsm[(stage * QS + 2 * QA + k) * NT + threadIdx.x], pp + k);
        }
      }
      if (ii.q > q0) tree_prev(ii, out_off, in_off);
      else more = false;
    }
    cp_async_commit();   // possibly empty: one group per slot keeps the wait count fixed
  };
#pragma unroll
  for (int k = 0; k < PF - 1; k++) issue(k);
  for (uint32_t idx = 0;; idx++) {
    issue((int)((idx + PF - 1) % PF));
    cp_async_wait<PF - 1>();   // this slot's group has landed
    const int stage = (int)(idx % PF);
    const uint4* sa = &tsm[(stage * QS) * NT + threadIdx.x];
    const uint32_t q = ci.q, i0 = ci.i0();
    Affine<F> a;
    a.x = fe_from_smem<F>(sa, NT);
    a.y = fe_from_smem<F>(sa + QF * NT, NT);
    if (tree_neg<L0>(ent, i0)) a.y = fe_canon(fe_neg(a.y));
    Affine<F> r = a;   // a carried element
    if (ci.pair()) {
      Affine<F> b;
      b.x = fe_from_smem<F>(sa + QA * NT, NT);
      b.y = fe_from_smem<F>(sa + (QA + QF) * NT, NT);
      if (tree_neg<L0>(ent, i0 + 1)) b.y = fe_canon(fe_neg(b.y));
      const uint32_t kind = tree_kind(a.x, a.y, b.x, b.y);
      if (kind == TREE_COPY1) {
        r = b;
      } else if (kind == TREE_INF) {
        r.x = fe_zero<F>();
        r.y = fe_zero<F>();
      } else if (kind >= TREE_ADD) {
        const Fe<F> den = kind == TREE_ADD ? fe_sub(b.x, a.x) : fe_add(a.y, a.y);
        Fe<F> inv;
        if (q > q0) {
          Fe<F> nacc;
          fe_mul2(inv, acc, fe_from_smem<F>(sa + 2 * QA * NT, NT), nacc, acc, den);
          acc = nacc;
        } else {
          inv = acc;
        }
        Fe<F> num;
        if (kind == TREE_ADD) {
          num = fe_sub(b.y, a.y);
        } else {
          const Fe<F> xx = fe_sqr(a.x);
          num = fe_add(fe_add(xx, xx), xx);
        }
        const Fe<F> lam = fe_mul(num, inv);
        const Fe<F> x3 = fe_sub(fe_sub(fe_sqr(lam), a.x), b.x);
        const Fe<F> y3 = fe_sub(fe_mul(lam, fe_sub(a.x, x3)), a.y);
        r.x = fe_canon(x3);
        r.y = fe_canon(y3);
      }
    }
    fe_store<F>(out + (size_t)q * AW, r.x);
    fe_store<F>(out + (size_t)q * AW + FW, r.y);
    if (q == q0) break;
    tree_prev(ci, out_off, in_off);
  }
  cp_async_wait<0>();
}

}  // namespace zkb
