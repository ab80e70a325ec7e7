// Fr vector operations on the device: the reference's *_arr_mont_* module
// (lib/cbits/curves/array/mont/bn128_arr_mont.c:24-278, BLS12-381 twin bls12_381_arr_mont.c)
// and the batch inversion it uses (lib/cbits/curves/fields/mont/bn128_Fr_mont.c:258-285).
//
// These are element-wise, HBM-bound kernels over 4 x 64-bit Montgomery elements (Fr of BN254 and
// of BLS12-381 are both 4 limbs). One grid-stride kernel per operation, with the arithmetic of the
// MSM/NTT kernels (fe_mul, fe_add, fe_sub, fe_neg). Operations whose reference loop carries a
// dependency are restated in parallel form with the same field values:
//   - powers: tgt[i] = A * B^i; thread t starts at A * B^t and steps by B^T (T threads);
//   - mul_by_powers: the reference loop starts at i = 1 with x = A, so tgt[0] is left unwritten
//     and tgt[i] = src[i] * A * B^(i-1) for i >= 1 (bn128_arr_mont.c:203-211); kept as is;
//   - batch inversion: Montgomery's trick over the strided subset i = t, t + T, ... of each
//     thread, the thread products combined across the block by two scans, one inversion (binary
//     extended Euclid) per block. The reference multiplies all n elements into one
//     product and inverts it, so one zero element makes every output zero; a device flag
//     reproduces that;
//   - dot product: block partial sums, then one block sums the partials (modular sums are exact
//     in any order);
//   - sparse matrix times vector (bn128_arr_mont.c:222-233): each non-zero's product is added as
//     eight 32-bit words into eight 64-bit atomic counters per row (no carry is lost: a counter
//     takes 2^32 additions), and the counters are folded mod r at the end:
//     sum_j acc_j 2^(32j) = sum_j mont(acc_j 2^(32j)) via products with 2^(32j) R^2 mod r.
#include <algorithm>
#include <cstring>
#include <vector>

#include "zkb_batch_inv.cuh"
#include "zkb_dpf.cuh"
#include "zkb_field.cuh"
#include "zkb_host_ec.h"
#include "zkb_runtime.h"

namespace zkb {

// Field types of these kernels: Fr with FP64-pipe products in the reference's radix (the same
// results as the 32-bit-limb product; ZKB_FR_DPF=0 selects the latter)
static const bool g_fr_dpf = [] {
  const char* v = std::getenv("ZKB_FR_DPF");
  return !(v && v[0] == '0');
}();

// element-wise kernel shape (ZKB_FR_MAP_MODE): 0 one element per iteration of a grid-stride loop
// over at most 8 blocks per SM (the fastest measured: a BN254 product kernel holds 60 registers, so
// 32 warps per SM keep enough loads in flight; a cp.async prefetch ring through shared memory
// measured 5-25% slower), 1 two elements per iteration with paired products, 2 one thread per
// element
static const int g_fr_map_mode = [] {
  const char* v = std::getenv("ZKB_FR_MAP_MODE");
  return v ? std::atoi(v) : 0;
}();

enum FrOp {
  FR_FROM_STD = ZKG_FR_FROM_STD, FR_TO_STD = ZKG_FR_TO_STD, FR_NEG = ZKG_FR_NEG, FR_ADD = ZKG_FR_ADD,
  FR_SUB = ZKG_FR_SUB, FR_SQR = ZKG_FR_SQR, FR_MUL = ZKG_FR_MUL, FR_INV = ZKG_FR_INV, FR_DIV = ZKG_FR_DIV,
  FR_MUL_ADD = ZKG_FR_MUL_ADD, FR_MUL_SUB = ZKG_FR_MUL_SUB, FR_SCALE = ZKG_FR_SCALE, FR_AXPY = ZKG_FR_AXPY,
  FR_AXPBY = ZKG_FR_AXPBY, FR_POWERS = ZKG_FR_POWERS, FR_MUL_BY_POWERS = ZKG_FR_MUL_BY_POWERS
};

// which inputs an operation reads: bit 0 a, 1 b, 2 c, 3 coefficient A, 4 coefficient B
static int fr_inputs(int op) {
  switch (op) {
    case FR_FROM_STD: case FR_TO_STD: case FR_NEG: case FR_SQR: case FR_INV: return 1;
    case FR_ADD: case FR_SUB: case FR_MUL: case FR_DIV: return 3;
    case FR_MUL_ADD: case FR_MUL_SUB: return 7;
    case FR_SCALE: return 1 | 8;
    case FR_AXPY: return 3 | 8;
    case FR_AXPBY: return 3 | 8 | 16;
    case FR_POWERS: return 8 | 16;
    case FR_MUL_BY_POWERS: return 1 | 8 | 16;
    default: return -1;
  }
}

template <class P>
__device__ __forceinline__ Fe<P> ld(const uint32_t* p, size_t i) { return fe_load<P>(p + 8 * i); }
template <class P>
__device__ __forceinline__ void st(uint32_t* p, size_t i, const Fe<P>& v) { fe_store<P>(p + 8 * i, v); }

// Element-wise operations, one element per iteration of a grid-stride loop (modes 0 and 2; 2 is
// launched with one thread per element). Pointers may alias (the reference's *_inplace forms).
template <class P, int OP>
__global__ void k_fr_map(int n, const uint32_t* a, const uint32_t* b, const uint32_t* c, const uint32_t* ka,
                         const uint32_t* kb, uint32_t* out) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  Fe<P> A, B;
  if (OP == FR_SCALE || OP == FR_AXPY || OP == FR_AXPBY) A = fe_load<P>(ka);
  if (OP == FR_AXPBY) B = fe_load<P>(kb);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) {
    const Fe<P> x = ld<P>(a, i);
    Fe<P> r;
    if (OP == FR_FROM_STD) r = fe_to_mont(x);
    else if (OP == FR_TO_STD) r = fe_from_mont(x);
    else if (OP == FR_NEG) r = fe_neg(x);
    else if (OP == FR_ADD) r = fe_add(x, ld<P>(b, i));
    else if (OP == FR_SUB) r = fe_sub(x, ld<P>(b, i));
    else if (OP == FR_SQR) r = fe_sqr(x);
    else if (OP == FR_MUL) r = fe_mul(x, ld<P>(b, i));
    else if (OP == FR_MUL_ADD) r = fe_add(fe_mul(x, ld<P>(b, i)), ld<P>(c, i));
    else if (OP == FR_MUL_SUB) r = fe_sub(fe_mul(x, ld<P>(b, i)), ld<P>(c, i));
    else if (OP == FR_SCALE) r = fe_mul(A, x);
    else if (OP == FR_AXPY) r = fe_add(fe_mul(A, x), ld<P>(b, i));
    else if (OP == FR_AXPBY) r = fe_add(fe_mul(A, x), fe_mul(B, ld<P>(b, i)));
    st<P>(out, i, r);
  }
}

// Mode 1 for the single-product operations (mul, sqr, scale, from / to standard form): two elements
// per iteration, both loaded before either product, and the two products in one paired call
// (twice the loads in flight and the products' ILP).
template <class P, int OP>
__global__ void k_fr_map_pair(int n, const uint32_t* a, const uint32_t* b, const uint32_t* ka, uint32_t* out) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  Fe<P> K;
  if (OP == FR_SCALE) K = fe_load<P>(ka);
  if (OP == FR_FROM_STD)
    for (int w = 0; w < P::N; w++) K.v[w] = P::r2(w);
  if (OP == FR_TO_STD) {
    K = fe_zero<P>();
    K.v[0] = 1;
  }
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += 2 * stride) {
    const size_t j = i + stride;
    const bool two = j < (size_t)n;
    const Fe<P> x0 = ld<P>(a, i);
    const Fe<P> x1 = two ? ld<P>(a, j) : x0;
    Fe<P> r0, r1;
    if (OP == FR_MUL) {
      const Fe<P> y0 = ld<P>(b, i);
      const Fe<P> y1 = two ? ld<P>(b, j) : y0;
      fe_mul2(r0, x0, y0, r1, x1, y1);
    } else if (OP == FR_SQR) {
      fe_sqr2(r0, x0, r1, x1);
    } else {
      fe_mul2(r0, x0, K, r1, x1, K);
    }
    st<P>(out, i, r0);
    if (two) st<P>(out, j, r1);
  }
}

template <class P>
__device__ __forceinline__ Fe<P> fe_pow_u32(const Fe<P>& a, uint32_t e) {
  const uint32_t w[1] = {e};
  return fe_pow<P, 1>(a, w);
}

// powers (shift 0): out[i] = A B^i for i < n. mul_by_powers (shift 1): out[i] = src[i] A B^(i-1)
// for 1 <= i < n, out[0] untouched.
template <class P>
__global__ void k_fr_powers(int n, int shift, const uint32_t* src, const uint32_t* ka, const uint32_t* kb,
                            uint32_t* out) {
  const uint32_t T = gridDim.x * blockDim.x;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t first = t + (shift && t == 0 ? T : 0);   // mul_by_powers skips element 0
  if (first >= (uint32_t)n) return;
  const Fe<P> B = fe_load<P>(kb);
  const Fe<P> step = fe_pow_u32(B, T);
  Fe<P> x = fe_mul(fe_load<P>(ka), fe_pow_u32(B, first - shift));
  for (uint32_t i = first; i < (uint32_t)n; i += T) {
    st<P>(out, i, shift ? fe_mul(ld<P>(src, i), x) : x);
    x = fe_mul(x, step);
  }
}

// Batch inversion with one inversion per block: each thread multiplies its strided subset
// (prefix products kept in scratch), the block combines the thread products by two scans, thread 0
// inverts the block's total, and each thread derives the inverse of its own product as
// inv(total) * (product of the threads before it) * (product of the threads after it), then
// runs its backward pass. A zero element makes the total zero and every output zero, as in the
// reference; *zero_flag records it for the operations that need it.
template <class P>
__global__ void __launch_bounds__(256) k_fr_batch_inv_blk(int n, const uint32_t* a, uint32_t* __restrict__ scratch,
                                                          uint32_t* out, int* __restrict__ zero_flag) {
  __shared__ Fe<P> sw[9];
  __shared__ Fe<P> s_inv;
  const size_t T = (size_t)gridDim.x * blockDim.x;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  Fe<P> acc = fe_one<P>();
  size_t last = t;
  for (size_t i = t; i < (size_t)n; i += T) {
    const Fe<P> x = ld<P>(a, i);
    if (fe_is_zero(x)) *zero_flag = 1;
    acc = fe_mul(acc, x);
    st<P>(scratch, i, acc);
    last = i;
  }
  Fe<P> total, total2;
  const Fe<P> before = block_mul_excl_scan<P, false>(acc, sw, total);
  const Fe<P> after = block_mul_excl_scan<P, true>(acc, sw, total2);
  if (threadIdx.x == 0) s_inv = fe_inv_binary(total);
  __syncthreads();
  if (t >= (size_t)n) return;
  Fe<P> inv = fe_mul(fe_mul(s_inv, before), after);   // inverse of this thread's product
  for (size_t i = last;; i -= T) {
    const Fe<P> x = ld<P>(a, i);      // read before out[i] is written (a may alias out)
    st<P>(out, i, i >= t + T ? fe_mul(inv, ld<P>(scratch, i - T)) : inv);
    inv = fe_mul(inv, x);
    if (i < t + T) break;
  }
}


__global__ void k_fr_zero_if(int n, const int* __restrict__ flag, uint32_t* out) {
  if (!*flag) return;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n * 2; i += stride)
    reinterpret_cast<uint4*>(out)[i] = make_uint4(0, 0, 0, 0);
}

// dot product: per-block partial sums, then one block folds them
template <class P>
__global__ void __launch_bounds__(256) k_fr_dot(int n, const uint32_t* a, const uint32_t* b, uint32_t* partial) {
  __shared__ __align__(16) uint32_t sh[256 * 8];
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  Fe<P> acc = fe_zero<P>();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride)
    acc = fe_add(acc, fe_mul(ld<P>(a, i), ld<P>(b, i)));
  fe_store<P>(sh + 8 * threadIdx.x, acc);
  __syncthreads();
  for (int w = 128; w >= 1; w >>= 1) {
    if ((int)threadIdx.x < w)
      fe_store<P>(sh + 8 * threadIdx.x, fe_add(fe_load<P>(sh + 8 * threadIdx.x), fe_load<P>(sh + 8 * (threadIdx.x + w))));
    __syncthreads();
  }
  if (threadIdx.x == 0) fe_store<P>(partial + 8 * blockIdx.x, fe_load<P>(sh));
}

template <class P>
__global__ void __launch_bounds__(256) k_fr_sum(int n, const uint32_t* in, uint32_t* out) {
  __shared__ __align__(16) uint32_t sh[256 * 8];
  Fe<P> acc = fe_zero<P>();
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc = fe_add(acc, ld<P>(in, i));
  fe_store<P>(sh + 8 * threadIdx.x, acc);
  __syncthreads();
  for (int w = 128; w >= 1; w >>= 1) {
    if ((int)threadIdx.x < w)
      fe_store<P>(sh + 8 * threadIdx.x, fe_add(fe_load<P>(sh + 8 * threadIdx.x), fe_load<P>(sh + 8 * (threadIdx.x + w))));
    __syncthreads();
  }
  if (threadIdx.x == 0) fe_store<P>(out, fe_load<P>(sh));
}

// predicates: *flag starts at 1 and is cleared by any element that fails
// which: 0 is_valid (< r), 1 is_zero, 2 is_one (Montgomery one), 3 is_equal
template <class P>
__global__ void k_fr_pred(int n, int which, const uint32_t* a, const uint32_t* b, int* __restrict__ flag) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) {
    const Fe<P> x = ld<P>(a, i);
    bool ok;
    if (which == 0) {
      ok = false;   // x < r, compared from the top word
      bool decided = false;
#pragma unroll
      for (int j = 7; j >= 0; j--) {
        if (!decided && x.v[j] != P::mod(j)) { ok = x.v[j] < P::mod(j); decided = true; }
      }
    } else if (which == 1) {
      ok = fe_is_zero(x);
    } else if (which == 2) {
      ok = fe_eq(x, fe_one<P>());
    } else {
      ok = fe_eq(x, ld<P>(b, i));
    }
    if (!ok) *flag = 0;
  }
}

// sparse A*v: accumulate 32-bit words of coeff[k] * src[col[k]] into 64-bit counters of row[k]
template <class P>
__global__ void k_fr_sparse_acc(int K, int N, int M, const uint64_t* __restrict__ rows, const uint64_t* __restrict__ cols,
                                const uint32_t* __restrict__ coeffs, const uint32_t* __restrict__ src,
                                unsigned long long* __restrict__ acc) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < (size_t)K; k += stride) {
    const int row = (int)rows[k], col = (int)cols[k];
    if (row < 0 || row >= N || col < 0 || col >= M) continue;   // rejected on the host beforehand
    const Fe<P> p = fe_mul(ld<P>(coeffs, k), ld<P>(src, col));
#pragma unroll
    for (int j = 0; j < 8; j++) atomicAdd(acc + (size_t)row * 8 + j, (unsigned long long)p.v[j]);
  }
}

// out[row] = (sum_j acc_j 2^(32 j)) mod r, with cj[j] = 2^(32 j) R^2 mod r (Montgomery factors)
template <class P>
__global__ void k_fr_sparse_fold(int N, const unsigned long long* __restrict__ acc, const uint32_t* __restrict__ cj,
                                 uint32_t* __restrict__ out) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < (size_t)N; r += stride) {
    Fe<P> s = fe_zero<P>();
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const unsigned long long v = acc[r * 8 + j];
      Fe<P> e = fe_zero<P>();
      e.v[0] = (uint32_t)v;
      e.v[1] = (uint32_t)(v >> 32);
      s = fe_add(s, fe_mul(e, fe_load<P>(cj + 8 * j)));
    }
    st<P>(out, r, fe_from_mont(s));
  }
}

// ----------------------------------------------------------------------------- host side
static inline size_t rup(size_t x) { return (x + 255) & ~size_t(255); }

static int grid_for(const Context& cx, size_t n, int per_sm = 8) {
  const size_t g = std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)cx.sm_count * per_sm));
  return (int)g;
}

template <class P>
static zkg_status fr_launch_map(Context& cx, int op, int n, const uint32_t* a, const uint32_t* b, const uint32_t* c,
                                const uint32_t* ka, const uint32_t* kb, uint32_t* out, uint32_t* scratch,
                                uint32_t* scratch2, int* flag, cudaStream_t st) {
  const dim3 blk(256), grid(grid_for(cx, (size_t)n));
  const dim3 gmap(g_fr_map_mode == 2 ? std::max<unsigned>(1u, (unsigned)(((size_t)n + 255) / 256)) : grid.x);
  switch (op) {
#define ZKB_FR_MAP_CASE(OPC)                                                                                \
  case OPC:                                                                                                 \
    if constexpr (OPC == FR_MUL || OPC == FR_SQR || OPC == FR_SCALE || OPC == FR_FROM_STD ||                \
                  OPC == FR_TO_STD)                                                                         \
      if (g_fr_map_mode == 1) return launch("fr_map_pair", k_fr_map_pair<P, OPC>, gmap, blk, 0, st, n, a, b, ka, out); \
    return launch("fr_map", k_fr_map<P, OPC>, gmap, blk, 0, st, n, a, b, c, ka, kb, out);
    ZKB_FR_MAP_CASE(FR_FROM_STD) ZKB_FR_MAP_CASE(FR_TO_STD) ZKB_FR_MAP_CASE(FR_NEG) ZKB_FR_MAP_CASE(FR_ADD)
    ZKB_FR_MAP_CASE(FR_SUB) ZKB_FR_MAP_CASE(FR_SQR) ZKB_FR_MAP_CASE(FR_MUL) ZKB_FR_MAP_CASE(FR_MUL_ADD)
    ZKB_FR_MAP_CASE(FR_MUL_SUB) ZKB_FR_MAP_CASE(FR_SCALE) ZKB_FR_MAP_CASE(FR_AXPY) ZKB_FR_MAP_CASE(FR_AXPBY)
#undef ZKB_FR_MAP_CASE
    case FR_POWERS:
    case FR_MUL_BY_POWERS: {
      const int T = (int)std::max<size_t>(1, std::min<size_t>((size_t)n, (size_t)cx.sm_count * 1024));
      return launch("fr_powers", k_fr_powers<P>, dim3((T + 255) / 256), blk, 0, st, n, op == FR_MUL_BY_POWERS ? 1 : 0,
                    a, ka, kb, out);
    }
    case FR_INV:
    case FR_DIV: {
      // about 32 elements per thread's chain, one inversion (binary extended Euclid) per block of
      // 256 threads, and at most one wave of resident blocks (a second wave would wait for the
      // first one's serial inversions before starting its own)
      static int inv_per_sm[64];   // resident blocks per SM, per device (the context lock is held)
      int& bps = inv_per_sm[cx.device & 63];
      if (bps == 0) {
        int k = 0;
        ZKB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, k_fr_batch_inv_blk<P>, 256, 0));
        bps = std::max(1, k);
      }
      const size_t wave = (size_t)cx.sm_count * bps * 256;
      const size_t T = std::min<size_t>(std::min<size_t>(((size_t)n + 255) & ~size_t(255), wave),
                                        std::max<size_t>(2048, (size_t)n / 32));
      const unsigned g = (unsigned)((T + 255) / 256);
      ZKB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
      uint32_t* inv_out = op == FR_INV ? out : scratch2;
      ZKB_TRY(launch("fr_batch_inv", k_fr_batch_inv_blk<P>, dim3(g), blk, 0, st, n, op == FR_INV ? a : b, scratch,
                     inv_out, flag));
      ZKB_TRY(launch("fr_zero_if", k_fr_zero_if, grid, blk, 0, st, n, (const int*)flag, inv_out));
      if (op == FR_DIV)
        ZKB_TRY(launch("fr_map", k_fr_map<P, FR_MUL>, grid, blk, 0, st, n, a, (const uint32_t*)scratch2, c, ka, kb,
                       out));
      return ZKG_OK;
    }
    default:
      return set_status(ZKG_ERR_ARG, "fr", "unknown operation");
  }
}

static zkg_status fr_check(zkg_curve curve, int op, int n, const void* a, const void* b, const void* c, const void* ka,
                           const void* kb, const void* out) {
  if (curve != ZKG_BN254 && curve != ZKG_BLS12_381) return set_status(ZKG_ERR_ARG, "fr", "unknown curve");
  const int need = fr_inputs(op);
  if (need < 0) return set_status(ZKG_ERR_ARG, "fr", "unknown operation");
  if (n < 0) return set_status(ZKG_ERR_ARG, "fr", "negative length");
  if (n == 0) return ZKG_OK;
  if (!out || ((need & 1) && !a) || ((need & 2) && !b) || ((need & 4) && !c) || ((need & 8) && !ka) ||
      ((need & 16) && !kb))
    return set_status(ZKG_ERR_ARG, "fr", "null pointer");
  return ZKG_OK;
}

// scratch layout: [a b c out] (host path) + [scratch scratch2] + coefficients + flag
template <class P>
static zkg_status fr_map_entry(int op, int n, const uint64_t* a, const uint64_t* b, const uint64_t* c,
                               const uint64_t* ka, const uint64_t* kb, uint64_t* out, bool device) {
  if (n == 0) return set_status(ZKG_OK, nullptr, nullptr);
  const int need = fr_inputs(op);
  if (device && ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(c) |
                  reinterpret_cast<uintptr_t>(out)) & 15))
    return set_status(ZKG_ERR_ARG, "fr", "device buffers must be 16-byte aligned");
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  const size_t vb = (size_t)n * 32;
  const bool inv = op == FR_INV || op == FR_DIV;
  size_t bytes = rup(64) + rup(sizeof(int));
  if (!device) bytes += 4 * rup(vb);
  if (inv) bytes += 2 * rup(vb);
  ZKB_TRY(cx.arena.reserve(bytes));
  cx.arena.reset();
  uint32_t* dk = static_cast<uint32_t*>(cx.arena.take(64));
  int* flag = static_cast<int*>(cx.arena.take(sizeof(int)));
  uint32_t *da = nullptr, *db = nullptr, *dc = nullptr, *dout = nullptr, *s1 = nullptr, *s2 = nullptr;
  if (!device) {
    da = static_cast<uint32_t*>(cx.arena.take(vb));
    db = static_cast<uint32_t*>(cx.arena.take(vb));
    dc = static_cast<uint32_t*>(cx.arena.take(vb));
    dout = static_cast<uint32_t*>(cx.arena.take(vb));
  } else {
    if (!cx.user_stream) ZKB_CUDA(cudaDeviceSynchronize());
    da = (uint32_t*)a; db = (uint32_t*)b; dc = (uint32_t*)c; dout = (uint32_t*)out;
  }
  if (inv) {
    s1 = static_cast<uint32_t*>(cx.arena.take(vb));
    s2 = static_cast<uint32_t*>(cx.arena.take(vb));
  }
  if (!dk || !flag || (!device && !dout) || (inv && !s2)) return set_status(ZKG_ERR_NOMEM, "fr", "arena");
  const cudaStream_t st = cx.compute();
  if (need & 24) {   // coefficients A, B (operations without them upload nothing)
    uint64_t kk[8] = {0};
    if (need & 8) std::memcpy(kk, ka, 32);
    if (need & 16) std::memcpy(kk + 4, kb, 32);
    ZKB_CUDA(cudaMemcpyAsync(dk, kk, 64, cudaMemcpyHostToDevice, st));
  }
  if (!device) {
    if (need & 1) ZKB_TRY(copy_h2d(cx, da, a, vb, st));
    if (need & 2) ZKB_TRY(copy_h2d(cx, db, b, vb, st));
    if (need & 4) ZKB_TRY(copy_h2d(cx, dc, c, vb, st));
  }
  ZKB_CUDA(cudaEventRecord(cx.ev_a, st));
  ZKB_TRY(fr_launch_map<P>(cx, op, n, da, db, dc, dk, dk + 8, dout, s1, s2, flag, st));
  ZKB_CUDA(cudaEventRecord(cx.ev_b, st));
  if (!device) {
    // mul_by_powers leaves element 0 of the target as it was
    const size_t skip = op == FR_MUL_BY_POWERS ? 32 : 0;
    if (vb > skip)
      ZKB_TRY(copy_d2h(cx, reinterpret_cast<char*>(out) + skip, reinterpret_cast<char*>(dout) + skip, vb - skip,
                       st));
  }
  ZKB_CUDA(cudaStreamSynchronize(st));
  ZKB_CUDA(cudaEventElapsedTime(&cx.last_kernel_ms, cx.ev_a, cx.ev_b));
  return set_status(ZKG_OK, nullptr, nullptr);
}

template <class P>
static zkg_status fr_dot_entry(int n, const uint64_t* a, const uint64_t* b, uint64_t* out, bool device) {
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  const size_t vb = (size_t)n * 32;
  const int grid = grid_for(cx, (size_t)n, 4);
  size_t bytes = rup((size_t)grid * 32) + rup(32) + (device ? 0 : 2 * rup(vb));
  ZKB_TRY(cx.arena.reserve(bytes));
  cx.arena.reset();
  uint32_t* part = static_cast<uint32_t*>(cx.arena.take((size_t)grid * 32));
  uint32_t* res = static_cast<uint32_t*>(cx.arena.take(32));
  const uint32_t *da = (const uint32_t*)a, *db = (const uint32_t*)b;
  const cudaStream_t st = cx.compute();
  if (!device) {
    uint32_t* ha = static_cast<uint32_t*>(cx.arena.take(vb));
    uint32_t* hb = static_cast<uint32_t*>(cx.arena.take(vb));
    if (!ha || !hb) return set_status(ZKG_ERR_NOMEM, "fr_dot", "arena");
    if (n) {
      ZKB_TRY(copy_h2d(cx, ha, a, vb, st));
      ZKB_TRY(copy_h2d(cx, hb, b, vb, st));
    }
    da = ha;
    db = hb;
  } else if (!cx.user_stream) {
    ZKB_CUDA(cudaDeviceSynchronize());
  }
  if (!part || !res) return set_status(ZKG_ERR_NOMEM, "fr_dot", "arena");
  ZKB_TRY(launch("fr_dot", k_fr_dot<P>, dim3(grid), dim3(256), 0, st, n, da, db, part));
  ZKB_TRY(launch("fr_sum", k_fr_sum<P>, dim3(1), dim3(256), 0, st, grid, (const uint32_t*)part, res));
  ZKB_CUDA(cudaMemcpyAsync(out, res, 32, cudaMemcpyDeviceToHost, st));
  ZKB_CUDA(cudaStreamSynchronize(st));
  return set_status(ZKG_OK, nullptr, nullptr);
}

template <class P>
static zkg_status fr_pred_entry(int which, int n, const uint64_t* a, const uint64_t* b, int* result, bool device) {
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  const size_t vb = (size_t)n * 32;
  size_t bytes = rup(sizeof(int)) + (device ? 0 : 2 * rup(vb));
  ZKB_TRY(cx.arena.reserve(bytes));
  cx.arena.reset();
  int* flag = static_cast<int*>(cx.arena.take(sizeof(int)));
  const uint32_t *da = (const uint32_t*)a, *db = (const uint32_t*)b;
  const cudaStream_t st = cx.compute();
  if (!device) {
    uint32_t* ha = static_cast<uint32_t*>(cx.arena.take(vb));
    uint32_t* hb = static_cast<uint32_t*>(cx.arena.take(vb));
    if (!ha || !hb) return set_status(ZKG_ERR_NOMEM, "fr_pred", "arena");
    ZKB_TRY(copy_h2d(cx, ha, a, vb, st));
    if (which == 3) ZKB_TRY(copy_h2d(cx, hb, b, vb, st));
    da = ha;
    db = hb;
  } else if (!cx.user_stream) {
    ZKB_CUDA(cudaDeviceSynchronize());
  }
  const int one = 1;
  ZKB_CUDA(cudaMemcpyAsync(flag, &one, sizeof(int), cudaMemcpyHostToDevice, st));
  ZKB_TRY(launch("fr_pred", k_fr_pred<P>, dim3(grid_for(cx, (size_t)n)), dim3(256), 0, st, n, which, da, db, flag));
  int h = 0;
  ZKB_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  ZKB_CUDA(cudaStreamSynchronize(st));
  *result = h;
  return set_status(ZKG_OK, nullptr, nullptr);
}

template <class P>
static zkg_status fr_sparse_entry(const host::Field<4>& Fr, int N, int K, const uint64_t* rows, const uint64_t* cols,
                                  const uint64_t* coeffs, const uint64_t* src, int M, uint64_t* tgt, bool device) {
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  const size_t nb = (size_t)N * 32, kb = (size_t)K * 32, mb = (size_t)M * 32, ib = (size_t)K * 8;
  size_t bytes = rup((size_t)N * 64) + rup(256) + (device ? 0 : rup(nb) + rup(kb) + rup(mb) + 2 * rup(ib));
  ZKB_TRY(cx.arena.reserve(bytes));
  cx.arena.reset();
  unsigned long long* acc = static_cast<unsigned long long*>(cx.arena.take((size_t)N * 64));
  uint32_t* dcj = static_cast<uint32_t*>(cx.arena.take(256));
  const cudaStream_t st = cx.compute();
  const uint64_t *drows = rows, *dcols = cols;
  const uint32_t *dco = (const uint32_t*)coeffs, *dsrc = (const uint32_t*)src;
  uint32_t* dout = (uint32_t*)tgt;
  if (!device) {
    uint64_t* r = static_cast<uint64_t*>(cx.arena.take(ib));
    uint64_t* c = static_cast<uint64_t*>(cx.arena.take(ib));
    uint32_t* co = static_cast<uint32_t*>(cx.arena.take(kb));
    uint32_t* s = static_cast<uint32_t*>(cx.arena.take(mb));
    dout = static_cast<uint32_t*>(cx.arena.take(nb));
    if (!r || !c || !co || !s || !dout) return set_status(ZKG_ERR_NOMEM, "fr_sparse", "arena");
    if (K) {
      ZKB_CUDA(cudaMemcpyAsync(r, rows, ib, cudaMemcpyHostToDevice, st));
      ZKB_CUDA(cudaMemcpyAsync(c, cols, ib, cudaMemcpyHostToDevice, st));
      ZKB_CUDA(cudaMemcpyAsync(co, coeffs, kb, cudaMemcpyHostToDevice, st));
    }
    if (M) ZKB_TRY(copy_h2d(cx, s, src, mb, st));
    drows = r; dcols = c; dco = co; dsrc = s;
  } else if (!cx.user_stream) {
    ZKB_CUDA(cudaDeviceSynchronize());
  }
  if (!acc || !dcj) return set_status(ZKG_ERR_NOMEM, "fr_sparse", "arena");
  // cj = 2^(32 j) * R^2 mod r
  uint64_t cj[32];
  host::El<4> f;
  std::memcpy(f.v, Fr.r2, 32);
  host::El<4> two32 = host::zero<4>();
  two32.v[0] = (uint64_t)1 << 32;
  const host::El<4> m32 = host::from_std(Fr, two32);   // Montgomery form of 2^32
  for (int j = 0; j < 8; j++) {
    std::memcpy(cj + 4 * j, f.v, 32);
    f = host::mul(Fr, f, m32);
  }
  ZKB_CUDA(cudaMemcpyAsync(dcj, cj, 256, cudaMemcpyHostToDevice, st));
  ZKB_CUDA(cudaMemsetAsync(acc, 0, (size_t)N * 64, st));
  if (K)
    ZKB_TRY(launch("fr_sparse_acc", k_fr_sparse_acc<P>, dim3(grid_for(cx, (size_t)K)), dim3(256), 0, st, K, N, M, drows,
                   dcols, dco, dsrc, acc));
  ZKB_TRY(launch("fr_sparse_fold", k_fr_sparse_fold<P>, dim3(grid_for(cx, (size_t)N)), dim3(256), 0, st, N,
                 (const unsigned long long*)acc, (const uint32_t*)dcj, dout));
  if (!device) ZKB_TRY(copy_d2h(cx, tgt, dout, nb, st));
  ZKB_CUDA(cudaStreamSynchronize(st));
  return set_status(ZKG_OK, nullptr, nullptr);
}

}  // namespace zkb

using namespace zkb;

extern "C" zkg_status zkg_fr_map(zkg_curve curve, int op, int n, const uint64_t* a, const uint64_t* b,
                                 const uint64_t* c, const uint64_t* coeff_a, const uint64_t* coeff_b, uint64_t* out) {
  ZKB_TRY(fr_check(curve, op, n, a, b, c, coeff_a, coeff_b, out));
  if (curve == ZKG_BN254) return g_fr_dpf ? fr_map_entry<BnFrE>(op, n, a, b, c, coeff_a, coeff_b, out, false) : fr_map_entry<BnFr>(op, n, a, b, c, coeff_a, coeff_b, out, false);
  return g_fr_dpf ? fr_map_entry<BlsFrE>(op, n, a, b, c, coeff_a, coeff_b, out, false) : fr_map_entry<BlsFr>(op, n, a, b, c, coeff_a, coeff_b, out, false);
}

extern "C" zkg_status zkg_fr_map_device(zkg_curve curve, int op, int n, const uint64_t* d_a, const uint64_t* d_b,
                                        const uint64_t* d_c, const uint64_t* coeff_a, const uint64_t* coeff_b,
                                        uint64_t* d_out) {
  ZKB_TRY(fr_check(curve, op, n, d_a, d_b, d_c, coeff_a, coeff_b, d_out));
  if (curve == ZKG_BN254) return g_fr_dpf ? fr_map_entry<BnFrE>(op, n, d_a, d_b, d_c, coeff_a, coeff_b, d_out, true) : fr_map_entry<BnFr>(op, n, d_a, d_b, d_c, coeff_a, coeff_b, d_out, true);
  return g_fr_dpf ? fr_map_entry<BlsFrE>(op, n, d_a, d_b, d_c, coeff_a, coeff_b, d_out, true) : fr_map_entry<BlsFr>(op, n, d_a, d_b, d_c, coeff_a, coeff_b, d_out, true);
}

static zkg_status fr_dot_any(zkg_curve curve, int n, const uint64_t* a, const uint64_t* b, uint64_t* out, bool device) {
  if (curve != ZKG_BN254 && curve != ZKG_BLS12_381) return set_status(ZKG_ERR_ARG, "fr_dot", "unknown curve");
  if (n < 0 || !out || (n > 0 && (!a || !b))) return set_status(ZKG_ERR_ARG, "fr_dot", "bad arguments");
  if (device && ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15))
    return set_status(ZKG_ERR_ARG, "fr_dot", "device buffers must be 16-byte aligned");
  if (curve == ZKG_BN254) return g_fr_dpf ? fr_dot_entry<BnFrE>(n, a, b, out, device) : fr_dot_entry<BnFr>(n, a, b, out, device);
  return g_fr_dpf ? fr_dot_entry<BlsFrE>(n, a, b, out, device) : fr_dot_entry<BlsFr>(n, a, b, out, device);
}
extern "C" zkg_status zkg_fr_dot(zkg_curve curve, int n, const uint64_t* a, const uint64_t* b, uint64_t* out) {
  return fr_dot_any(curve, n, a, b, out, false);
}
extern "C" zkg_status zkg_fr_dot_device(zkg_curve curve, int n, const uint64_t* d_a, const uint64_t* d_b, uint64_t* out) {
  return fr_dot_any(curve, n, d_a, d_b, out, true);
}

static zkg_status fr_pred_any(zkg_curve curve, int which, int n, const uint64_t* a, const uint64_t* b, int* result,
                              bool device) {
  if (curve != ZKG_BN254 && curve != ZKG_BLS12_381) return set_status(ZKG_ERR_ARG, "fr_pred", "unknown curve");
  if (which < 0 || which > 3 || n < 0 || !result || (n > 0 && (!a || (which == 3 && !b))))
    return set_status(ZKG_ERR_ARG, "fr_pred", "bad arguments");
  if (device && ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15))
    return set_status(ZKG_ERR_ARG, "fr_pred", "device buffers must be 16-byte aligned");
  if (n == 0) {
    *result = 1;
    return set_status(ZKG_OK, nullptr, nullptr);
  }
  if (curve == ZKG_BN254) return g_fr_dpf ? fr_pred_entry<BnFrE>(which, n, a, b, result, device) : fr_pred_entry<BnFr>(which, n, a, b, result, device);
  return g_fr_dpf ? fr_pred_entry<BlsFrE>(which, n, a, b, result, device) : fr_pred_entry<BlsFr>(which, n, a, b, result, device);
}
extern "C" zkg_status zkg_fr_predicate(zkg_curve curve, int which, int n, const uint64_t* a, const uint64_t* b,
                                       int* result) {
  return fr_pred_any(curve, which, n, a, b, result, false);
}
extern "C" zkg_status zkg_fr_predicate_device(zkg_curve curve, int which, int n, const uint64_t* d_a,
                                              const uint64_t* d_b, int* result) {
  return fr_pred_any(curve, which, n, d_a, d_b, result, true);
}

static zkg_status fr_sparse_any(zkg_curve curve, int N, int K, const uint64_t* rows, const uint64_t* cols,
                                const uint64_t* coeffs, const uint64_t* src, int M, uint64_t* tgt, bool device) {
  if (curve != ZKG_BN254 && curve != ZKG_BLS12_381) return set_status(ZKG_ERR_ARG, "fr_sparse", "unknown curve");
  if (N < 0 || K < 0 || M < 0 || (N > 0 && !tgt) || (K > 0 && (!rows || !cols || !coeffs || !src)))
    return set_status(ZKG_ERR_ARG, "fr_sparse", "bad arguments");
  if (N == 0) return set_status(ZKG_OK, nullptr, nullptr);
  if (curve == ZKG_BN254) return g_fr_dpf ? fr_sparse_entry<BnFrE>(host::BN_FR, N, K, rows, cols, coeffs, src, M, tgt, device) : fr_sparse_entry<BnFr>(host::BN_FR, N, K, rows, cols, coeffs, src, M, tgt, device);
  return g_fr_dpf ? fr_sparse_entry<BlsFrE>(host::BLS_FR, N, K, rows, cols, coeffs, src, M, tgt, device) : fr_sparse_entry<BlsFr>(host::BLS_FR, N, K, rows, cols, coeffs, src, M, tgt, device);
}
extern "C" zkg_status zkg_fr_sparse_matrix_mul(zkg_curve curve, int N, int K, const uint64_t* rows,
                                               const uint64_t* cols, const uint64_t* coeffs, const uint64_t* src,
                                               uint64_t* tgt) {
  // the source length is the largest column index + 1; an index outside the matrix is an error
  int M = 0;
  for (int k = 0; k < K; k++) {
    if (!rows || !cols) break;
    const long long r = (long long)(int)rows[k], c = (long long)(int)cols[k];
    if (r < 0 || r >= N || c < 0 || c >= 0x7fffffff) return set_status(ZKG_ERR_ARG, "fr_sparse", "index outside the matrix");
    if (c >= M) M = (int)c + 1;
  }
  return fr_sparse_any(curve, N, K, rows, cols, coeffs, src, M, tgt, false);
}
extern "C" zkg_status zkg_fr_sparse_matrix_mul_device(zkg_curve curve, int N, int K, const uint64_t* d_rows,
                                                      const uint64_t* d_cols, const uint64_t* d_coeffs,
                                                      const uint64_t* d_src, int M, uint64_t* d_tgt) {
  return fr_sparse_any(curve, N, K, d_rows, d_cols, d_coeffs, d_src, M, d_tgt, true);
}
