// NTT planning and entry points (kernels: zkb_ntt_kernels.cuh).
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
// 32-byte elements. The tile lives in shared memory; each thread runs 3 butterfly stages at a
// time on 8 elements held in registers.
#include <algorithm>
#include <cstring>
#include <cstdlib>
#include <vector>

#include "zkb_dpf.cuh"
#include "zkb_field.cuh"
#include "zkb_host_ec.h"
#include "zkb_ntt.h"
#include "zkb_runtime.h"

namespace zkb {

// --------------------------------------------------------------------------- planning

static int g_ntt_kmax = 8;
// NTT passes with FP64-pipe products (tables in radix R' = 2^260, zkb_dpf.cuh); ZKB_NTT_DPF=0
// keeps every table in the reference's radix and the products on the integer pipes
static int g_ntt_dpf = [] {
  const char* v = std::getenv("ZKB_NTT_DPF");
  return v ? std::atoi(v) : 1;
}();
static bool g_ntt_kmax_set = false;       // an explicit zkg_set_ntt_kmax overrides tuning
static int g_ntt_tuned[2][NTT_MMAX + 1] = {{0}};    // tuned largest pass per curve and m (0 = untuned)

static std::once_flag g_ntt_tune_once[2];

static int effective_kmax(int curve, int m) {
  std::call_once(g_ntt_tune_once[curve], [curve] {   // persisted tuning (ZKG_TUNE_CACHE), once
    const int sms = device_sm_count();
    for (int mm = 0; mm <= NTT_MMAX; mm++) {
      int k = 0;
      if (tune_cache_get("ntt", curve, mm, sms, &k, 1) && k >= 1 && k <= NTT_KMAX) g_ntt_tuned[curve][mm] = k;
    }
  });
  if (!g_ntt_kmax_set && m >= 0 && m <= NTT_MMAX && g_ntt_tuned[curve][m] > 0) return g_ntt_tuned[curve][m];
  return g_ntt_kmax;
}

static std::vector<NttPass> ntt_schedule(int m, int kmax) {
  std::vector<NttPass> ps;
  if (m == 0) return ps;
  const int np = (m + kmax - 1) / kmax;
  int s = 0;
  for (int p = 0; p < np; p++) {
    const int rem = m - s, left = np - p;
    const int k = (rem + left - 1) / left;   // larger passes first
    NttPass q;
    q.k = k;
    q.s = s;
    q.Mp = m - s - k;
    ps.push_back(q);
    s += k;
  }
  return ps;
}

template <int NL>
static host::El<NL> el_from_u64(const uint64_t* p) {
  host::El<NL> r;
  std::memcpy(r.v, p, sizeof(r.v));
  return r;
}

static zkg_status upload(uint32_t** dst, const std::vector<host::El<4>>& v) {
  ZKB_CUDA(cudaMalloc(dst, v.size() * 32));
  ZKB_CUDA(cudaMemcpy(*dst, v.data(), v.size() * 32, cudaMemcpyHostToDevice));
  return ZKG_OK;
}

template <class P>
static zkg_status build_plan_uncached(const host::Field<4>& F, int curve, int m, const uint64_t* gen, int inverse,
                                      int kmax, cudaStream_t stream, NttPlan** out) {
  NttPlan* pl = new NttPlan();
  pl->curve = curve;
  pl->m = m;
  pl->inverse = inverse;
  pl->kmax = kmax;
  std::memcpy(pl->gen, gen, 32);
  pl->passes = ntt_schedule(m, kmax);
  pl->dpf = g_ntt_dpf != 0;
  // tables in radix R' when the passes multiply on the FP64 pipe: x R -> x R R' / R
  using PD = typename DpfOf<P>::type;
  host::El<4> rp = host::zero<4>();   // R' mod r as a standard integer
  for (int w = 0; w < 8; w++) rp.v[w >> 1] |= (uint64_t)PD::one(w) << (32 * (w & 1));
  auto conv = [&](std::vector<host::El<4>>& v) {
    if (pl->dpf)
      for (auto& e : v) e = host::mul(F, e, rp);
  };
  host::El<4> g = el_from_u64<4>(gen);
  host::El<4> h = inverse ? host::inv(F, g) : g;   // network generator
  // small-network tables: w_k = h^(2^(m-k)), powers 0 .. 2^(k-1)-1
  for (const NttPass& q : pl->passes) {
    if (pl->d_om[q.k]) continue;
    host::El<4> w = h;
    for (int i = 0; i < m - q.k; i++) w = host::mul(F, w, w);
    std::vector<host::El<4>> tab((size_t)1 << (q.k - 1));
    host::El<4> x = host::one(F);
    for (auto& e : tab) { e = x; x = host::mul(F, x, w); }
    conv(tab);
    zkg_status st = upload(&pl->d_om[q.k], tab);
    if (st != ZKG_OK) { delete pl; return st; }
  }
  // (1/2)^m, the inverse's final scale (bn128_poly_mont.c:565-622 halves at every level)
  host::El<4> scale = host::one(F);
  if (inverse) {
    host::El<4> two = host::zero<4>();
    two.v[0] = 2;
    scale = host::pow_u64(F, host::inv(F, host::from_std(F, two)), (uint64_t)m);
  }
  if (pl->passes.size() >= 2) {
    const uint32_t N = 1u << m;
    const int a = (m + 1) / 2;
    std::vector<host::El<4>> A((size_t)1 << a), Bt((size_t)1 << (m - a));
    host::El<4> x = host::one(F);
    for (auto& e : A) { e = x; x = host::mul(F, x, h); }
    const host::El<4> step = x;   // h^(2^a)
    x = host::one(F);
    for (auto& e : Bt) { e = x; x = host::mul(F, x, step); }
    // the inverse's last pass multiplies its inputs by the twiddles anyway: a copy of the table
    // scaled by (1/2)^m (A[j] (1/2)^m times Bt[i]) folds the final scale into that product
    std::vector<host::El<4>> As;
    if (inverse)
      for (const auto& e : A) As.push_back(host::mul(F, e, scale));
    conv(A);
    conv(Bt);
    conv(As);
    uint32_t *dA = nullptr, *dB = nullptr, *dAs = nullptr;
    zkg_status st = upload(&dA, A);
    if (st == ZKG_OK) st = upload(&dB, Bt);
    if (st == ZKG_OK && inverse) st = upload(&dAs, As);
    if (st == ZKG_OK && (cudaMalloc(&pl->d_tw, (size_t)N * 32) != cudaSuccess ||
                         (inverse && cudaMalloc(&pl->d_tw_last, (size_t)N * 32) != cudaSuccess))) {
      (void)cudaGetLastError();
      st = set_status(ZKG_ERR_NOMEM, "ntt plan", "twiddle table");
    }
    if (st == ZKG_OK)
      st = pl->dpf ? ntt_launch_table<PD>(pl->d_tw, dA, dB, a, N, stream)
                   : ntt_launch_table<P>(pl->d_tw, dA, dB, a, N, stream);
    if (st == ZKG_OK && inverse)
      st = pl->dpf ? ntt_launch_table<PD>(pl->d_tw_last, dAs, dB, a, N, stream)
                   : ntt_launch_table<P>(pl->d_tw_last, dAs, dB, a, N, stream);
    if (st == ZKG_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = set_status(ZKG_ERR_CUDA, "ntt plan", "sync");
    if (dA) cudaFree(dA);
    if (dB) cudaFree(dB);
    if (dAs) cudaFree(dAs);
    if (st != ZKG_OK) { delete pl; return st; }
    pl->bytes += (size_t)N * 32 * (inverse ? 2 : 1);
  }
  if (inverse) {
    std::vector<host::El<4>> sc(1, scale);
    conv(sc);
    zkg_status st = upload(&pl->d_scale, sc);
    if (st != ZKG_OK) { delete pl; return st; }
  }
  *out = pl;
  return ZKG_OK;
}

template <class P>
static zkg_status build_plan(Context& cx, const host::Field<4>& F, int curve, int m, const uint64_t* gen, int inverse,
                             NttPlan** out) {
  for (NttPlan* p : cx.ntt_plans)
    if (p->curve == curve && p->m == m && p->inverse == inverse && p->kmax == effective_kmax(curve, m) &&
        p->dpf == (g_ntt_dpf != 0) && std::memcmp(p->gen, gen, 32) == 0) {
      *out = p;
      return ZKG_OK;
    }
  NttPlan* pl = nullptr;
  ZKB_TRY(build_plan_uncached<P>(F, curve, m, gen, inverse, effective_kmax(curve, m), cx.stream, &pl));
  // bounded cache: drop the oldest plans beyond 64 plans or 4 GiB of tables (a 2^24 forward and
  // inverse pair holds 1.5 GiB)
  cx.ntt_plans.push_back(pl);
  auto table_bytes = [&] {
    size_t b = 0;
    for (NttPlan* p : cx.ntt_plans) b += p->bytes;
    return b;
  };
  while (cx.ntt_plans.size() > 1 && (cx.ntt_plans.size() > 64 || table_bytes() > ((size_t)4 << 30))) {
    delete cx.ntt_plans.front();
    cx.ntt_plans.erase(cx.ntt_plans.begin());
  }
  *out = pl;
  return ZKG_OK;
}

// Runs the plan d_src -> d_tgt; scratch (N elements) needed when there are >= 2 passes.
template <class P>
static zkg_status ntt_run(Context& cx, const NttPlan& pl, const uint32_t* d_src, uint32_t* d_tgt, uint32_t* scratch,
                          cudaStream_t st) {
  const int np = (int)pl.passes.size();
  const size_t N = (size_t)1 << pl.m;
  if (np == 0) {   // m = 0: copy (bn128_poly_mont.c:420-423)
    ZKB_CUDA(cudaMemcpyAsync(d_tgt, d_src, N * 32, cudaMemcpyDeviceToDevice, st));
    return ZKG_OK;
  }
  const uint32_t* in = d_src;
  for (int i = 0; i < np; i++) {
    // the i-th executed pass writes tgt when (np-1-i) is even, scratch otherwise
    uint32_t* out = ((np - 1 - i) % 2 == 0) ? d_tgt : scratch;
    const NttPass& q = pl.inverse ? pl.passes[np - 1 - i] : pl.passes[i];
    if (pl.dpf) ZKB_TRY(ntt_launch_pass<typename DpfOf<P>::type>(pl, q, in, out, pl.inverse && i == np - 1, st));
    else ZKB_TRY(ntt_launch_pass<P>(pl, q, in, out, pl.inverse && i == np - 1, st));
    in = out;
  }
  return ZKG_OK;
}

template <class P>
static zkg_status ntt_entry(const host::Field<4>& F, int curve, int m, const uint64_t* gen, const uint64_t* src,
                            uint64_t* tgt, int inverse, bool device_ptrs) {
  NvtxRange nvtx("zkb.ntt");
  if (m < 0 || m > NTT_MMAX) return set_status(ZKG_ERR_ARG, "ntt", "m out of range [0, 30]");
  if (!gen || !src || !tgt) return set_status(ZKG_ERR_ARG, "ntt", "null pointer");
  if (src == tgt) return set_status(ZKG_ERR_ARG, "ntt", "src and tgt must not alias");
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  NttPlan* pl = nullptr;
  ZKB_TRY(build_plan<P>(cx, F, curve, m, gen, inverse, &pl));
  const size_t N = (size_t)1 << m, bytes = N * 32, rb = (bytes + 255) & ~size_t(255);
  const bool need_scratch = pl->passes.size() >= 2;
  if (device_ptrs) {
    ZKB_TRY(cx.arena.reserve(need_scratch ? rb : 256));
    cx.arena.reset();
    uint32_t* scratch = static_cast<uint32_t*>(cx.arena.take(need_scratch ? bytes : 32));
    const cudaStream_t st = cx.compute();
    if (!cx.user_stream) ZKB_CUDA(cudaDeviceSynchronize());   // inputs may come from any stream
    ZKB_CUDA(cudaEventRecord(cx.ev_a, st));
    ZKB_TRY(ntt_run<P>(cx, *pl, reinterpret_cast<const uint32_t*>(src), reinterpret_cast<uint32_t*>(tgt), scratch,
                       st));
    ZKB_CUDA(cudaEventRecord(cx.ev_b, st));
    ZKB_CUDA(cudaStreamSynchronize(st));
  } else {
    ZKB_TRY(cx.arena.reserve(3 * rb));
    cx.arena.reset();
    uint32_t* d_src = static_cast<uint32_t*>(cx.arena.take(bytes));
    uint32_t* d_tgt = static_cast<uint32_t*>(cx.arena.take(bytes));
    uint32_t* scratch = static_cast<uint32_t*>(cx.arena.take(bytes));
    const cudaStream_t st = cx.compute();
    ZKB_TRY(copy_h2d(cx, d_src, src, bytes, st));
    ZKB_CUDA(cudaEventRecord(cx.ev_a, st));
    ZKB_TRY(ntt_run<P>(cx, *pl, d_src, d_tgt, scratch, st));
    ZKB_CUDA(cudaEventRecord(cx.ev_b, st));
    ZKB_TRY(copy_d2h(cx, tgt, d_tgt, bytes, st));
  }
  ZKB_CUDA(cudaEventElapsedTime(&cx.last_kernel_ms, cx.ev_a, cx.ev_b));
  return set_status(ZKG_OK, nullptr, nullptr);
}

// ------------------------------------------------------------- shifted / asymmetric NTT
// out[i] = in[i] * eta^i with eta^i = A[i mod 2^a] * Bt[i >> a]
template <class P>
__global__ void k_ntt_scale_pow(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t N,
                                const uint32_t* __restrict__ A, const uint32_t* __restrict__ Bt, int a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const Fe<P> pw = fe_mul(fe_load_nc<P>(A + (size_t)(i & ((1u << a) - 1)) * 8), fe_load_nc<P>(Bt + (size_t)(i >> a) * 8));
  fe_store<P>(out + (size_t)i * 8, fe_mul(fe_load_nc<P>(in + (size_t)i * 8), pw));
}

// out[i K + k] = in[i]
__global__ void k_ntt_interleave(const uint4* __restrict__ in, uint4* __restrict__ out, uint32_t Ns, uint32_t K,
                                 uint32_t k) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Ns) return;
  out[((size_t)i * K + k) * 2] = in[(size_t)i * 2];
  out[((size_t)i * K + k) * 2 + 1] = in[(size_t)i * 2 + 1];
}

// Powers eta^j (j < 2^a) and eta^(j 2^a) (j < 2^(m-a)) for the scaling kernel.
static void pow_tables(const host::Field<4>& F, const host::El<4>& eta, int m, int a, std::vector<host::El<4>>& A,
                       std::vector<host::El<4>>& Bt) {
  A.assign((size_t)1 << a, host::El<4>());
  Bt.assign((size_t)1 << (m - a), host::El<4>());
  host::El<4> x = host::one(F);
  for (auto& e : A) { e = x; x = host::mul(F, x, eta); }
  const host::El<4> step = x;
  x = host::one(F);
  for (auto& e : Bt) { e = x; x = host::mul(F, x, step); }
}

// Shifted (coset) NTT on host buffers: forward = NTT of src[i] eta^i
// (bn128_poly_mont.c:477-488); inverse = inverse NTT, then output i times eta^i (:626-641).
template <class P>
static zkg_status ntt_shifted_entry(const host::Field<4>& F, int curve, const uint64_t* eta, int m,
                                   const uint64_t* gen, const uint64_t* src, uint64_t* tgt, int inverse) {
  if (m < 0 || m > NTT_MMAX) return set_status(ZKG_ERR_ARG, "ntt_shifted", "m out of range [0, 30]");
  if (!eta || !gen || !src || !tgt) return set_status(ZKG_ERR_ARG, "ntt_shifted", "null pointer");
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  NttPlan* pl = nullptr;
  ZKB_TRY(build_plan<P>(cx, F, curve, m, gen, inverse, &pl));
  const size_t N = (size_t)1 << m, bytes = N * 32, rb = (bytes + 255) & ~size_t(255);
  const int a = (m + 1) / 2;
  std::vector<host::El<4>> A, Bt;
  host::El<4> e;
  std::memcpy(e.v, eta, 32);
  pow_tables(F, e, m, a, A, Bt);
  const size_t tb = ((A.size() + Bt.size()) * 32 + 511) & ~size_t(255);
  ZKB_TRY(cx.arena.reserve(4 * rb + tb));
  cx.arena.reset();
  uint32_t* d_a = static_cast<uint32_t*>(cx.arena.take(bytes));
  uint32_t* d_b = static_cast<uint32_t*>(cx.arena.take(bytes));
  uint32_t* d_c = static_cast<uint32_t*>(cx.arena.take(bytes));
  uint32_t* scratch = static_cast<uint32_t*>(cx.arena.take(bytes));
  uint32_t* dA = static_cast<uint32_t*>(cx.arena.take(A.size() * 32));
  uint32_t* dB = static_cast<uint32_t*>(cx.arena.take(Bt.size() * 32));
  const cudaStream_t st = cx.compute();
  ZKB_CUDA(cudaMemcpyAsync(dA, A.data(), A.size() * 32, cudaMemcpyHostToDevice, st));
  ZKB_CUDA(cudaMemcpyAsync(dB, Bt.data(), Bt.size() * 32, cudaMemcpyHostToDevice, st));
  ZKB_TRY(copy_h2d(cx, d_a, src, bytes, st));
  ZKB_CUDA(cudaEventRecord(cx.ev_a, st));
  const dim3 g((uint32_t)((N + 255) / 256));
  if (!inverse) {
    ZKB_TRY(launch("ntt_scale_pow", k_ntt_scale_pow<P>, g, dim3(256), 0, st, (const uint32_t*)d_a, d_b, (uint32_t)N,
                   (const uint32_t*)dA, (const uint32_t*)dB, a));
    ZKB_TRY(ntt_run<P>(cx, *pl, d_b, d_c, scratch, st));
  } else {
    ZKB_TRY(ntt_run<P>(cx, *pl, d_a, d_b, scratch, st));
    ZKB_TRY(launch("ntt_scale_pow", k_ntt_scale_pow<P>, g, dim3(256), 0, st, (const uint32_t*)d_b, d_c, (uint32_t)N,
                   (const uint32_t*)dA, (const uint32_t*)dB, a));
  }
  ZKB_CUDA(cudaEventRecord(cx.ev_b, st));
  ZKB_TRY(copy_d2h(cx, tgt, d_c, bytes, st));
  ZKB_CUDA(cudaEventElapsedTime(&cx.last_kernel_ms, cx.ev_a, cx.ev_b));
  return set_status(ZKG_OK, nullptr, nullptr);
}

// Asymmetric NTT (bn128_poly_mont.c:492-555): for k < K = 2^(m_tgt - m_src), the forward NTT
// (generator gen_src) of src[i] gen_tgt^(k i), written to tgt[i K + k].
template <class P>
static zkg_status ntt_asym_entry(const host::Field<4>& F, int curve, int m_src, int m_tgt, const uint64_t* gen_src,
                                 const uint64_t* gen_tgt, const uint64_t* src, uint64_t* tgt) {
  if (m_src < 0 || m_tgt < m_src || m_tgt > NTT_MMAX)
    return set_status(ZKG_ERR_ARG, "ntt_asymmetric", "need 0 <= m_src <= m_tgt <= 30");
  if (!gen_src || !gen_tgt || !src || !tgt) return set_status(ZKG_ERR_ARG, "ntt_asymmetric", "null pointer");
  Context* cxp = nullptr;
  ZKB_TRY(get_context(&cxp));
  Context& cx = *cxp;
  std::lock_guard<std::mutex> lk(cx.mu);
  NttPlan* pl = nullptr;
  ZKB_TRY(build_plan<P>(cx, F, curve, m_src, gen_src, 0, &pl));
  const size_t Ns = (size_t)1 << m_src, K = (size_t)1 << (m_tgt - m_src), bs = Ns * 32;
  const size_t rbs = (bs + 255) & ~size_t(255), bt = Ns * K * 32, rbt = (bt + 255) & ~size_t(255);
  const int a = (m_src + 1) / 2;
  const size_t tb = ((((size_t)1 << a) + ((size_t)1 << (m_src - a))) * 32 + 511) & ~size_t(255);
  ZKB_TRY(cx.arena.reserve(4 * rbs + rbt + tb));
  cx.arena.reset();
  uint32_t* d_src = static_cast<uint32_t*>(cx.arena.take(bs));
  uint32_t* d_sh = static_cast<uint32_t*>(cx.arena.take(bs));
  uint32_t* d_out = static_cast<uint32_t*>(cx.arena.take(bs));
  uint32_t* scratch = static_cast<uint32_t*>(cx.arena.take(bs));
  uint32_t* d_tgt = static_cast<uint32_t*>(cx.arena.take(bt));
  uint32_t* dA = static_cast<uint32_t*>(cx.arena.take(((size_t)32) << a));
  uint32_t* dB = static_cast<uint32_t*>(cx.arena.take(((size_t)32) << (m_src - a)));
  const cudaStream_t st = cx.compute();
  ZKB_TRY(copy_h2d(cx, d_src, src, bs, st));
  ZKB_CUDA(cudaEventRecord(cx.ev_a, st));
  host::El<4> gt, eta = host::one(F);
  std::memcpy(gt.v, gen_tgt, 32);
  std::vector<host::El<4>> A, Bt;
  const dim3 g((uint32_t)((Ns + 255) / 256));
  for (size_t k = 0; k < K; k++) {
    if (k) eta = host::mul(F, eta, gt);
    pow_tables(F, eta, m_src, a, A, Bt);
    ZKB_CUDA(cudaMemcpyAsync(dA, A.data(), A.size() * 32, cudaMemcpyHostToDevice, st));
    ZKB_CUDA(cudaMemcpyAsync(dB, Bt.data(), Bt.size() * 32, cudaMemcpyHostToDevice, st));
    ZKB_TRY(launch("ntt_scale_pow", k_ntt_scale_pow<P>, g, dim3(256), 0, st, (const uint32_t*)d_src, d_sh,
                   (uint32_t)Ns, (const uint32_t*)dA, (const uint32_t*)dB, a));
    ZKB_TRY(ntt_run<P>(cx, *pl, d_sh, d_out, scratch, st));
    ZKB_TRY(launch("ntt_interleave", k_ntt_interleave, g, dim3(256), 0, st, (const uint4*)d_out, (uint4*)d_tgt,
                   (uint32_t)Ns, (uint32_t)K, (uint32_t)k));
    ZKB_CUDA(cudaStreamSynchronize(st));   // the host-side tables are rewritten for the next k
  }
  ZKB_CUDA(cudaEventRecord(cx.ev_b, st));
  ZKB_TRY(copy_d2h(cx, tgt, d_tgt, bt, st));
  ZKB_CUDA(cudaEventElapsedTime(&cx.last_kernel_ms, cx.ev_a, cx.ev_b));
  return set_status(ZKG_OK, nullptr, nullptr);
}

zkg_status ntt_plan_new(int curve, int m, const uint64_t* gen, int inverse, int kmax, cudaStream_t st,
                        NttPlan** out) {
  if (m < 0 || m > NTT_MMAX) return set_status(ZKG_ERR_ARG, "ntt", "m out of range [0, 30]");
  if (kmax <= 0) kmax = effective_kmax(curve, m);
  if (curve == ZKG_BN254) return build_plan_uncached<BnFr>(host::BN_FR, curve, m, gen, inverse, kmax, st, out);
  if (curve == ZKG_BLS12_381) return build_plan_uncached<BlsFr>(host::BLS_FR, curve, m, gen, inverse, kmax, st, out);
  return set_status(ZKG_ERR_ARG, "ntt", "unknown curve");
}

zkg_status ntt_plan_execute(const NttPlan& pl, const uint32_t* d_src, uint32_t* d_tgt, uint32_t* scratch,
                            cudaStream_t st) {
  Context* cx = nullptr;
  ZKB_TRY(get_context(&cx));
  if (pl.curve == ZKG_BN254) return ntt_run<BnFr>(*cx, pl, d_src, d_tgt, scratch, st);
  return ntt_run<BlsFr>(*cx, pl, d_src, d_tgt, scratch, st);
}

}  // namespace zkb

extern "C" {

zkg_status zkg_ntt(zkg_curve curve, int m, const uint64_t* gen, const uint64_t* src, uint64_t* tgt, int inverse) {
  if (curve == ZKG_BN254) return zkb::ntt_entry<zkb::BnFr>(zkb::host::BN_FR, curve, m, gen, src, tgt, inverse, false);
  if (curve == ZKG_BLS12_381)
    return zkb::ntt_entry<zkb::BlsFr>(zkb::host::BLS_FR, curve, m, gen, src, tgt, inverse, false);
  return zkb::set_status(ZKG_ERR_ARG, "zkg_ntt", "unknown curve");
}

zkg_status zkg_ntt_device(zkg_curve curve, int m, const uint64_t* gen, const uint64_t* d_src, uint64_t* d_tgt,
                          int inverse) {
  if (curve == ZKG_BN254) return zkb::ntt_entry<zkb::BnFr>(zkb::host::BN_FR, curve, m, gen, d_src, d_tgt, inverse, true);
  if (curve == ZKG_BLS12_381)
    return zkb::ntt_entry<zkb::BlsFr>(zkb::host::BLS_FR, curve, m, gen, d_src, d_tgt, inverse, true);
  return zkb::set_status(ZKG_ERR_ARG, "zkg_ntt_device", "unknown curve");
}

zkg_status zkg_ntt_shifted(zkg_curve curve, const uint64_t* eta, int m, const uint64_t* gen, const uint64_t* src,
                           uint64_t* tgt, int inverse) {
  if (curve == ZKG_BN254) return zkb::ntt_shifted_entry<zkb::BnFr>(zkb::host::BN_FR, curve, eta, m, gen, src, tgt, inverse);
  if (curve == ZKG_BLS12_381)
    return zkb::ntt_shifted_entry<zkb::BlsFr>(zkb::host::BLS_FR, curve, eta, m, gen, src, tgt, inverse);
  return zkb::set_status(ZKG_ERR_ARG, "zkg_ntt_shifted", "unknown curve");
}

zkg_status zkg_ntt_asymmetric(zkg_curve curve, int m_src, int m_tgt, const uint64_t* gen_src, const uint64_t* gen_tgt,
                              const uint64_t* src, uint64_t* tgt) {
  if (curve == ZKG_BN254)
    return zkb::ntt_asym_entry<zkb::BnFr>(zkb::host::BN_FR, curve, m_src, m_tgt, gen_src, gen_tgt, src, tgt);
  if (curve == ZKG_BLS12_381)
    return zkb::ntt_asym_entry<zkb::BlsFr>(zkb::host::BLS_FR, curve, m_src, m_tgt, gen_src, gen_tgt, src, tgt);
  return zkb::set_status(ZKG_ERR_ARG, "zkg_ntt_asymmetric", "unknown curve");
}

zkg_status zkg_release_cache(void) {
  zkb::Context* cx = nullptr;
  zkg_status st = zkb::get_context(&cx);
  if (st != ZKG_OK) return st;
  std::lock_guard<std::mutex> lk(cx->mu);
  cudaDeviceSynchronize();
  for (zkb::NttPlan* p : cx->ntt_plans) delete p;
  cx->ntt_plans.clear();
  if (cx->arena.base) cudaFree(cx->arena.base);
  cx->arena.base = nullptr;
  cx->arena.cap = cx->arena.used = 0;
  return ZKG_OK;
}

int zkg_set_ntt_kmax(int k) {
  const int prev = zkb::g_ntt_kmax;
  if (k >= 1 && k <= zkb::NTT_KMAX) {
    zkb::g_ntt_kmax = k;
    zkb::g_ntt_kmax_set = true;
  } else if (k == 0) {
    zkb::g_ntt_kmax = 8;
    zkb::g_ntt_kmax_set = false;
  }
  return prev;
}

// Times the largest pass size 7..11 for each m in [m_min, m_max] (forward transform on random
// device data) and keeps the fastest per size.
zkg_status zkg_autotune_ntt(zkg_curve curve, int m_min, int m_max, int* chosen) {
  if ((curve != ZKG_BN254 && curve != ZKG_BLS12_381) || m_min < 1 || m_max < m_min || m_max > 26)
    return zkb::set_status(ZKG_ERR_ARG, "zkg_autotune_ntt", "need 1 <= m_min <= m_max <= 26");
  uint32_t *d_x = nullptr, *d_y = nullptr;
  const size_t bytes = (size_t)32 << m_max;
  if (cudaMalloc(&d_x, bytes) != cudaSuccess || cudaMalloc(&d_y, bytes) != cudaSuccess) {
    if (d_x) cudaFree(d_x);
    return zkb::set_status(ZKG_ERR_NOMEM, "zkg_autotune_ntt", "buffers");
  }
  cudaMemset(d_x, 0x11, bytes);   // below both moduli word-wise; timing does not depend on values
  const uint64_t gen[4] = {0x0123456789abcdefULL, 0x0fedcba987654321ULL, 0x1111111111111111ULL, 0x0222222222222222ULL};
  const bool was_set = zkb::g_ntt_kmax_set;
  const int was_k = zkb::g_ntt_kmax;
  zkg_status st = ZKG_OK;
  for (int m = m_min; m <= m_max && st == ZKG_OK; m++) {
    float best = 1e30f;
    int bestk = 8;
    for (int k = 6; k <= zkb::NTT_KMAX && st == ZKG_OK; k++) {
      zkb::g_ntt_kmax = k;
      zkb::g_ntt_kmax_set = true;
      float t = 1e30f;
      for (int rep = 0; rep < 3 && st == ZKG_OK; rep++) {
        st = zkg_ntt_device(curve, m, gen, reinterpret_cast<const uint64_t*>(d_x), reinterpret_cast<uint64_t*>(d_y), 0);
        if (rep > 0) t = std::min(t, zkg_last_kernel_ms());
      }
      if (st == ZKG_OK && t < best) { best = t; bestk = k; }
    }
    if (st == ZKG_OK) {
      zkb::effective_kmax(curve, m);   // loads the persisted entries first, so they are not lost
      zkb::g_ntt_tuned[curve][m] = bestk;
      zkb::tune_cache_put("ntt", curve, m, zkb::device_sm_count(), &bestk, 1);
      if (chosen) chosen[m - m_min] = bestk;
    }
  }
  zkb::g_ntt_kmax = was_k;
  zkb::g_ntt_kmax_set = was_set;
  cudaFree(d_x);
  cudaFree(d_y);
  return st;
}

}  // extern "C"
