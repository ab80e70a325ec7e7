// NTT entry point that allocates no memory: zkg_ntt_device_noalloc.
//
// Some callers cannot call cudaMalloc: a process whose framework memory pool already owns the
// device memory (the caching allocator of an ML framework reserves most of HBM, so a foreign
// cudaMalloc fails or fragments it), or a host application that gives this library a fixed
// device-memory quota of zero. zkg_ntt_device allocates its scratch buffer and twiddle tables on
// first use; this variant keeps all of them in one fixed-size array in the library's own device
// memory instead.
//
// The array below is part of the library's device image: every GPU that loads the library holds
// it (4 MiB + 24 KiB) until the process exits. It bounds the transform size to 2^16 elements.
// Every call shares it and leaves the last call's contents behind; nothing in it has to start at
// zero, because each call writes every word it later reads. Calls that overlapped on the GPU
// would race on it, so calls are serialised by a lock and each call returns only after its work
// on the device has finished.
//
// Every call synchronises the whole device: it waits for all earlier device work (the inputs may
// come from any stream), copies its small tables with blocking copies and waits for its own
// kernels before it returns. It is therefore not for latency-critical loops, and it must not be
// called while any stream capture is active in the process (the synchronisation would end the
// capture with an error).
//
// In host code `g_ntt_noalloc_scratch` names a host-side stand-in, not device memory: a kernel
// given that name faults or silently uses the wrong memory. The device address is looked up with
// cudaGetSymbolAddress once per device (with that device current) on the first call there.
#include <cstring>
#include <mutex>

#include "zkb_host_ec.h"
#include "zkb_ntt_kernels.cuh"
#include "zkb_runtime.h"

namespace zkb {

static constexpr int NA_MAX_LOG = 16;                  // largest supported transform: 2^16 elements
static constexpr int NA_KMAX = 8;                      // pass size; m <= 16 gives at most 2 passes
static constexpr size_t NA_N = (size_t)1 << NA_MAX_LOG;
// word offsets inside the scratch array (8 words per Fr element)
static constexpr size_t NA_BUF = 0;                              // inter-pass buffer, NA_N elements
static constexpr size_t NA_TW = NA_BUF + NA_N * 8;                // inter-pass twiddles, NA_N elements
static constexpr size_t NA_A = NA_TW + NA_N * 8;                  // h^j, j < 2^8
static constexpr size_t NA_BT = NA_A + 256 * 8;                   // h^(j*2^a), j < 2^8
static constexpr size_t NA_OM0 = NA_BT + 256 * 8;                 // network powers, first pass size
static constexpr size_t NA_OM1 = NA_OM0 + 128 * 8;                // network powers, second pass size
static constexpr size_t NA_SCALE = NA_OM1 + 128 * 8;              // (1/2)^m
static constexpr size_t NA_WORDS = NA_SCALE + 8;

static __device__ __align__(256) uint32_t g_ntt_noalloc_scratch[NA_WORDS];

static std::mutex g_na_mu;
static uint32_t* g_na_ptr[64] = {nullptr};   // device address of the scratch, per device

template <class P, int K>
static zkg_status na_pass(const NttPass& q, int m, const uint32_t* in, uint32_t* out, const uint32_t* om,
                          const uint32_t* tw, const uint32_t* scale, bool inverse, cudaStream_t st) {
  const int E = (1 << K) < 8 ? (1 << K) : 8;
  const int W = 256 * E >> K;
  const uint32_t ncols = 1u << (m - K);
  const uint32_t grid = (ncols + W - 1) / W;
  const size_t smem = (size_t)W * ((size_t)1 << K) * 32;
  if (!inverse) {
    ZKB_CUDA(cudaFuncSetAttribute(k_ntt_fwd<P, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    return launch("ntt_fwd_noalloc", k_ntt_fwd<P, K>, dim3(grid), dim3(256), smem, st, in, out, m, q.Mp, q.s, om,
                  tw, W);
  }
  ZKB_CUDA(cudaFuncSetAttribute(k_ntt_inv<P, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
  return launch("ntt_inv_noalloc", k_ntt_inv<P, K>, dim3(grid), dim3(256), smem, st, in, out, m, q.Mp, q.s, om,
                tw, scale, W);
}

template <class P>
static zkg_status na_dispatch(const NttPass& q, int m, const uint32_t* in, uint32_t* out, const uint32_t* om,
                              const uint32_t* tw, const uint32_t* scale, bool inverse, cudaStream_t st) {
  switch (q.k) {
    case 1: return na_pass<P, 1>(q, m, in, out, om, tw, scale, inverse, st);
    case 2: return na_pass<P, 2>(q, m, in, out, om, tw, scale, inverse, st);
    case 3: return na_pass<P, 3>(q, m, in, out, om, tw, scale, inverse, st);
    case 4: return na_pass<P, 4>(q, m, in, out, om, tw, scale, inverse, st);
    case 5: return na_pass<P, 5>(q, m, in, out, om, tw, scale, inverse, st);
    case 6: return na_pass<P, 6>(q, m, in, out, om, tw, scale, inverse, st);
    case 7: return na_pass<P, 7>(q, m, in, out, om, tw, scale, inverse, st);
    case 8: return na_pass<P, 8>(q, m, in, out, om, tw, scale, inverse, st);
  }
  return set_status(ZKG_ERR_ARG, "ntt_noalloc", "pass size");
}

// Same transform as zkg_ntt_device (same pass schedule and exact field operations) on the
// 32-bit-limb kernels (BnFr / BlsFr products; zkg_ntt_device multiplies on the FP64 pipe, and
// both are exact, so the outputs are identical), with every table and intermediate in the
// static scratch. Host-side tables live in fixed stack arrays.
template <class P>
static zkg_status ntt_noalloc(const host::Field<4>& F, int m, const uint64_t* gen, const uint64_t* d_src,
                              uint64_t* d_tgt, int inverse) {
  if (m < 0 || m > NA_MAX_LOG)
    return set_status(ZKG_ERR_ARG, "zkg_ntt_device_noalloc",
                      "m out of range: this entry point supports transforms of at most 2^16 elements "
                      "(use zkg_ntt_device above that)");
  if (!gen || !d_src || !d_tgt) return set_status(ZKG_ERR_ARG, "zkg_ntt_device_noalloc", "null pointer");
  const size_t N = (size_t)1 << m, bytes = N * 32;
  const char* s0 = reinterpret_cast<const char*>(d_src);
  const char* t0 = reinterpret_cast<const char*>(d_tgt);
  if (s0 < t0 + bytes && t0 < s0 + bytes)
    return set_status(ZKG_ERR_ARG, "zkg_ntt_device_noalloc", "src and tgt must not overlap");

  int dev = 0;
  ZKB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_status(ZKG_ERR_ARG, "zkg_ntt_device_noalloc", "device index out of range");
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_ptr[dev]) {   // once per device, with that device current
    uint32_t* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_ntt_noalloc_scratch);
    if (e != cudaSuccess) return set_status(ZKG_ERR_CUDA, "cudaGetSymbolAddress", cudaGetErrorString(e));
    g_na_ptr[dev] = p;
  }
  uint32_t* scr = g_na_ptr[dev];
  const cudaStream_t st = 0;
  ZKB_CUDA(cudaDeviceSynchronize());   // the inputs may have been written on any stream

  if (m == 0) {   // copy (bn128_poly_mont.c:420-423)
    ZKB_CUDA(cudaMemcpyAsync(d_tgt, d_src, 32, cudaMemcpyDeviceToDevice, st));
    ZKB_CUDA(cudaStreamSynchronize(st));
    return set_status(ZKG_OK, nullptr, nullptr);
  }

  // pass schedule (as zkg_ntt_device with passes of at most 8 bits)
  NttPass ps[2];
  const int np = (m + NA_KMAX - 1) / NA_KMAX;
  int sbits = 0;
  for (int p = 0; p < np; p++) {
    const int rem = m - sbits, left = np - p;
    ps[p].k = (rem + left - 1) / left;
    ps[p].s = sbits;
    ps[p].Mp = m - sbits - ps[p].k;
    sbits += ps[p].k;
  }

  host::El<4> g;
  std::memcpy(g.v, gen, 32);
  const host::El<4> h = inverse ? host::inv(F, g) : g;
  // small-network powers w_k^j, w_k = h^(2^(m-k)), for each distinct pass size
  host::El<4> om[2][128];
  int om_k[2] = {0, 0};
  for (int p = 0; p < np; p++) {
    const int slot = (p == 0 || ps[p].k == ps[0].k) ? 0 : 1;
    if (om_k[slot] == ps[p].k) continue;
    om_k[slot] = ps[p].k;
    host::El<4> w = h;
    for (int i = 0; i < m - ps[p].k; i++) w = host::mul(F, w, w);
    host::El<4> x = host::one(F);
    for (int j = 0; j < (1 << (ps[p].k - 1)); j++) { om[slot][j] = x; x = host::mul(F, x, w); }
    ZKB_CUDA(cudaMemcpy(scr + (slot ? NA_OM1 : NA_OM0), om[slot], (size_t)32 << (ps[p].k - 1),
                        cudaMemcpyHostToDevice));
  }
  if (np >= 2) {   // inter-pass twiddles T[e] = h^e, e < N, from two tables of 2^8 entries
    const int a = (m + 1) / 2;
    host::El<4> A[256], Bt[256];
    host::El<4> x = host::one(F);
    for (int j = 0; j < (1 << a); j++) { A[j] = x; x = host::mul(F, x, h); }
    const host::El<4> step = x;
    x = host::one(F);
    for (int j = 0; j < (1 << (m - a)); j++) { Bt[j] = x; x = host::mul(F, x, step); }
    ZKB_CUDA(cudaMemcpy(scr + NA_A, A, (size_t)32 << a, cudaMemcpyHostToDevice));
    ZKB_CUDA(cudaMemcpy(scr + NA_BT, Bt, (size_t)32 << (m - a), cudaMemcpyHostToDevice));
    ZKB_TRY(ntt_launch_table<P>(scr + NA_TW, scr + NA_A, scr + NA_BT, a, (uint32_t)N, st));
  }
  if (inverse) {
    host::El<4> two = host::zero<4>();
    two.v[0] = 2;
    const host::El<4> sc = host::pow_u64(F, host::inv(F, host::from_std(F, two)), (uint64_t)m);
    ZKB_CUDA(cudaMemcpy(scr + NA_SCALE, sc.v, 32, cudaMemcpyHostToDevice));
  }

  const uint32_t* in = reinterpret_cast<const uint32_t*>(d_src);
  for (int i = 0; i < np; i++) {
    uint32_t* out = (np - 1 - i) % 2 == 0 ? reinterpret_cast<uint32_t*>(d_tgt) : scr + NA_BUF;
    const NttPass& q = inverse ? ps[np - 1 - i] : ps[i];
    const uint32_t* omp = scr + ((q.k == om_k[0]) ? NA_OM0 : NA_OM1);
    ZKB_TRY(na_dispatch<P>(q, m, in, out, omp, q.Mp > 0 ? scr + NA_TW : nullptr,
                           (inverse && i == np - 1) ? scr + NA_SCALE : nullptr, inverse != 0, st));
    in = out;
  }
  ZKB_CUDA(cudaStreamSynchronize(st));
  return set_status(ZKG_OK, nullptr, nullptr);
}

}  // namespace zkb

extern "C" zkg_status zkg_ntt_device_noalloc(zkg_curve curve, int m, const uint64_t* gen, const uint64_t* d_src,
                                             uint64_t* d_tgt, int inverse) {
  if (curve == ZKG_BN254) return zkb::ntt_noalloc<zkb::BnFr>(zkb::host::BN_FR, m, gen, d_src, d_tgt, inverse);
  if (curve == ZKG_BLS12_381)
    return zkb::ntt_noalloc<zkb::BlsFr>(zkb::host::BLS_FR, m, gen, d_src, d_tgt, inverse);
  return zkb::set_status(ZKG_ERR_ARG, "zkg_ntt_device_noalloc", "unknown curve");
}
