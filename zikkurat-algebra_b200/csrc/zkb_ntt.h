// NTT plan types shared by the planner (zkb_ntt.cu) and the per-field kernel units
// (zkb_ntt_bn.cu, zkb_ntt_bls.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "zkb_runtime.h"

namespace zkb {

static constexpr int NTT_KMAX = 11;
// Largest transform: 2^30 points, the bound of the reference's `int N = 1 << m`
// (bn128_poly_mont.c:453; any generator is accepted, so m is not bounded by the field's
// two-adicity). The reference itself stops earlier: its twiddle buffer size 8*NLIMBS*halfN is an
// int that overflows from m = 27, so its malloc fails and it aborts; every m it runs, this runs.
static constexpr int NTT_MMAX = 30;
static constexpr int NTT_THREADS = 256;   // threads per NTT pass CTA

struct NttPass {
  int k, s, Mp;   // bits in this pass, bits before it, bits after it (forward order)
};

struct NttPlan {
  int curve = -1, m = -1, inverse = 0, kmax = 0;
  bool dpf = false;                  // tables in radix R' = 2^260: passes multiply on the FP64 pipe
  uint64_t gen[4] = {0, 0, 0, 0};
  std::vector<NttPass> passes;
  uint32_t* d_tw = nullptr;          // N inter-pass twiddles (only with >= 2 passes)
  uint32_t* d_tw_last = nullptr;     // inverse with >= 2 passes: d_tw times (1/2)^m, for the last pass
  uint32_t* d_om[NTT_KMAX + 1] = {nullptr};
  uint32_t* d_scale = nullptr;       // (1/2)^m for the inverse
  size_t bytes = 0;
  ~NttPlan() {
    if (d_tw) cudaFree(d_tw);
    if (d_tw_last) cudaFree(d_tw_last);
    for (auto p : d_om) if (p) cudaFree(p);
    if (d_scale) cudaFree(d_scale);
  }
};

// One pass of the plan on stream st (defined per field in zkb_ntt_bn.cu / zkb_ntt_bls.cu).
template <class P>
zkg_status ntt_launch_pass(const NttPlan& pl, const NttPass& q, const uint32_t* in, uint32_t* out,
                           bool last_inverse, cudaStream_t st);
// T[e] = A[e mod 2^a] * Bt[e >> a] for e < N.
template <class P>
zkg_status ntt_launch_table(uint32_t* T, const uint32_t* A, const uint32_t* Bt, int a, uint32_t N, cudaStream_t st);

// A plan owned by the caller (not entered in the context's cache): for batches and servers that
// keep plans alive across graph replays. Built synchronously on stream st.
zkg_status ntt_plan_new(int curve, int m, const uint64_t* gen, int inverse, int kmax, cudaStream_t st,
                        NttPlan** out);
// Runs a plan d_src -> d_tgt on stream st; scratch (2^m elements) is needed with >= 2 passes.
zkg_status ntt_plan_execute(const NttPlan& pl, const uint32_t* d_src, uint32_t* d_tgt, uint32_t* scratch,
                            cudaStream_t st);

}  // namespace zkb
