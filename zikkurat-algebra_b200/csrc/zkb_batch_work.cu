// The batched mode's persistent kernel (see zkb_batch_work.h for the work-queue types): one
// launch drains a queue of MSM accumulation blocks and NTT pass tiles.
#include <cstdlib>

#include "zkb_batch_work.h"
#include "zkb_msm_accum.cuh"
#include "zkb_ntt_kernels.cuh"

namespace zkb {

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// true once *cnt >= target; false when the error word is set or the limit runs out (then it is
// set here)
__device__ bool wait_count(const uint32_t* cnt, uint32_t target, uint32_t limit, uint32_t* err) {
  for (uint32_t it = 0; it < limit; it++) {
    if (ld_acquire_u32(cnt) >= target) return true;
    if (*(volatile uint32_t*)err) return false;
    __nanosleep(128);
  }
  atomicExch(err, 1u);
  return false;
}

template <class PD, bool CG>
__device__ __noinline__ void ntt_tile_dispatch(const NttPassDesc& d, uint32_t tile, uint32_t* sm) {
#define ZKB_NTT_TILE(K)                                                                              \
  case K:                                                                                          \
    if (d.inverse) ntt_inv_tile<PD, K, CG>(tile, d.in, d.out, d.m, d.Mp, d.s, d.om, d.tw, d.scale, d.W, sm); \
    else ntt_fwd_tile<PD, K, CG>(tile, d.in, d.out, d.m, d.Mp, d.s, d.om, d.tw, d.W, sm);          \
    break;
  switch (d.K) {
    ZKB_NTT_TILE(1) ZKB_NTT_TILE(2) ZKB_NTT_TILE(3) ZKB_NTT_TILE(4) ZKB_NTT_TILE(5) ZKB_NTT_TILE(6)
    ZKB_NTT_TILE(7) ZKB_NTT_TILE(8) ZKB_NTT_TILE(9) ZKB_NTT_TILE(10) ZKB_NTT_TILE(11)
    default: break;
  }
#undef ZKB_NTT_TILE
}

template <class CD, class PD, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_batch_work(const BatchWork W) {
  extern __shared__ uint4 smem_u4[];
  __shared__ uint2 s_task;
  __shared__ int s_go;
  for (;;) {
    __syncthreads();   // the previous task is finished by every thread; s_task may be rewritten
    if (threadIdx.x == 0) {
      const uint32_t t = atomicAdd(W.next, 1u);
      s_task = (t < W.ntasks && *(volatile uint32_t*)W.error == 0u) ? W.tasks[t] : make_uint2(0xffffffffu, 0u);
    }
    __syncthreads();
    const uint2 task = s_task;
    if (task.x == 0xffffffffu) return;
    if (task.x == 0) {
      accum_block<CD, 2, NT>(task.y, W.ent, W.off, W.nseg, W.nch, W.L, W.bases, W.bsum, W.key, W.pt, smem_u4);
      continue;
    }
    const NttPassDesc& d = W.descs[task.x - 1];
    if (threadIdx.x == 0) {
      s_go = d.dep < 0 ? 1 : (wait_count(W.done + d.dep, d.dep_count, W.wait_limit, W.error) ? 1 : 0);
      __threadfence();
    }
    __syncthreads();
    if (!s_go) continue;
    uint32_t* sm = reinterpret_cast<uint32_t*>(smem_u4);
    if (d.dep < 0) ntt_tile_dispatch<PD, false>(d, task.y, sm);
    else ntt_tile_dispatch<PD, true>(d, task.y, sm);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();   // release: this tile's output before its count
      atomicAdd(W.done + (task.x - 1), 1u);
    }
  }
}

// CTA shape: BN254 runs two 256-thread CTAs per SM (measured faster over a mixed queue than one
// 384-thread CTA per SM, whose NTT tiles leave a third of the threads idle), BLS12-381 one
// 256-thread CTA per SM. ZKB_BATCH_THREADS=384 selects one 384-thread CTA per SM for BN254.
static const int g_batch_threads = [] {
  const char* v = std::getenv("ZKB_BATCH_THREADS");
  return v && std::atoi(v) == 384 ? 384 : 256;
}();

int batch_work_threads(int curve) { return curve == ZKG_BN254 ? g_batch_threads : 256; }

template <class CD, class PD, int NT, int MINB>
static zkg_status prepare(int* per_sm) {
  ZKB_CUDA(cudaFuncSetAttribute(k_batch_work<CD, PD, NT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)BATCH_WORK_SMEM));
  ZKB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_batch_work<CD, PD, NT, MINB>, NT, BATCH_WORK_SMEM));
  return ZKG_OK;
}

zkg_status batch_work_prepare(int curve, int* per_sm) {
  if (curve == ZKG_BN254) {
    if (g_batch_threads == 384) return prepare<MsmCurve<BN254>::type, BnFrD, 384, 1>(per_sm);
    return prepare<MsmCurve<BN254>::type, BnFrD, 256, 2>(per_sm);
  }
  return prepare<MsmCurve<BLS12_381>::type, BlsFrD, 256, 1>(per_sm);
}

zkg_status batch_work_launch(int curve, const BatchWork& W, int grid, cudaStream_t st) {
  if (curve == ZKG_BN254) {
    if (g_batch_threads == 384)
      return launch("batch_work", k_batch_work<MsmCurve<BN254>::type, BnFrD, 384, 1>, dim3(grid), dim3(384),
                    BATCH_WORK_SMEM, st, W);
    return launch("batch_work", k_batch_work<MsmCurve<BN254>::type, BnFrD, 256, 2>, dim3(grid), dim3(256),
                  BATCH_WORK_SMEM, st, W);
  }
  return launch("batch_work", k_batch_work<MsmCurve<BLS12_381>::type, BlsFrD, 256, 1>, dim3(grid), dim3(256),
                BATCH_WORK_SMEM, st, W);
}

}  // namespace zkb
