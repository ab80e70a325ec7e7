// Block-level pieces of batch inversion (Montgomery's simultaneous inversion): multiplicative
// scans over the threads of a block. Used by the Fr vector operations' batch inverse
// (zkb_fr.cu) and by the MSM's affine bucket tree (zkb_msm_tree.cuh).
#pragma once
#include "zkb_field.cuh"

namespace zkb {

// Multiplicative exclusive scan over the threads of a block (REV: over the threads in reverse
// order, i.e. the product of the values of the threads after this one). The block's total
// product is returned in `total`. sw holds blockDim.x / 32 + 1 elements. Every thread of the
// block must call it.
template <class P, bool REV>
__device__ __forceinline__ Fe<P> block_mul_excl_scan(const Fe<P>& v, Fe<P>* sw, Fe<P>& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  auto shfl = [&](const Fe<P>& x, int d) {
    Fe<P> y;
#pragma unroll
    for (int k = 0; k < P::N; k++) y.v[k] = REV ? __shfl_down_sync(0xffffffffu, x.v[k], d) : __shfl_up_sync(0xffffffffu, x.v[k], d);
    return y;
  };
  const int pos = REV ? 31 - lane : lane;   // position along the scan direction
  Fe<P> incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Fe<P> y = shfl(incl, d);
    if (pos >= d) incl = fe_mul(incl, y);
  }
  Fe<P> excl = shfl(incl, 1);
  if (pos == 0) excl = fe_one<P>();
  const int wpos = REV ? nw - 1 - wid : wid;
  if (pos == 31) sw[wpos] = incl;   // the warp's total, by position along the scan
  __syncthreads();
  if (threadIdx.x == 0) {   // few warps: prefix products of the warp totals, one thread
    Fe<P> run = fe_one<P>();
    for (int w = 0; w < nw; w++) {
      const Fe<P> t = sw[w];
      sw[w] = run;
      run = fe_mul(run, t);
    }
    sw[nw] = run;
  }
  __syncthreads();
  total = sw[nw];
  const Fe<P> r = fe_mul(sw[wpos], excl);
  __syncthreads();   // sw may be reused by the next call
  return r;
}

}  // namespace zkb
