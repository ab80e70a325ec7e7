// NTT kernel instantiations for BnFr (split from the planner so the fields compile in parallel).
#include "zkb_dpf.cuh"
#include "zkb_ntt_kernels.cuh"

namespace zkb {
template zkg_status ntt_launch_pass<BnFr>(const NttPlan&, const NttPass&, const uint32_t*, uint32_t*, bool, cudaStream_t);
template zkg_status ntt_launch_table<BnFr>(uint32_t*, const uint32_t*, const uint32_t*, int, uint32_t, cudaStream_t);
template zkg_status ntt_launch_pass<BnFrD>(const NttPlan&, const NttPass&, const uint32_t*, uint32_t*, bool, cudaStream_t);
template zkg_status ntt_launch_table<BnFrD>(uint32_t*, const uint32_t*, const uint32_t*, int, uint32_t, cudaStream_t);
}  // namespace zkb
