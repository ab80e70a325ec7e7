// NTT kernel instantiations for BlsFr (split from the planner so the fields compile in parallel).
#include "zkb_dpf.cuh"
#include "zkb_ntt_kernels.cuh"

namespace zkb {
template zkg_status ntt_launch_pass<BlsFr>(const NttPlan&, const NttPass&, const uint32_t*, uint32_t*, bool, cudaStream_t);
template zkg_status ntt_launch_table<BlsFr>(uint32_t*, const uint32_t*, const uint32_t*, int, uint32_t, cudaStream_t);
template zkg_status ntt_launch_pass<BlsFrD>(const NttPlan&, const NttPass&, const uint32_t*, uint32_t*, bool, cudaStream_t);
template zkg_status ntt_launch_table<BlsFrD>(uint32_t*, const uint32_t*, const uint32_t*, int, uint32_t, cudaStream_t);
}  // namespace zkb
