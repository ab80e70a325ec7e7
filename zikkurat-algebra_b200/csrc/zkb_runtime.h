// Per-device runtime state for the zkb200 library: streams, a grow-only scratch arena,
// pinned staging memory, events, the NTT plan cache and the resident base sets.
//
// The reference entry points are synchronous, caller-owned-buffer C calls with no global
// state (lib/cbits/curves/g1/proj/bn128_G1_proj.c:506-586 mallocs and frees per call). Here
// device memory is kept between calls instead, because cudaMalloc/cudaFree per call would
// cost more than a small MSM. Calls on one device are serialised by a mutex, which keeps the
// entry points safe to call from several host threads (the Haskell FFI with -threaded).
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/zkb200.h"

namespace zkb {

// NVTX range over a scope (host side): entry points and the MSM / NTT phases show up by name in
// a profiler's timeline (nsys, ncu's NVTX filters); without an attached tool the calls do nothing.
struct NvtxRange {
  bool open = true;
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  void end() {   // close early (the destructor then does nothing)
    if (open) nvtxRangePop();
    open = false;
  }
  ~NvtxRange() { end(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Records a status for zkg_last_status() and returns it.
zkg_status set_status(zkg_status s, const char* where, const char* detail);

#define ZKB_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return ::zkb::set_status(ZKG_ERR_CUDA, #call, cudaGetErrorString(e_));             \
  } while (0)

#define ZKB_TRY(expr)                                                                    \
  do {                                                                                   \
    zkg_status s_ = (expr);                                                              \
    if (s_ != ZKG_OK) return s_;                                                         \
  } while (0)

// Grow-only device arena. take() hands out 256-byte aligned sub-ranges of one buffer; reset()
// makes the whole buffer reusable. Growing frees the old buffer, so pointers from take() are
// valid only until the next reserve().
struct Arena {
  char* base = nullptr;
  size_t cap = 0;
  size_t used = 0;
  zkg_status reserve(size_t bytes);
  void reset() { used = 0; }
  void* take(size_t bytes) {
    size_t off = (used + 255) & ~size_t(255);
    if (off + bytes > cap) return nullptr;
    used = off + bytes;
    return base + off;
  }
};

struct NttPlan;  // zkb_ntt.cu

struct Context {
  int device = -1;
  int sm_count = 0;
  cudaStream_t stream = nullptr;    // main compute stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_copy = nullptr;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  Arena arena;                      // per-call scratch
  void* pinned = nullptr;           // small pinned staging for results
  size_t pinned_cap = 0;
  std::mutex mu;
  std::vector<NttPlan*> ntt_plans;  // LRU-less cache, bounded by count
  float last_kernel_ms = 0.f;       // device time of the last hot-kernel region (for the bench)
  cudaEvent_t ev_phase[8] = {nullptr};
  cudaEvent_t ev_part[4] = {nullptr};   // host->device copy of MSM part q's bases finished
  cudaEvent_t ev_scal[4] = {nullptr};   // host->device copy of MSM part q's scalars finished
  cudaEvent_t ev_acc[4] = {nullptr};    // MSM part q's level-1 accumulation finished
  cudaEvent_t ev_fold[4] = {nullptr};   // MSM part q's fold levels finished (on side_stream)
  cudaStream_t side_stream = nullptr;   // MSM fold levels of a part, overlapping the next part
  float last_phase_ms[8] = {0.f};   // MSM: sort, accumulate (level 1), fold levels, bucket reduce
  int nphase = 0;
  uint32_t last_msm_entries = 0;    // non-zero digits of the last MSM (= bucket mixed additions)
  int last_msm_c = 0, last_msm_nwin = 0;
  cudaStream_t user_stream = nullptr;   // compute stream chosen by the caller (0 = own stream)
  // page-locked staging slots for copies of pageable caller buffers (copy_h2d / copy_d2h)
  static constexpr int NSTAGE = 3;
  void* stage[NSTAGE] = {nullptr};
  size_t stage_bytes = 0;
  cudaEvent_t stage_ev[NSTAGE] = {nullptr};
  unsigned stage_next = 0;
  cudaStream_t compute() const { return user_stream ? user_stream : stream; }
  uint32_t* d_check = nullptr;      // device bounds-check word (ZKB_DEVICE_CHECKS=1), else null
};

// Device bounds checks (environment ZKB_DEVICE_CHECKS=1; off by default). Kernels given a non-null
// check word test the indices they derive from data (digit buckets, entry positions, gathered
// point indices, segment ids) before using them; a failed test sets a bit in the word and the
// access is skipped or redirected to a valid element, so the kernel never leaves its buffers.
// After the call the host reads the word and reports ZKG_ERR_CUDA with the bits. These checks
// stand in for compute-sanitizer, which is not available here.
enum DevCheckBits : uint32_t {
  CHK_BUCKET = 1u,     // a digit's bucket outside [1, 2^(c-1)]
  CHK_ENTRY = 2u,      // a scatter position outside the entry array
  CHK_POINT = 4u,      // a gathered point index outside the base set
  CHK_SEGMENT = 8u,    // a segment id outside the segment table
};
extern const bool g_dev_checks;
// The context's check word when checks are on (allocated on first use), else null.
uint32_t* dev_check_word(Context& cx);
// Reads and clears the word after the call's work finished; a non-zero word becomes an error.
zkg_status dev_check_report(Context& cx, const char* where);

// Context of the current CUDA device, created on first use.
zkg_status get_context(Context** out);
zkg_status pinned_reserve(Context& cx, size_t bytes);

// Copies between caller host buffers and the device. A page-locked host buffer goes straight to
// the copy engine (asynchronous on st). A pageable one (the usual case: GHC's pinned arrays are
// not page-locked for CUDA) is staged through the context's page-locked slots in chunks, the
// host memcpy of each chunk spread over a pool of host threads and overlapping the DMA of the
// previous chunk; copy_h2d returns once the last chunk's DMA is queued on st (the source may be
// reused then), copy_d2h once the data are in dst. ZKB_STAGE=0 sends everything through
// cudaMemcpyAsync.
zkg_status copy_h2d(Context& cx, void* dst, const void* src, size_t bytes, cudaStream_t st);
zkg_status copy_d2h(Context& cx, void* dst, const void* src, size_t bytes, cudaStream_t st);

// Persisted autotuning results. When the environment variable ZKG_TUNE_CACHE names a file,
// tuned settings are read from it on first use and every autotuner run rewrites it, so later
// processes (the drop-in entry points included) start with the tuned choices. One entry per
// line: "<kind> <curve> <size> <sm_count> <values...>"; entries recorded on a GPU with another
// SM count are kept in the file but not used. Without the variable the results live for the
// process only.
bool tune_cache_get(const char* kind, int curve, int size, int sms, int* vals, int nvals);
void tune_cache_put(const char* kind, int curve, int size, int sms, const int* vals, int nvals);
int device_sm_count();

// Kernel launch with launch counting and error check.
extern std::atomic<uint64_t> g_launches;
template <typename... KArgs, typename... Args>
inline zkg_status launch(const char* name, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                         cudaStream_t st, Args... args) {
  if (grid.x == 0 || grid.y == 0 || grid.z == 0) return ZKG_OK;
  kern<<<grid, block, smem, st>>>(args...);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_status(ZKG_ERR_CUDA, name, cudaGetErrorString(e));
  return ZKG_OK;
}

}  // namespace zkb
