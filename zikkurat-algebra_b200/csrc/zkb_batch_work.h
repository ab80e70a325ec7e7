// The batched mode's persistent kernel: work-queue types shared by the batch planner
// (zkb_msm.cu) and the kernel (zkb_batch_work.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "zkb_runtime.h"

namespace zkb {

// ============================================================ the batch's persistent kernel
//
// One launch drains a work queue that holds every request's share of the bucket accumulation
// (blocks of 256 accumulation chunks of the batch's segmented MSM pipeline) and every tile of
// every NTT pass of the batch. CTAs take tasks in queue order with one atomic counter. A tile of
// NTT pass p reads all of pass p - 1's output, so it first waits until pass p - 1's tile counter
// is complete; the queue lists all first-pass tiles, then the accumulation blocks, then the
// second-pass tiles, and so on, so every task a tile waits for was taken earlier by a running
// CTA and finishes without waiting for anything later (no deadlock, whatever the grid size).
// The wait is a bounded spin: after `wait_limit` polls the CTA sets the error word, which stops
// every CTA at its next task, and the host reports ZKG_ERR_TIMEOUT. Data written by a pass are
// read by the next pass through L2 only (ld.global.cg), after an acquire on the counter.
struct NttPassDesc {
  const uint32_t* in;
  uint32_t* out;
  const uint32_t* om;
  const uint32_t* tw;
  const uint32_t* scale;
  int m, Mp, s, K, W, inverse;
  uint32_t ntiles;
  int dep;              // pass whose output this pass reads (-1: the NTT's input)
  uint32_t dep_count;   // tiles of that pass
};

struct BatchWork {
  const uint2* tasks;   // x = 0: accumulation block y; x = d + 1: tile y of NTT pass d
  uint32_t ntasks;
  uint32_t* next;       // queue position (zeroed before each run)
  uint32_t* done;       // completed tiles per pass (zeroed before each run)
  uint32_t* error;      // set by a wait that ran out
  const NttPassDesc* descs;
  uint32_t wait_limit;
  // the accumulation (k_msm_accum's arguments)
  const uint32_t* ent;
  const uint32_t* off;
  uint32_t nseg, nch, L;
  const uint32_t* bases;
  uint32_t *bsum, *key, *pt;
};

// Shared memory of one k_batch_work CTA: the largest NTT tile (2048 elements) or accumulation
// prefetch stages (at most 48 KB: 384 threads x 2 stages x 64-byte bases, or 256 x 2 x 96).
static constexpr size_t BATCH_WORK_SMEM = 64 * 1024;

// Sets the kernel's shared-memory limit and returns its resident CTAs per SM (curve: ZKG_BN254 /
// ZKG_BLS12_381; the MSM pipeline's and the FP64 NTT's field types of that curve).
zkg_status batch_work_prepare(int curve, int* per_sm);
// Threads per k_batch_work CTA for a curve (an accumulation task covers that many chunks).
int batch_work_threads(int curve);
// Enqueues one k_batch_work launch on st.
zkg_status batch_work_launch(int curve, const BatchWork& W, int grid, cudaStream_t st);

}  // namespace zkb
