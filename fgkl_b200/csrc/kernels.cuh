// Launch interface of the sm_100a PairHMM kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "program.h"

namespace fgkl {

// Arithmetic of one kernel instantiation.
enum class Kind : int {
  kPackedF32 = 0,  // two reads per lane set, FP32x2 arithmetic, rows-per-lane 1..8
  kOneF32 = 1,     // one read, FP32, rows-per-lane 10..20 (even)
  kOneF64 = 2,     // one read, FP64, rows-per-lane 1..8 and 10..20 (even)
};

struct LaunchArgs {
  BatchView v;
  const Task* tasks;     // this launch's tasks
  int n_tasks;           // host-known count, or the capacity when `count` is set
  const int* count;      // device-side task count (recomputation queues), or nullptr
  int* task_counter;     // zeroed before the launch
  char* scratch;
  size_t scratch_stride; // bytes per warp
  int min_accept_plain;  // 1: results below the single-precision threshold are lost
};

// The pass between the first pass and the recomputation: queues lost pairs.
struct CollectArgs {
  BatchView v;
  Task* queue;           // recomputation queue: (read, distinct haplotype) FP64 tasks
  const int* queue_off;  // per rows-per-lane bin: first queue index (one past the last bin at the end)
  int* queue_tail;       // per bin: tasks queued
};

// Rows per lane the instantiations cover.
int max_rows(Kind k);
// Bytes of per-warp scratch one task of this instantiation needs.
size_t scratch_bytes(Kind k, int rows, int max_slots, int max_nodes, int max_segs);
// Resident blocks per SM and threads per block of an instantiation.
void occupancy(Kind k, int rows, int* blocks_per_sm, int* threads_per_block);
// Launches one persistent grid of `blocks` blocks.
cudaError_t launch(Kind k, int rows, int blocks, const LaunchArgs& args, cudaStream_t stream);
// Launches the lost-pair collection over `n_regions` regions.
cudaError_t launch_collect(const CollectArgs& args, int n_regions, cudaStream_t stream);

}  // namespace fgkl
