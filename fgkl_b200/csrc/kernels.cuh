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
  int use_prefix;        // 1: run the prefix-only program
  int rescue;            // 1: write only pairs whose output is NaN
  Task* queue;           // recomputation queue (single-read double-precision tasks), or nullptr
  const int* queue_off;  // per rows-per-lane bin: first queue index
  int* queue_tail;       // per bin: tasks queued
  int min_accept_plain;  // 1: results below the single-precision threshold are lost
};

// Rows per lane the instantiations cover.
int max_rows(Kind k);
// Bytes of per-warp scratch one task of this instantiation needs.
size_t scratch_bytes(Kind k, int rows, int max_slots, int max_nodes, int max_segs);
// Resident blocks per SM and threads per block of an instantiation.
void occupancy(Kind k, int rows, int* blocks_per_sm, int* threads_per_block);
// Launches one persistent grid of `blocks` blocks.
cudaError_t launch(Kind k, int rows, int blocks, const LaunchArgs& args, cudaStream_t stream);

}  // namespace fgkl
