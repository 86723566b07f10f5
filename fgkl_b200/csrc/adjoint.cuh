// Adjoint (gradient) path: d(sum of log10 L)/d(per-read-position parameters) over every read x
// haplotype pair of a batch. There is no counterpart in fgkl; the recurrence is fgkl's PairHMM
// (reference.rs:20-64) under a continuous parameterisation, per read position:
//   MI = dI (insertion gap open), MD = dD (deletion gap open), II = DD = eps (gap continuation),
//   IM = 1 - eps, MM = 1 - dI - dD, priors 1 - e (match) and e / 3 (mismatch) (e = base error).
// fgkl's quantized match-to-match table agrees with MM = 1 - dI - dD to about 1e-6
// (model.rs:125-130) but is not differentiable, hence the continuous form.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "program.h"

namespace fgkl {

// Device view of an adjoint batch.
struct AdjView {
  const uint8_t* bases;
  const int64_t* read_off;  // global read -> first position
  const double* d_ins;      // per read position
  const double* d_del;
  const double* eps;
  const double* err;
  const uint8_t* hap_bases;
  const int64_t* hap_off;   // global haplotype -> first base
  const int32_t* read_region;  // global read -> region
  const int32_t* region_hap;   // region -> first global haplotype
  const int32_t* region_nhap;  // region -> haplotype count
  const int32_t* region_read;  // region -> first global read
  const int64_t* region_out;   // region -> first output element
  double* out;              // log10 L, row-major per region (reads x haplotypes)
  double* g_ins;            // gradients, per read position
  double* g_del;
  double* g_eps;
  double* g_err;
  unsigned long long* lost; // FP32 reads handed to FP64
};

struct AdjLaunch {
  AdjView v;
  const int32_t* tasks;  // global read indices
  int n_tasks;           // count, or the capacity when `count` is set
  const int* count;      // device-side count (FP64 recomputation queue), or nullptr
  int* task_counter;     // zeroed before the launch
  char* scratch;
  size_t scratch_stride; // bytes per warp: a pair whose backward columns exceed it runs with checkpoints
  int32_t* queue;        // FP32 launches: reads lost in FP32, for FP64 (per-bin slices), or nullptr
  const int* queue_off;  // per rows-per-lane bin: first queue slot (kAdjRowBins + 1 entries)
  int* queue_tail;       // per bin
};

constexpr int kAdjRowBins = 21;

// Rows per lane for a read of `len` positions (31 * rows >= len; even above 8).
__host__ __device__ inline int adj_rows(int len) {
  int rows = (len + 30) / 31;
  if (rows > 8) rows = (rows + 1) & ~1;
  return rows;
}
// Steps per recomputed block for a pair of `steps` forward steps whose per-warp scratch holds `cap`
// values per lane, with backward records of `rec` values and saved backward states of `state` values:
// the largest K >= min_k with K * rec + ceil(steps / K) * state <= cap, or 0 when there is none.
__host__ __device__ inline int adj_block_steps(long long cap, int steps, int rec, int state, int min_k) {
  long long K = (cap - state) / rec;
  if (K > steps) K = steps;
  for (int it = 0; it < 4096 && K >= min_k; ++it) {
    const long long nb = (steps + K - 1) / K;
    if (K * rec + nb * state <= cap) return static_cast<int>(K);
    const long long k2 = (cap - nb * state) / rec;
    K = k2 < K ? k2 : K - 1;
  }
  return 0;
}

// Bytes of per-warp scratch that store every backward column of haplotypes of at most
// `max_hap_len` bases.
size_t adj_scratch_bytes(bool dbl, int rows, int max_hap_len);
// The least per-warp scratch with which haplotypes of at most `max_hap_len` bases run with
// checkpoints: backward states saved every K steps and each block of K columns recomputed before the
// forward sweep reads it (about sqrt of the stored-column bytes).
size_t adj_checkpoint_bytes(bool dbl, int rows, int max_hap_len);
// Bytes of per-warp scratch that store `columns` backward columns.
size_t adj_column_bytes(bool dbl, int rows, int columns);
// `checkpointed`: the instantiation that recomputes backward columns from checkpoints for pairs whose
// columns exceed the launch's per-warp scratch (the other has no such path and must not get them).
void adj_occupancy(bool dbl, int rows, bool checkpointed, int* blocks_per_sm, int* threads_per_block);
cudaError_t adj_launch(bool dbl, int rows, bool checkpointed, int blocks, const AdjLaunch& a, cudaStream_t stream);

}  // namespace fgkl
