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
  double* g_ins;            // gradients, per read position; zero before the first launch, then summed into
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
  size_t scratch_stride; // bytes per warp (adj_scratch_bytes of the launch's largest pair)
  int32_t* queue;        // FP32 launches: reads lost in FP32, for FP64 (per-bin slices), or nullptr
  const int* queue_off;  // per rows-per-lane bin: first queue slot (kAdjRowBins + 1 entries)
  int* queue_tail;       // per bin
};

constexpr int kAdjRowBins = 21;
constexpr int kAdjMaxBlockRead = 620;  // longest read one 32 x 20-row block holds
constexpr int kAdjLongRows = 8;        // rows per lane of longer reads, strip-mined over row blocks

// Rows per lane for a read of `len` positions: 31 * rows >= len (even above 8) up to 620 bases,
// kAdjLongRows beyond.
__host__ __device__ inline int adj_rows(int len) {
  if (len > kAdjMaxBlockRead) return kAdjLongRows;
  int rows = (len + 30) / 31;
  if (rows > 8) rows = (rows + 1) & ~1;
  return rows;
}
// Row blocks of 32 * rows rows that a read of `len` positions spans, with at least one padding row
// above the read (the row that collects the backward start mass): 1 up to 620 bases.
__host__ __device__ inline int adj_row_blocks(int len, int rows) { return (len + 32 * rows) / (32 * rows); }

// Bytes of per-warp scratch a pair of a `read_len`-position read and a `hap_len`-base haplotype
// needs: the backward checkpoints of every row block, and, for a strip-mined read, the rows that
// pass between row blocks.
size_t adj_scratch_bytes(bool dbl, int rows, int read_len, int hap_len);
void adj_occupancy(bool dbl, int rows, int* blocks_per_sm, int* threads_per_block);
cudaError_t adj_launch(bool dbl, int rows, int blocks, const AdjLaunch& a, cudaStream_t stream);

}  // namespace fgkl
