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
  kOneF32Pd = 3,   // PD-HMM, one read, FP32, rows-per-lane 1..8 and 10..20 (even)
  kOneF64Pd = 4,   // PD-HMM, one read, FP64, same rows
  kPackedF32Pd = 5,  // PD-HMM, two reads per lane set in FP32x2, rows-per-lane 1..8
  // Reads longer than kMaxBlockRead bases: one read against one distinct haplotype, unshared, the
  // rows strip-mined over blocks of 32 * R rows (rows-per-lane R from long_rows).
  kLongF32 = 6,
  kLongF64 = 7,
  kLongF32Pd = 8,
  kLongF64Pd = 9,
  // PD-HMM regions whose reads hold more read bytes than the class bit sets cover: every pair as in
  // the long kinds, with the prior decided by comparing bytes (any read length).
  kGenericF32Pd = 10,
  kGenericF64Pd = 11,
};
constexpr int kNumKinds = 12;

// Longest read a single 32 * R-row block holds (lane 0 is padding: 31 rows per lane x 20).
constexpr int kMaxBlockRead = 620;
// Rows-per-lane values of the strip-mined kinds: 8, 10, 12 and 16 for plain FP32 (kLongF32); 4, 6
// and 8 for the others, whose per-row state (FP64 values, PD branch values) takes more registers.
constexpr int kNumLongRows = 4;
__host__ __device__ constexpr int long_rows_value(int i, bool wide) {
  return wide ? (i == 0 ? 8 : (i == 1 ? 10 : (i == 2 ? 12 : 16))) : (i == 0 ? 4 : (i == 1 ? 6 : 8));
}
__host__ __device__ constexpr int long_rows_count(bool wide) { return wide ? 4 : 3; }
// Rows per lane of a strip-mined read of `len` bases: the value whose blocks waste the fewest
// padding rows (ties: the smaller). Blocks = ceil(len / (32 * R)). `wide`: the plain FP32 kind.
__host__ __device__ inline int long_rows(int len, bool wide) {
  int best = 8;
  long long best_rows = -1;
  for (int i = 0; i < long_rows_count(wide); ++i) {
    const int r = long_rows_value(i, wide);
    const long long rows = (static_cast<long long>(len) + 32 * r - 1) / (32 * r) * (32 * r);
    if (best_rows < 0 || rows < best_rows) {
      best_rows = rows;
      best = r;
    }
  }
  return best;
}
__host__ __device__ inline int long_blocks(int len, int rows) { return (len + 32 * rows - 1) / (32 * rows); }

// Recomputation queue bins: rows-per-lane 1..20 of single-block reads, then kRowBins + R for
// strip-mined reads and 2 * kRowBins + R for the pairs of byte-compared PD regions.
constexpr int kRowBins = 21;
constexpr int kQueueBins = 3 * kRowBins;
__host__ __device__ inline int queue_bin(int len, bool generic) {
  if (generic) return 2 * kRowBins + long_rows(len, false);
  if (len > kMaxBlockRead) return kRowBins + long_rows(len, false);
  int rows = (len + 30) / 31;
  if (rows > 8) rows = (rows + 1) & ~1;
  return rows;
}
__host__ __device__ inline int queue_bin_rows(int bin) { return bin % kRowBins; }

inline bool is_long(Kind k) { return static_cast<int>(k) >= static_cast<int>(Kind::kLongF32); }
inline bool is_pd(Kind k) {
  return k == Kind::kOneF32Pd || k == Kind::kOneF64Pd || k == Kind::kPackedF32Pd || k == Kind::kLongF32Pd ||
         k == Kind::kLongF64Pd || k == Kind::kGenericF32Pd || k == Kind::kGenericF64Pd;
}

// The PD instantiation a PD kind selects.
enum class PdForm : int { kOneF32 = 0, kOneF64 = 1, kPackedF32 = 2 };
inline PdForm pd_form(Kind k) {
  return k == Kind::kOneF64Pd ? PdForm::kOneF64 : (k == Kind::kPackedF32Pd ? PdForm::kPackedF32 : PdForm::kOneF32);
}

struct LaunchArgs {
  BatchView v;
  const Task* tasks;     // this launch's tasks
  int n_tasks;           // host-known count, or the capacity when `count` is set
  const int* count;      // device-side task count (recomputation queues), or nullptr
  int* task_counter;     // zeroed before the launch
  char* scratch;
  size_t scratch_stride; // bytes per warp
  int min_accept_plain;  // 1: results below the single-precision threshold are lost
  int only_lost;         // recomputation: a whole-program task writes only pairs whose result is NaN
};

// The pass between the first pass and the recomputation: queues lost pairs.
struct CollectArgs {
  BatchView v;
  Task* queue;           // recomputation queue: (read, distinct haplotype) FP64 tasks, and dense reads
  const int* queue_off;  // per rows-per-lane bin: first queue index (one past the last bin at the end)
  int* queue_tail;       // per bin: tasks queued
  int dense;             // 1 after an FP32 pass: a read lost against a third of its haplotypes or more
                         // is queued once, as a whole-program FP64 task (fgkl lib.rs:495-520)
};

// Rows per lane the instantiations cover.
int max_rows(Kind k);
// Bytes of per-warp scratch one task of this instantiation needs.
size_t scratch_bytes(Kind k, int rows, int max_slots, int max_nodes, int max_segs);
// Resident blocks per SM and threads per block of an instantiation.
void occupancy(Kind k, int rows, int* blocks_per_sm, int* threads_per_block, int warps_per_block = 4);
// Launches one persistent grid of `blocks` blocks.
cudaError_t launch(Kind k, int rows, int blocks, const LaunchArgs& args, cudaStream_t stream, int warps_per_block = 4);
// PD-HMM instantiations (pd_kernels.cu).
size_t pd_scratch_bytes(PdForm form, int rows, int max_slots, int max_segs);
void pd_occupancy(PdForm form, int rows, int* blocks_per_sm, int* threads_per_block, int warps_per_block = 4);
cudaError_t pd_launch(PdForm form, int rows, int blocks, const LaunchArgs& args, cudaStream_t stream, int warps_per_block = 4);
// Strip-mined kinds (is_long): per-warp scratch for haplotypes of at most `max_hap_len` bases (the
// bottom row a block hands to the next, plus the pair's result), occupancy and launch. The plain
// ones live in kernels.cu, the PD ones in pd_kernels.cu.
size_t long_scratch_bytes(Kind k, int rows, int max_hap_len);
void long_occupancy(Kind k, int rows, int* blocks_per_sm, int* threads_per_block);
cudaError_t long_launch(Kind k, int rows, int blocks, const LaunchArgs& args, cudaStream_t stream);
size_t pd_long_scratch_bytes(Kind k, int rows, int max_hap_len);
void pd_long_occupancy(Kind k, int rows, int* blocks_per_sm, int* threads_per_block);
cudaError_t pd_long_launch(Kind k, int rows, int blocks, const LaunchArgs& args, cudaStream_t stream);

// Launches the lost-pair collection over `n_regions` regions.
cudaError_t launch_collect(const CollectArgs& args, int n_regions, cudaStream_t stream);

// ---- allocation-free entry (file-scope device scratch; see capi.cpp) ----
constexpr size_t kMaxQualTable = 255;  // error-probability entries
constexpr size_t kM2MTable = 32640;    // match-to-match entries

// Per-device state of the allocation-free entry, filled once by noalloc_setup.
struct NoAllocDevice {
  bool ready = false;
  char* scratch = nullptr;  // the file-scope scratch array: header (pair counter), then per-warp slots
  double* err = nullptr;
  double* m2m = nullptr;
  uint8_t* codes = nullptr;
  size_t scratch_bytes = 0, header_bytes = 0, per_warp_bytes = 0;
  int blocks_per_sm[21] = {};
  int sms = 0;
};

// One call's caller-owned device arrays.
struct NoAllocCall {
  const uint8_t *bases, *quals, *ins, *del, *gcp;
  const int64_t* read_off;
  const uint8_t* hap_bases;
  const int64_t* hap_off;
  int n_reads, n_haps;
  double* out;
};

// Rows per lane for reads of at most `max_read_len` bases.
int noalloc_rows(int max_read_len);
// The current device's address of the file-scope scratch array (changes when the device's primary
// context is reset and recreated).
cudaError_t noalloc_scratch_address(char** scratch);
// Resolves the file-scope arrays of the current device and uploads the tables (synchronous).
cudaError_t noalloc_setup(NoAllocDevice* d, const double* err, size_t n_err, const double* m2m, size_t n_m2m,
                          const uint8_t codes[256]);
// Zeroes the pair counter and launches `blocks` blocks on `stream`; allocates nothing.
cudaError_t noalloc_launch(const NoAllocDevice& d, const NoAllocCall& c, int rows, int blocks, cudaStream_t stream);

}  // namespace fgkl
