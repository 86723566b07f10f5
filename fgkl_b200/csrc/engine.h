// Host orchestration of the sm_100a PairHMM kernels: plans a batch of regions, uploads it, runs the
// first pass and the double-precision recomputation, and brings the results back. One Engine owns a
// device stream and grow-only device buffers (fgkl keeps per-thread workspaces the same way,
// kernel.rs:144-163).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "program.h"

namespace fgkl {

// Failure injection (fgkl_set_allocation_limit): a call that needs a device or page-locked host
// buffer larger than this many bytes fails as if out of memory, whether or not a buffer that large
// is already held (which is kept); 0 = no limit.
int64_t allocation_limit();
int64_t set_allocation_limit(int64_t bytes);
bool over_allocation_limit(size_t bytes);
// cudaMalloc / cudaMallocHost under that limit.
cudaError_t device_alloc(void** p, size_t bytes);
cudaError_t pinned_alloc(void** p, size_t bytes);

// Makes `device` current for its scope and gives the calling thread its own current device back at
// the end, so an engine's calls leave the caller's device as they found it.
class DeviceGuard {
 public:
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&prev_) != cudaSuccess) {
      cudaGetLastError();
      prev_ = -1;
    }
    if (prev_ != device) cudaSetDevice(device);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev_ >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev_) cudaSetDevice(prev_);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;

 private:
  int prev_ = -1;
};

struct EngineConfig {
  bool double_precision = false;  // Precision::Double (lib.rs:72-77)
  bool double_fallback = true;    // recompute lost pairs (lib.rs:218-222)
  bool share_suffixes = true;     // suffix sharing (lib.rs:223-226)
};

// A batch of regions in host memory (reads and haplotypes concatenated, region sizes apart).
struct BatchInput {
  int32_t num_regions = 0;
  const int32_t* region_reads = nullptr;
  const int32_t* region_haps = nullptr;
  const uint8_t *bases = nullptr, *quals = nullptr, *ins = nullptr, *del = nullptr, *gcp = nullptr;
  const int64_t* read_off = nullptr;  // total_reads + 1
  const uint8_t* hap_bases = nullptr;
  const uint8_t* hap_flags = nullptr; // PD-HMM: per-base flags (same layout as hap_bases); nullptr = plain
  const int64_t* hap_off = nullptr;   // total_haps + 1
};

struct BatchStats {
  uint64_t fallback_pairs = 0;
  uint64_t rescue_reads = 0;
  uint64_t nominal_cells = 0;       // Σ per region of Σ read lengths x Σ haplotype lengths
  uint64_t computed_cells = 0;      // forward + backward cells of the first pass
  uint64_t forward_cells = 0;
  uint64_t backward_cells = 0;
  uint64_t prefix_only_cells = 0;   // forward cells prefix sharing alone would compute
  uint64_t kernel_launches = 0;     // launches issued by the last run()
  double host_plan_ms = 0;          // sorting, planning and program emission
  double host_pack_ms = 0;          // concatenation into pinned staging
  double host_upload_ms = 0;        // enqueueing the uploads
  double host_fetch_ms = 0;         // waiting for the kernels and copying results out
};

// Per region, the DP cells a batched run of `in` computes (forward and backward, as the planner
// emits them): the cost to balance when regions are split across devices. Host only.
int plan_region_cells(const BatchInput& in, const EngineConfig& cfg, uint64_t* cells, std::string* error);

class Engine {
 public:
  explicit Engine(int device, cudaStream_t stream = nullptr);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // Plans `in` and uploads it on the engine's copy stream; returns 0 or a negative FGKL_E_* code
  // (message in error()). Waits only for this engine's own earlier batch, never for other work on
  // the compute stream, so engines sharing one compute stream can plan one batch while another runs.
  int prepare(const BatchInput& in, const EngineConfig& cfg);
  // Makes the compute stream wait for the prepared batch's uploads. Called before run() or before
  // launching a graph captured from run(), outside any capture.
  int begin_run();
  // Enqueues the first pass and the recomputation on the stream (no host synchronisation).
  int run();
  // Marks the end of the batch's kernels on the compute stream; called after run() or the graph.
  int end_run();
  // Copies the results (and counters) back on the copy stream once the batch's kernels are done,
  // and waits for that copy alone.
  int fetch(double* out, int64_t out_len, BatchStats* stats);
  // prepare + run + fetch.
  int compute(const BatchInput& in, const EngineConfig& cfg, double* out, int64_t out_len, BatchStats* stats);

  const std::string& error() const { return error_; }
  cudaStream_t stream() const { return stream_; }
  int64_t output_len() const { return out_len_; }
  // Host-side planning statistics of the prepared batch.
  const BatchStats& planned() const { return planned_; }
  // Device pointer to the output, for callers that keep results on the device.
  const double* device_output() const { return d_out_; }

  // Per-launch timing: with profiling on, run() records CUDA events around every launch on the
  // stream it is issued to (so run() must not be captured); bin_profile() waits and reads them.
  struct BinProfile {
    int kind, rows, n_tasks, blocks;
    int rescue;
    uint64_t fwd_cells, bwd_cells;
    float ms;
  };
  void set_profiling(bool on) { profile_ = on; }
  bool profiling() const { return profile_; }
  int bin_profile(std::vector<BinProfile>* out);

  // Launch configuration of the batched form: how many streams the launches of one pass spread
  // over (1: one after another; more: bins overlap, the largest first), each first-pass persistent
  // grid as a percentage of the resident-block limit, how many reads an FP32 PD-HMM warp carries
  // (two in FP32x2 at 8 warps per SM, or one at 12), and the first pass's tile shape: rows per lane
  // of the plain FP32 reads (the fewest that hold the read, or the next the kernels instantiate)
  // and warps per block of the FP32 first-pass kernels. None changes a result bit. Applies from the
  // next prepare().
  struct Tuning {
    int streams = 8;
    int grid_percent = 100;
    int reads_per_warp = 2;   // FP32 PD-HMM reads of at most 248 bases: 2 (FP32x2 pairs) or 1
    int rows_extra = 0;       // 1: plain FP32 reads one rows-per-lane step above the fewest
    int warps_per_block = 4;  // FP32 first-pass kernels: 1, 2 or 4
  };
  void set_tuning(const Tuning& t);
  const Tuning& tuning() const { return tuning_; }
  // Times the prepared batch's kernels (direct launches on the stream, after one untimed run):
  // the median of `repeats` runs, in milliseconds. Host-synchronous.
  int time_run(int repeats, double* ms);

 private:
  struct Bin {
    Kind kind;
    int rows;
    int task_off;  // into the device task array
    int n_tasks;
    int blocks;
    size_t stride;       // scratch bytes per warp
    size_t scratch_off;  // this bin's slice of the scratch
    uint64_t fwd_cells = 0, bwd_cells = 0;  // DP cells its tasks compute (first pass)
    int queue_bin = 0;   // recomputation bins: the queue bin (queue_bin) the tasks come from
    int warps = 4;       // warps per block
  };
  static constexpr int kAuxStreams = 8;
  Tuning tuning_;
  template <class T>
  T* grow(T*& ptr, size_t& cap, size_t n);
  int fail(int code, const std::string& msg);
  int check(cudaError_t e, const char* what);

  int device_ = 0;
  int sms_ = 0;
  cudaStream_t stream_ = nullptr;  // compute: the batch's kernels (may be shared with other engines)
  bool own_stream_ = false;
  cudaStream_t copy_ = nullptr;    // this engine's uploads and downloads
  cudaEvent_t uploaded_ = nullptr;  // after the last batch's uploads (copy stream)
  cudaEvent_t computed_ = nullptr;  // after the last batch's kernels (compute stream)
  cudaEvent_t fetched_ = nullptr;   // after the last batch's downloads (copy stream)
  cudaStream_t aux_[kAuxStreams] = {};
  cudaEvent_t join_[kAuxStreams] = {};
  cudaEvent_t fork_ = nullptr;
  std::string error_;
  EngineConfig cfg_;
  BatchStats planned_;

  // Device buffers (grow-only).
  uint8_t* d_reads_ = nullptr;
  size_t cap_reads_ = 0;
  int64_t* d_read_off_ = nullptr;
  size_t cap_read_off_ = 0;
  uint8_t* d_plan_ = nullptr;  // regions, haps, stream, segs, slot/node lists, code tables
  size_t cap_plan_ = 0;
  Task* d_tasks_ = nullptr;
  size_t cap_tasks_ = 0;
  Task* d_queue_ = nullptr;
  size_t cap_queue_ = 0;
  int* d_small_ = nullptr;  // task counters, queue offsets and tails
  size_t cap_small_ = 0;
  double* d_out_ = nullptr;
  size_t cap_out_ = 0;
  Counters* d_counters_ = nullptr;
  char* d_scratch_ = nullptr;
  size_t cap_scratch_ = 0;
  double* d_err_ = nullptr;
  double* d_m2m_ = nullptr;

  // Pinned host staging.
  uint8_t* h_stage_ = nullptr;
  size_t cap_stage_ = 0;
  uint8_t* h_reads_ = nullptr;  // pinned staging of the five read arrays, filled while planning runs
  size_t cap_h_reads_ = 0;
  size_t out_stage_ = 0;  // results and counters come back here

  // Prepared batch.
  BatchView view_{};
  std::vector<Bin> bins_, rescue_bins_;
  int64_t out_len_ = 0;
  int n_regions_ = 0;
  bool profile_ = false;
  std::vector<cudaEvent_t> ev_;  // begin/end per launch of the last profiled run
  int n_small_ = 0;
};

}  // namespace fgkl
