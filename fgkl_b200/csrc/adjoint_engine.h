// Host side of the adjoint path: uploads a batch of regions with per-read-position continuous
// parameters, runs the FP32 adjoint kernels (FP64 for reads FP32 loses, or for everything in double
// precision) and brings back log10 likelihoods and per-position gradients.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "adjoint.cuh"

namespace fgkl {

struct AdjointInput {
  int32_t num_regions = 0;
  const int32_t* region_reads = nullptr;
  const int32_t* region_haps = nullptr;
  const uint8_t* bases = nullptr;
  const int64_t* read_off = nullptr;  // total_reads + 1
  const double* d_ins = nullptr;      // per read position
  const double* d_del = nullptr;
  const double* eps = nullptr;
  const double* err = nullptr;
  const uint8_t* hap_bases = nullptr;
  const int64_t* hap_off = nullptr;   // total_haps + 1
};

class AdjointEngine {
 public:
  AdjointEngine(int device, cudaStream_t stream);
  ~AdjointEngine();
  AdjointEngine(const AdjointEngine&) = delete;
  AdjointEngine& operator=(const AdjointEngine&) = delete;

  int prepare(const AdjointInput& in, bool double_precision);
  int run();
  // Likelihoods (Σ reads x haplotypes) and the four gradient arrays (Σ read lengths).
  int fetch(double* out, int64_t out_len, double* g_ins, double* g_del, double* g_eps, double* g_err, int64_t grad_len,
            uint64_t* fp64_reads);
  const std::string& error() const { return error_; }
  int64_t output_len() const { return out_len_; }
  int64_t grad_len() const { return grad_len_; }
  uint64_t launches() const { return launches_; }

 private:
  struct Bin {
    bool dbl;
    int rows;
    int task_off;
    int n_tasks;
    int blocks;
    size_t stride;
  };
  int fail(int code, const std::string& msg);
  int check(cudaError_t e, const char* what);
  template <class T>
  T* grow(T*& p, size_t& cap, size_t n);

  int device_ = 0, sms_ = 0;
  cudaStream_t stream_ = nullptr;
  std::string error_;
  bool dbl_ = false;
  int64_t out_len_ = 0, grad_len_ = 0;
  uint64_t launches_ = 0;
  std::vector<Bin> bins_, rescue_;
  AdjView view_{};
  // Device buffers (grow-only).
  uint8_t* d_bytes_ = nullptr;  // bases | hap bases
  size_t cap_bytes_ = 0;
  double* d_params_ = nullptr;  // d_ins | d_del | eps | err
  size_t cap_params_ = 0;
  int64_t* d_off_ = nullptr;    // read offsets | haplotype offsets | region output offsets
  size_t cap_off_ = 0;
  int32_t* d_idx_ = nullptr;    // read regions | region first hap | count | first read | tasks | queue
  size_t cap_idx_ = 0;
  double* d_out_ = nullptr;     // likelihoods | 4 gradient arrays
  size_t cap_out_ = 0;
  int* d_small_ = nullptr;      // task counters | queue offsets | queue tails
  size_t cap_small_ = 0;
  unsigned long long* d_lost_ = nullptr;
  char* d_scratch_ = nullptr;
  size_t cap_scratch_ = 0;
  int32_t* tasks_ = nullptr;  // per bin, inside d_idx_
  int32_t* queue_ = nullptr;  // FP64 recomputation queue, inside d_idx_
  int n_small_ = 0;
};

}  // namespace fgkl
