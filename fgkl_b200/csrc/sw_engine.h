// Host side of the Smith-Waterman batch: validation, the persistent launch over the pairs (costliest
// first) and the copies of the CIGARs and offsets back. One engine owns a stream and grow-only
// device buffers, like the PairHMM engine.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "sw.cuh"

namespace fgkl {

struct SwBatch {
  int64_t num_pairs = 0;
  const uint8_t* ref = nullptr;
  const int64_t* ref_off = nullptr;  // num_pairs + 1
  const uint8_t* alt = nullptr;
  const int64_t* alt_off = nullptr;  // num_pairs + 1
};

struct SwScores {
  int32_t match, mismatch, open, extend;  // GATK's SWParameters (fgkl lib.rs:42-66)
};

// Elements a pair's CIGAR may need: every element covers at least one reference or alternate base,
// and at most one clip or trailing gap covers none of the aligned ones.
inline int64_t sw_cigar_slot(int64_t ref_len, int64_t alt_len) { return ref_len + alt_len + 2; }

class SwEngine {
 public:
  explicit SwEngine(int device, cudaStream_t stream = nullptr);
  ~SwEngine();
  SwEngine(const SwEngine&) = delete;
  SwEngine& operator=(const SwEngine&) = delete;

  // Aligns every pair (host arrays in and out, synchronous). Pair k's elements land in
  // cigar[slot_k ...], slot_k = Σ_{j<k} sw_cigar_slot(ref_j, alt_j), `counts[k]` of them; cigar_len
  // must reach the sum over all pairs. Returns 0 or a negative FGKL_E_* code (message in error()).
  int align(const SwBatch& in, const SwScores& s, int strategy, uint32_t* cigar, int64_t cigar_len, int32_t* counts,
            int32_t* offsets);
  const std::string& error() const { return error_; }
  // Duration of the last align call's fill-and-traceback launch (CUDA events on the engine's stream),
  // or -1 before the first.
  float last_kernel_ms() const { return kernel_ms_; }

 private:
  int fail(int code, const std::string& msg);
  int check(cudaError_t e, const char* what);
  template <class T>
  T* grow(T*& p, size_t& cap, size_t n);

  int device_ = 0, sms_ = 0;
  cudaStream_t stream_ = nullptr;
  bool own_stream_ = false;
  std::string error_;
  uint8_t* d_seq_ = nullptr;    // references | alternates
  size_t cap_seq_ = 0;
  int64_t* d_idx_ = nullptr;    // ref offsets | alt offsets | cigar slots
  size_t cap_idx_ = 0;
  int32_t* d_small_ = nullptr;  // order | counts | offsets | counter
  size_t cap_small_ = 0;
  uint32_t* d_cigar_ = nullptr;  // slot layout | packed elements
  size_t cap_cigar_ = 0;
  char* d_scratch_ = nullptr;
  size_t cap_scratch_ = 0;
  std::vector<uint32_t> packed_;  // the batch's CIGAR elements, pair after pair
  cudaEvent_t ev_[2] = {nullptr, nullptr};  // around the fill-and-traceback launch
  float kernel_ms_ = -1.f;
};

}  // namespace fgkl
