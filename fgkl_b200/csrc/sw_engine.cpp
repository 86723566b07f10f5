#include "sw_engine.h"

#include <algorithm>
#include <numeric>
#include <vector>

#include "../../include/fgkl_b200.h"
#include "engine.h"

namespace fgkl {

namespace {
constexpr int kWarps = 4;                           // warps per block of the kernel
constexpr size_t kScratchBudget = size_t{8} << 30;  // per-warp traceback scratch of one launch
}  // namespace

SwEngine::SwEngine(int device, cudaStream_t stream) : device_(device), stream_(stream) {
  DeviceGuard device_guard(device_);
  cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_);
  if (!stream_) {
    cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    own_stream_ = true;
  }
}

SwEngine::~SwEngine() {
  DeviceGuard device_guard(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  cudaFree(d_seq_);
  cudaFree(d_idx_);
  cudaFree(d_small_);
  cudaFree(d_cigar_);
  cudaFree(d_scratch_);
  for (cudaEvent_t e : ev_)
    if (e) cudaEventDestroy(e);
  if (own_stream_) cudaStreamDestroy(stream_);
}

int SwEngine::fail(int code, const std::string& msg) {
  error_ = msg;
  return code;
}

int SwEngine::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FGKL_OK;
  return fail(FGKL_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T* SwEngine::grow(T*& p, size_t& cap, size_t n) {
  const size_t bytes = std::max<size_t>(n * sizeof(T), 256);
  if (over_allocation_limit(bytes)) return nullptr;  // the buffer held so far is kept
  if (bytes > cap) {
    const size_t want = cap > 0 ? std::max(bytes, cap + cap / 2) : bytes;
    cudaFree(p);
    p = nullptr;
    if (device_alloc(reinterpret_cast<void**>(&p), want) == cudaSuccess) {
      cap = want;
    } else if (want > bytes && (cudaGetLastError(), device_alloc(reinterpret_cast<void**>(&p), bytes) == cudaSuccess)) {
      cap = bytes;
    } else {
      cudaGetLastError();
      cap = 0;
      p = nullptr;
      return nullptr;
    }
  }
  return p;
}

int SwEngine::align(const SwBatch& in, const SwScores& s, int strategy, uint32_t* cigar, int64_t cigar_len, int32_t* counts,
                    int32_t* offsets) {
  DeviceGuard device_guard(device_);
  error_.clear();
  kernel_ms_ = -1.f;
  const int64_t P = in.num_pairs;
  if (P < 0) return fail(FGKL_E_INVALID_ARGUMENT, "negative pair count");
  if (strategy < kSwSoftClip || strategy > kSwIgnore) return fail(FGKL_E_INVALID_ARGUMENT, "unknown overhang strategy code " + std::to_string(strategy));
  if (P == 0) return FGKL_OK;
  if (P > INT32_MAX) return fail(FGKL_E_INVALID_ARGUMENT, "at most 2^31 - 1 pairs per call; split the batch");
  if (!in.ref || !in.ref_off || !in.alt || !in.alt_off || !cigar || !counts || !offsets)
    return fail(FGKL_E_INVALID_ARGUMENT, "null argument");
  if (in.ref_off[0] != 0 || in.alt_off[0] != 0) return fail(FGKL_E_BAD_OFFSETS, "offset tables must start at zero");
  // Slots, sizes and costs (lib.rs: both sequences must be non-empty).
  std::vector<int64_t> slot(static_cast<size_t>(P) + 1, 0);
  size_t stride = 256;
  std::vector<std::pair<int64_t, int32_t>> cost(static_cast<size_t>(P));
  for (int64_t k = 0; k < P; ++k) {
    const int64_t n = in.ref_off[k + 1] - in.ref_off[k], m = in.alt_off[k + 1] - in.alt_off[k];
    if (n < 0 || m < 0) return fail(FGKL_E_BAD_OFFSETS, "offset tables must be non-decreasing");
    if (n == 0 || m == 0) return fail(FGKL_E_EMPTY_SEQUENCE, "pair " + std::to_string(k) + " has an empty sequence");
    if (n > (int64_t{1} << 28) || m > (int64_t{1} << 28)) return fail(FGKL_E_UNSUPPORTED, "sequences of at most 2^28 bases");
    slot[k + 1] = slot[k] + sw_cigar_slot(n, m);
    stride = std::max(stride, sw_scratch_bytes(n, m));
    cost[k] = {n * m, static_cast<int32_t>(k)};
  }
  if (cigar_len < slot[P])
    return fail(FGKL_E_OUTPUT_LENGTH, "the CIGAR array holds " + std::to_string(cigar_len) + " elements; the batch needs " +
                                          std::to_string(slot[P]));
  std::stable_sort(cost.begin(), cost.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  std::vector<int32_t> order(static_cast<size_t>(P));
  for (int64_t k = 0; k < P; ++k) order[k] = cost[k].second;
  stride = (stride + 255) / 256 * 256;

  int per_sm = 0, threads = 0;
  sw_occupancy(&per_sm, &threads);
  if (per_sm <= 0) return fail(FGKL_E_CUDA, "Smith-Waterman kernel unavailable on this device");
  int64_t blocks = std::min<int64_t>((P + kWarps - 1) / kWarps, static_cast<int64_t>(per_sm) * sms_);
  blocks = std::max<int64_t>(1, std::min<int64_t>(blocks, static_cast<int64_t>(kScratchBudget / (kWarps * stride))));

  const int64_t ref_bytes = in.ref_off[P], alt_bytes = in.alt_off[P];
  if (!grow(d_seq_, cap_seq_, static_cast<size_t>(ref_bytes + alt_bytes) + 16) || !grow(d_idx_, cap_idx_, 3 * static_cast<size_t>(P + 1)) ||
      !grow(d_small_, cap_small_, 3 * static_cast<size_t>(P) + 1) || !grow(d_cigar_, cap_cigar_, 2 * static_cast<size_t>(slot[P])) ||
      !grow(d_scratch_, cap_scratch_, static_cast<size_t>(blocks) * kWarps * stride))
    return fail(FGKL_E_OUT_OF_MEMORY, "device allocation failed");
  int rc;
  auto up = [&](void* dst, const void* src, size_t bytes, const char* what) {
    return bytes ? check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), what) : FGKL_OK;
  };
  int64_t* d_ref_off = d_idx_;
  int64_t* d_alt_off = d_idx_ + (P + 1);
  int64_t* d_slot = d_idx_ + 2 * (P + 1);
  int32_t* d_order = d_small_;
  int32_t* d_counts = d_small_ + P;
  int32_t* d_offsets = d_small_ + 2 * P;
  int* d_counter = d_small_ + 3 * P;
  if ((rc = up(d_seq_, in.ref, static_cast<size_t>(ref_bytes), "upload references")) ||
      (rc = up(d_seq_ + ref_bytes, in.alt, static_cast<size_t>(alt_bytes), "upload alternates")) ||
      (rc = up(d_ref_off, in.ref_off, 8 * static_cast<size_t>(P + 1), "upload offsets")) ||
      (rc = up(d_alt_off, in.alt_off, 8 * static_cast<size_t>(P + 1), "upload offsets")) ||
      (rc = up(d_slot, slot.data(), 8 * static_cast<size_t>(P + 1), "upload slots")) ||
      (rc = up(d_order, order.data(), 4 * static_cast<size_t>(P), "upload order")))
    return rc;
  if ((rc = check(cudaMemsetAsync(d_counter, 0, sizeof(int), stream_), "reset counter"))) return rc;
  SwArgs a{};
  a.ref = d_seq_;
  a.ref_off = d_ref_off;
  a.alt = d_seq_ + ref_bytes;
  a.alt_off = d_alt_off;
  a.order = d_order;
  a.n_pairs = static_cast<int>(P);
  a.match = s.match;
  a.mismatch = s.mismatch;
  a.open = s.open;
  a.extend = s.extend;
  a.strategy = strategy;
  a.scratch = d_scratch_;
  a.stride = stride;
  a.cigar = d_cigar_;
  a.cigar_slot = d_slot;
  a.count = d_counts;
  a.offset = d_offsets;
  a.counter = d_counter;
  if (!ev_[0] || !ev_[1]) {
    for (cudaEvent_t& e : ev_)
      if (!e && cudaEventCreate(&e) != cudaSuccess) e = nullptr;
    if (!ev_[0] || !ev_[1]) return fail(FGKL_E_CUDA, "event creation failed");
  }
  if ((rc = check(cudaEventRecord(ev_[0], stream_), "event")) ||
      (rc = check(sw_launch(static_cast<int>(blocks), a, stream_), "Smith-Waterman launch")) ||
      (rc = check(cudaEventRecord(ev_[1], stream_), "event")))
    return rc;
  // Only the elements produced cross to the host: packed pair after pair on the device, then
  // scattered into the caller's slots (a CIGAR is a few elements; its slot holds ref + alt + 2).
  uint32_t* d_packed = d_cigar_ + slot[P];
  if ((rc = check(sw_compact(d_cigar_, d_slot, d_counts, static_cast<int>(P), d_packed, stream_), "CIGAR packing")) ||
      (rc = check(cudaMemcpyAsync(counts, d_counts, 4 * static_cast<size_t>(P), cudaMemcpyDeviceToHost, stream_), "download counts")) ||
      (rc = check(cudaMemcpyAsync(offsets, d_offsets, 4 * static_cast<size_t>(P), cudaMemcpyDeviceToHost, stream_), "download offsets")) ||
      (rc = check(cudaStreamSynchronize(stream_), "Smith-Waterman kernel")))
    return rc;
  // Measurement only: a failed query leaves the time unknown (-1) and the alignment stands.
  if (cudaEventElapsedTime(&kernel_ms_, ev_[0], ev_[1]) != cudaSuccess) {
    kernel_ms_ = -1.f;
    cudaGetLastError();
  }
  int64_t total = 0;
  for (int64_t k = 0; k < P; ++k) {
    if (counts[k] < 0 || counts[k] > sw_cigar_slot(in.ref_off[k + 1] - in.ref_off[k], in.alt_off[k + 1] - in.alt_off[k]))
      return fail(FGKL_E_CUDA, "Smith-Waterman kernel returned an impossible CIGAR length");
    total += counts[k];
  }
  packed_.resize(static_cast<size_t>(total));
  if (total > 0 &&
      ((rc = check(cudaMemcpyAsync(packed_.data(), d_packed, 4 * static_cast<size_t>(total), cudaMemcpyDeviceToHost, stream_),
                   "download CIGARs")) ||
       (rc = check(cudaStreamSynchronize(stream_), "download CIGARs"))))
    return rc;
  for (int64_t k = 0, pos = 0; k < P; ++k) {
    std::copy(packed_.begin() + pos, packed_.begin() + pos + counts[k], cigar + slot[k]);
    pos += counts[k];
  }
  return FGKL_OK;
}

}  // namespace fgkl
