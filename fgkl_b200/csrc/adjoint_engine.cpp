#include "adjoint_engine.h"

#include <algorithm>
#include <cstring>
#include <map>

#include "../../include/fgkl_b200.h"
#include "engine.h"

namespace fgkl {

namespace {

constexpr int kWarps = 4;                             // warps per block of the adjoint kernels
constexpr size_t kScratchBudget = size_t{8} << 30;    // per-warp checkpoints of one launch, at most 8 GiB

size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

}  // namespace

AdjointEngine::AdjointEngine(int device, cudaStream_t stream) : device_(device), stream_(stream) {
  DeviceGuard device_guard(device_);
  cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_);
  cudaMalloc(&d_lost_, sizeof(unsigned long long));
}

AdjointEngine::~AdjointEngine() {
  DeviceGuard device_guard(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  cudaFree(d_bytes_);
  cudaFree(d_params_);
  cudaFree(d_off_);
  cudaFree(d_idx_);
  cudaFree(d_out_);
  cudaFree(d_small_);
  cudaFree(d_lost_);
  cudaFree(d_scratch_);
}

int AdjointEngine::fail(int code, const std::string& msg) {
  error_ = msg;
  return code;
}

int AdjointEngine::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FGKL_OK;
  return fail(FGKL_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T* AdjointEngine::grow(T*& p, size_t& cap, size_t n) {
  const size_t bytes = std::max<size_t>(n * sizeof(T), 256);
  if (over_allocation_limit(bytes)) return nullptr;  // the buffer held so far is kept
  if (bytes > cap) {
    // Half as much again as the old size: a caller whose batches vary in size stops reallocating
    // after a few calls (cudaFree waits for the whole device, other callers' streams included).
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

int AdjointEngine::prepare(const AdjointInput& in, bool double_precision) {
  DeviceGuard device_guard(device_);
  error_.clear();
  dbl_ = double_precision;
  bins_.clear();
  rescue_.clear();
  const int N = in.num_regions;
  if (N < 0) return fail(FGKL_E_INVALID_ARGUMENT, "negative region count");
  if (N > 0 && (!in.region_reads || !in.region_haps || !in.read_off || !in.hap_off))
    return fail(FGKL_E_INVALID_ARGUMENT, "null argument");
  std::vector<int64_t> first_read(N + 1, 0), first_hap(N + 1, 0), out_off(N + 1, 0);
  for (int g = 0; g < N; ++g) {
    if (in.region_reads[g] < 0 || in.region_haps[g] < 0) return fail(FGKL_E_INVALID_ARGUMENT, "negative region size");
    first_read[g + 1] = first_read[g] + in.region_reads[g];
    first_hap[g + 1] = first_hap[g] + in.region_haps[g];
    out_off[g + 1] = out_off[g] + static_cast<int64_t>(in.region_reads[g]) * in.region_haps[g];
  }
  const int64_t total_reads = first_read[N], total_haps = first_hap[N];
  if (total_reads > INT32_MAX || total_haps > INT32_MAX) return fail(FGKL_E_INVALID_ARGUMENT, "batch too large; split it");
  out_len_ = out_off[N];
  grad_len_ = total_reads > 0 ? in.read_off[total_reads] : 0;
  const int64_t hap_bytes = total_haps > 0 ? in.hap_off[total_haps] : 0;
  if (grad_len_ > 0 && (!in.bases || !in.d_ins || !in.d_del || !in.eps || !in.err))
    return fail(FGKL_E_INVALID_ARGUMENT, "null read array");
  if (hap_bytes > 0 && !in.hap_bases) return fail(FGKL_E_INVALID_ARGUMENT, "null haplotype array");
  int max_hap = 1;
  for (int64_t r = 0; r < total_reads; ++r) {
    const int64_t len = in.read_off[r + 1] - in.read_off[r];
    if (len <= 0) return fail(FGKL_E_EMPTY_READ, "read " + std::to_string(r) + " has no bases");
    if (len > (int64_t{1} << 24)) return fail(FGKL_E_UNSUPPORTED, "read longer than 2^24 bases");
  }
  for (int64_t h = 0; h < total_haps; ++h) {
    const int64_t len = in.hap_off[h + 1] - in.hap_off[h];
    if (len <= 0) return fail(FGKL_E_EMPTY_HAPLOTYPE, "haplotype " + std::to_string(h) + " has no bases");
    if (len > (int64_t{1} << 24)) return fail(FGKL_E_UNSUPPORTED, "haplotype longer than 2^24 bases");
    max_hap = std::max<int>(max_hap, static_cast<int>(len));
  }

  // Tasks: one per read, binned by rows per lane, costliest first. Each bin's per-warp scratch is
  // what its largest pair needs (adj_scratch_bytes: the read's length and its region's longest
  // haplotype).
  std::vector<int32_t> read_region(static_cast<size_t>(total_reads));
  std::map<int, std::vector<std::pair<int64_t, int32_t>>> by_rows;
  std::vector<int> per_rows(kAdjRowBins, 0);
  std::vector<size_t> need(kAdjRowBins, 0);
  for (int g = 0; g < N; ++g) {
    const int64_t hap_sum = total_haps > 0 ? in.hap_off[first_hap[g + 1]] - in.hap_off[first_hap[g]] : 0;
    int longest = 1;
    for (int64_t h = first_hap[g]; h < first_hap[g + 1]; ++h)
      longest = std::max(longest, static_cast<int>(in.hap_off[h + 1] - in.hap_off[h]));
    for (int64_t r = first_read[g]; r < first_read[g + 1]; ++r) {
      read_region[r] = g;
      if (in.region_haps[g] == 0) continue;
      const int len = static_cast<int>(in.read_off[r + 1] - in.read_off[r]);
      const int rows = adj_rows(len);
      by_rows[rows].push_back({static_cast<int64_t>(rows) * adj_row_blocks(len, rows) * hap_sum, static_cast<int32_t>(r)});
      per_rows[rows]++;
      need[rows] = std::max(need[rows], std::max(adj_scratch_bytes(dbl_, rows, len, longest), adj_scratch_bytes(true, rows, len, longest)));
    }
  }
  std::vector<int32_t> tasks;
  for (auto& [rows, list] : by_rows) {
    std::stable_sort(list.begin(), list.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    Bin b{dbl_, rows, static_cast<int>(tasks.size()), static_cast<int>(list.size()), 0, 0};
    for (auto& e : list) tasks.push_back(e.second);
    bins_.push_back(b);
  }
  std::vector<int> queue_off(kAdjRowBins + 1, 0);
  for (int r = 0; r < kAdjRowBins; ++r) queue_off[r + 1] = queue_off[r] + (dbl_ ? 0 : per_rows[r]);
  if (!dbl_)
    for (int r = 1; r < kAdjRowBins; ++r)
      if (per_rows[r]) rescue_.push_back(Bin{true, r, queue_off[r], per_rows[r], 0, 0});
  // Bins run one after another, so they share the scratch; a bin's grid shrinks only when its warps'
  // scratch would exceed the budget (very long pairs).
  size_t scratch = 256;
  for (auto* list : {&bins_, &rescue_})
    for (Bin& b : *list) {
      int per_sm = 0, threads = 0;
      adj_occupancy(b.dbl, b.rows, &per_sm, &threads);
      if (per_sm <= 0) return fail(FGKL_E_CUDA, "adjoint kernel unavailable on this device");
      const int64_t want = std::min<int64_t>((b.n_tasks + kWarps - 1) / kWarps, static_cast<int64_t>(per_sm) * sms_);
      b.stride = align_up(std::max<size_t>(need[b.rows], 256));
      const int64_t by_budget = static_cast<int64_t>(kScratchBudget / (kWarps * b.stride));
      b.blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, by_budget)));
      scratch = std::max(scratch, static_cast<size_t>(b.blocks) * kWarps * b.stride);
    }

  // Device buffers.
  const size_t n_bytes = static_cast<size_t>(grad_len_) + static_cast<size_t>(hap_bytes) + 16;
  const size_t n_off = static_cast<size_t>(total_reads + 1 + total_haps + 1 + N);
  const size_t n_idx = static_cast<size_t>(total_reads + 3 * N) + tasks.size() + static_cast<size_t>(queue_off[kAdjRowBins]);
  n_small_ = static_cast<int>(bins_.size() + rescue_.size()) + 2 * kAdjRowBins + 1;
  if (!grow(d_bytes_, cap_bytes_, n_bytes) || !grow(d_params_, cap_params_, 4 * static_cast<size_t>(grad_len_) + 1) ||
      !grow(d_off_, cap_off_, n_off + 1) || !grow(d_idx_, cap_idx_, n_idx + 1) ||
      !grow(d_out_, cap_out_, static_cast<size_t>(out_len_) + 4 * static_cast<size_t>(grad_len_) + 1) ||
      !grow(d_small_, cap_small_, static_cast<size_t>(n_small_)) || !grow(d_scratch_, cap_scratch_, scratch))
    return fail(FGKL_E_OUT_OF_MEMORY, "device allocation failed");

  std::vector<int32_t> region_hap(N), region_nhap(N), region_read(N);
  for (int g = 0; g < N; ++g) {
    region_hap[g] = static_cast<int32_t>(first_hap[g]);
    region_nhap[g] = in.region_haps[g];
    region_read[g] = static_cast<int32_t>(first_read[g]);
  }
  int rc;
  auto up = [&](void* dst, const void* src, size_t bytes, const char* what) {
    if (bytes == 0) return FGKL_OK;
    return check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), what);
  };
  uint8_t* d_bases = d_bytes_;
  uint8_t* d_haps = d_bytes_ + grad_len_;
  const size_t G = static_cast<size_t>(grad_len_);
  if ((rc = up(d_bases, in.bases, G, "upload bases")) || (rc = up(d_haps, in.hap_bases, static_cast<size_t>(hap_bytes), "upload haplotypes")) ||
      (rc = up(d_params_, in.d_ins, G * 8, "upload parameters")) || (rc = up(d_params_ + G, in.d_del, G * 8, "upload parameters")) ||
      (rc = up(d_params_ + 2 * G, in.eps, G * 8, "upload parameters")) ||
      (rc = up(d_params_ + 3 * G, in.err, G * 8, "upload parameters")))
    return rc;
  int64_t* d_read_off = d_off_;
  int64_t* d_hap_off = d_off_ + total_reads + 1;
  int64_t* d_region_out = d_hap_off + total_haps + 1;
  if ((rc = up(d_read_off, in.read_off, (total_reads + 1) * 8, "upload offsets")) ||
      (rc = up(d_hap_off, in.hap_off, (total_haps + 1) * 8, "upload offsets")) ||
      (rc = up(d_region_out, out_off.data(), static_cast<size_t>(N) * 8, "upload offsets")))
    return rc;
  int32_t* d_read_region = d_idx_;
  int32_t* d_region_hap = d_read_region + total_reads;
  int32_t* d_region_nhap = d_region_hap + N;
  int32_t* d_region_read = d_region_nhap + N;
  int32_t* d_tasks = d_region_read + N;
  tasks_ = d_tasks;
  queue_ = d_tasks + tasks.size();
  if ((rc = up(d_read_region, read_region.data(), read_region.size() * 4, "upload regions")) ||
      (rc = up(d_region_hap, region_hap.data(), static_cast<size_t>(N) * 4, "upload regions")) ||
      (rc = up(d_region_nhap, region_nhap.data(), static_cast<size_t>(N) * 4, "upload regions")) ||
      (rc = up(d_region_read, region_read.data(), static_cast<size_t>(N) * 4, "upload regions")) ||
      (rc = up(d_tasks, tasks.data(), tasks.size() * 4, "upload tasks")) ||
      (rc = up(d_small_ + (n_small_ - 2 * kAdjRowBins - 1), queue_off.data(), queue_off.size() * 4, "upload queue offsets")))
    return rc;
  // The host vectors above go out of scope: wait for the copies.
  if ((rc = check(cudaStreamSynchronize(stream_), "upload"))) return rc;

  view_ = AdjView{};
  view_.bases = d_bases;
  view_.read_off = d_read_off;
  view_.d_ins = d_params_;
  view_.d_del = d_params_ + G;
  view_.eps = d_params_ + 2 * G;
  view_.err = d_params_ + 3 * G;
  view_.hap_bases = d_haps;
  view_.hap_off = d_hap_off;
  view_.read_region = d_read_region;
  view_.region_hap = d_region_hap;
  view_.region_nhap = d_region_nhap;
  view_.region_read = d_region_read;
  view_.region_out = d_region_out;
  view_.out = d_out_;
  view_.g_ins = d_out_ + out_len_;
  view_.g_del = view_.g_ins + G;
  view_.g_eps = view_.g_del + G;
  view_.g_err = view_.g_eps + G;
  view_.lost = d_lost_;
  return FGKL_OK;
}

int AdjointEngine::run() {
  DeviceGuard device_guard(device_);
  int rc;
  const size_t n_launch = bins_.size() + rescue_.size();
  int* counters = d_small_;
  int* queue_off = d_small_ + (n_small_ - 2 * kAdjRowBins - 1);
  int* queue_tail = d_small_ + (n_small_ - kAdjRowBins);
  if ((rc = check(cudaMemsetAsync(counters, 0, n_launch * sizeof(int), stream_), "reset counters"))) return rc;
  if ((rc = check(cudaMemsetAsync(queue_tail, 0, kAdjRowBins * sizeof(int), stream_), "reset queues"))) return rc;
  if ((rc = check(cudaMemsetAsync(d_lost_, 0, sizeof(unsigned long long), stream_), "reset counters"))) return rc;
  // The kernels add each pair's gradient terms into the per-position arrays.
  if (grad_len_ > 0 &&
      (rc = check(cudaMemsetAsync(view_.g_ins, 0, 4 * static_cast<size_t>(grad_len_) * sizeof(double), stream_), "reset gradients")))
    return rc;
  launches_ = 0;
  int i = 0;
  for (int pass = 0; pass < 2; ++pass) {
    const auto& list = pass == 0 ? bins_ : rescue_;
    for (const Bin& b : list) {
      AdjLaunch a{};
      a.v = view_;
      a.tasks = (pass == 0 ? tasks_ : queue_) + b.task_off;
      a.n_tasks = b.n_tasks;
      a.count = pass == 0 ? nullptr : queue_tail + b.rows;
      a.task_counter = counters + i++;
      a.scratch = d_scratch_;
      a.scratch_stride = b.stride;
      a.queue = (pass == 0 && !dbl_) ? queue_ : nullptr;
      a.queue_off = queue_off;
      a.queue_tail = queue_tail;
      if ((rc = check(adj_launch(b.dbl, b.rows, b.blocks, a, stream_), "adjoint launch"))) return rc;
      ++launches_;
    }
  }
  return FGKL_OK;
}

int AdjointEngine::fetch(double* out, int64_t out_len, double* g_ins, double* g_del, double* g_eps, double* g_err, int64_t grad_len,
                         uint64_t* fp64_reads) {
  DeviceGuard device_guard(device_);
  if (out_len != out_len_) return fail(FGKL_E_OUTPUT_LENGTH, "likelihood output has the wrong length");
  if (grad_len != grad_len_) return fail(FGKL_E_OUTPUT_LENGTH, "gradient arrays must hold one value per read position");
  int rc;
  auto down = [&](void* dst, const void* src, size_t bytes) {
    if (bytes == 0 || dst == nullptr) return FGKL_OK;
    return check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream_), "download");
  };
  const size_t G = static_cast<size_t>(grad_len_) * 8;
  unsigned long long lost = 0;
  if ((rc = down(out, view_.out, static_cast<size_t>(out_len_) * 8)) || (rc = down(g_ins, view_.g_ins, G)) ||
      (rc = down(g_del, view_.g_del, G)) || (rc = down(g_eps, view_.g_eps, G)) || (rc = down(g_err, view_.g_err, G)) ||
      (rc = down(&lost, d_lost_, sizeof lost)))
    return rc;
  if ((rc = check(cudaStreamSynchronize(stream_), "adjoint kernels"))) return rc;
  if (fp64_reads) *fp64_reads = lost;
  return FGKL_OK;
}

}  // namespace fgkl
