#include "engine.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <thread>

#include "../../include/fgkl_b200.h"
#include "planner.h"
#include "tables.h"

namespace fgkl {

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kRowBins = 21;  // rows-per-lane values 1..20 index the recomputation queues
constexpr int64_t kMaxReadLen = 620;  // 31 rows per lane x 20 rows

// Rows per lane: lane 0 holds only padding rows, so 31 * rows >= len.
int packed_rows(int len) { return (len + 30) / 31; }

size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// Rows per lane for one read on the single-read kinds: 31 * rows >= len, even above 8.
int single_rows(int len) {
  int rows = packed_rows(len);
  if (rows > 8) rows = (rows + 1) & ~1;
  return rows;
}

struct RegionPlan {
  ProgramBuild shared, prefix;
  std::vector<HapInfo> haps;
  uint8_t codes[256];
  SharedColumns cols;
  uint64_t read_bases = 0, hap_bases = 0;
  bool extra_codes = false;  // a haplotype byte outside ACGTN: the region runs on the FP64 kernel
};

void plan_region(const BatchInput& in, int g, int64_t first_read, int64_t first_hap, bool share, RegionPlan& out) {
  const int n_haps = in.region_haps[g], n_reads = in.region_reads[g];
  std::vector<HapView> views(static_cast<size_t>(n_haps));
  for (int h = 0; h < n_haps; ++h) {
    const int64_t lo = in.hap_off[first_hap + h], hi = in.hap_off[first_hap + h + 1];
    views[h] = HapView{in.hap_bases + lo, static_cast<int32_t>(hi - lo)};
    out.hap_bases += static_cast<uint64_t>(hi - lo);
  }
  for (int r = 0; r < n_reads; ++r)
    out.read_bases += static_cast<uint64_t>(in.read_off[first_read + r + 1] - in.read_off[first_read + r]);
  if (n_haps == 0 || n_reads == 0) return;
  const SortedHaps s = SortedHaps::make(views, share);
  emit_program(s, share, out.shared);
  emit_program(s, false, out.prefix);
  code_table(s, out.codes);
  out.extra_codes = s.num_codes() > 5;
  out.cols = s.columns();
  out.haps.resize(static_cast<size_t>(n_haps));
  int seg = -1;
  for (int k = 0; k < n_haps; ++k) {
    if (!s.dup[k]) ++seg;
    int src = k;
    while (src > 0 && s.dup[src]) --src;
    out.haps[k] = HapInfo{s.order[k], seg, src, 0};
  }
}

template <class T>
void append_section(std::vector<uint8_t>& blob, const std::vector<T>& v, size_t& off) {
  off = align_up(blob.size(), 16);
  blob.resize(off + v.size() * sizeof(T));
  if (!v.empty()) std::memcpy(blob.data() + off, v.data(), v.size() * sizeof(T));
}

}  // namespace

Engine::Engine(int device, cudaStream_t stream) : device_(device), stream_(stream) {
  cudaSetDevice(device_);
  cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_);
  if (!stream_) {
    cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    own_stream_ = true;
  }
  const Tables& t = tables();
  cudaMalloc(&d_err_, sizeof(double) * t.error_prob.size());
  cudaMalloc(&d_m2m_, sizeof(double) * t.m2m.size());
  cudaMemcpy(d_err_, t.error_prob.data(), sizeof(double) * t.error_prob.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d_m2m_, t.m2m.data(), sizeof(double) * t.m2m.size(), cudaMemcpyHostToDevice);
  cudaMalloc(&d_counters_, sizeof(Counters));
  for (int i = 0; i < kAuxStreams; ++i) {
    cudaStreamCreateWithFlags(&aux_[i], cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&join_[i], cudaEventDisableTiming);
  }
  cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming);
}

Engine::~Engine() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  cudaFree(d_reads_);
  cudaFree(d_read_off_);
  cudaFree(d_plan_);
  cudaFree(d_tasks_);
  cudaFree(d_queue_);
  cudaFree(d_small_);
  cudaFree(d_out_);
  cudaFree(d_counters_);
  cudaFree(d_scratch_);
  cudaFree(d_err_);
  cudaFree(d_m2m_);
  if (h_stage_) cudaFreeHost(h_stage_);
  for (int i = 0; i < kAuxStreams; ++i) {
    cudaStreamDestroy(aux_[i]);
    cudaEventDestroy(join_[i]);
  }
  cudaEventDestroy(fork_);
  if (own_stream_) cudaStreamDestroy(stream_);
}

int Engine::fail(int code, const std::string& msg) {
  error_ = msg;
  return code;
}

int Engine::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FGKL_OK;
  return fail(FGKL_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T* Engine::grow(T*& ptr, size_t& cap, size_t n) {
  const size_t bytes = std::max<size_t>(n * sizeof(T), 256);
  if (bytes > cap) {
    cudaFree(ptr);
    ptr = nullptr;
    if (cudaMalloc(&ptr, bytes) != cudaSuccess) {
      cap = 0;
      ptr = nullptr;
      return nullptr;
    }
    cap = bytes;
  }
  return ptr;
}

int Engine::prepare(const BatchInput& in, const EngineConfig& cfg) {
  cudaSetDevice(device_);
  cfg_ = cfg;
  error_.clear();
  planned_ = BatchStats{};
  bins_.clear();
  rescue_bins_.clear();
  const int N = in.num_regions;
  if (N < 0) return fail(FGKL_E_INVALID_ARGUMENT, "negative region count");

  // Region starts and validation (lib.rs:278-290).
  std::vector<int64_t> first_read(N + 1, 0), first_hap(N + 1, 0), out_off(N + 1, 0);
  for (int g = 0; g < N; ++g) {
    if (in.region_reads[g] < 0 || in.region_haps[g] < 0) return fail(FGKL_E_INVALID_ARGUMENT, "negative region size");
    first_read[g + 1] = first_read[g] + in.region_reads[g];
    first_hap[g + 1] = first_hap[g] + in.region_haps[g];
    out_off[g + 1] = out_off[g] + static_cast<int64_t>(in.region_reads[g]) * in.region_haps[g];
  }
  const int64_t total_reads = first_read[N], total_haps = first_hap[N];
  out_len_ = out_off[N];
  for (int g = 0; g < N; ++g) {
    for (int64_t r = first_read[g]; r < first_read[g + 1]; ++r) {
      const int64_t len = in.read_off[r + 1] - in.read_off[r];
      if (len <= 0) return fail(FGKL_E_EMPTY_READ, "read " + std::to_string(r - first_read[g]) + " has no bases");
      if (len > kMaxReadLen)
        return fail(FGKL_E_UNSUPPORTED, "read " + std::to_string(r - first_read[g]) + " has " + std::to_string(len) +
                                            " bases; reads of at most 620 bases are supported");
    }
    for (int64_t h = first_hap[g]; h < first_hap[g + 1]; ++h)
      if (in.hap_off[h + 1] - in.hap_off[h] <= 0)
        return fail(FGKL_E_EMPTY_HAPLOTYPE, "haplotype " + std::to_string(h - first_hap[g]) + " has no bases");
  }

  // Plan the regions in parallel.
  std::vector<RegionPlan> plans(static_cast<size_t>(N));
  const bool share = cfg.share_suffixes;
  {
    const int threads = std::max(1, std::min<int>(static_cast<int>(std::thread::hardware_concurrency()), (N + 7) / 8));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t] {
        for (int g = t; g < N; g += threads) plan_region(in, g, first_read[g], first_hap[g], share, plans[g]);
      });
    for (auto& th : pool) th.join();
  }

  // Concatenate the programs; each stream gets kStreamPad zero entries on both sides.
  std::vector<Region> regions(static_cast<size_t>(N));
  std::vector<HapInfo> haps;
  std::vector<uint32_t> stream(kStreamPad, 0u);
  std::vector<Segment> segs;
  std::vector<Sweep> sweeps;
  std::vector<uint8_t> codes(static_cast<size_t>(N) * 256);
  int max_slots = 1, max_nodes = 1, max_segs = 1;
  auto put_stream = [&](const std::vector<uint32_t>& v, int32_t& off, int32_t& len) {
    off = static_cast<int32_t>(stream.size());
    len = v.empty() ? 0 : static_cast<int32_t>(v.size()) - 1;  // the last entry only carries post events
    stream.insert(stream.end(), v.begin(), v.end());
    stream.insert(stream.end(), kStreamPad, 0u);
  };
  auto put_program = [&](const ProgramBuild& b, Program& p) {
    put_stream(b.fwd, p.fwd_off, p.fwd_len);
    put_stream(b.bwd, p.bwd_off, p.bwd_len);
    p.seg_off = static_cast<int32_t>(segs.size());
    p.n_segs = static_cast<int32_t>(b.segs.size());
    segs.insert(segs.end(), b.segs.begin(), b.segs.end());
    p.sweep_off = static_cast<int32_t>(sweeps.size());
    p.n_sweeps = static_cast<int32_t>(b.sweeps.size());
    sweeps.insert(sweeps.end(), b.sweeps.begin(), b.sweeps.end());
    p.n_slots = b.n_slots;
    p.n_nodes = b.n_nodes;
    max_slots = std::max(max_slots, b.n_slots);
    max_nodes = std::max(max_nodes, b.n_nodes);
    max_segs = std::max(max_segs, static_cast<int>(b.segs.size()));
  };
  for (int g = 0; g < N; ++g) {
    RegionPlan& rp = plans[g];
    Region& R = regions[g];
    std::memset(&R, 0, sizeof R);
    put_program(rp.shared, R.shared);
    put_program(rp.prefix, R.prefix);
    R.hap_off = static_cast<int32_t>(haps.size());
    R.n_haps = in.region_haps[g];
    R.read_off = static_cast<int32_t>(first_read[g]);
    R.n_reads = in.region_reads[g];
    R.out_off = out_off[g];
    R.code_off = g * 256;
    haps.insert(haps.end(), rp.haps.begin(), rp.haps.end());
    if (!rp.haps.empty()) std::memcpy(codes.data() + static_cast<size_t>(g) * 256, rp.codes, 256);
    planned_.nominal_cells += rp.read_bases * rp.hap_bases;
    planned_.forward_cells += rp.read_bases * rp.shared.fwd_columns;
    planned_.backward_cells += rp.read_bases * rp.shared.bwd_columns;
    planned_.prefix_only_cells += rp.read_bases * rp.cols.prefix_only;
  }
  planned_.computed_cells = planned_.forward_cells + planned_.backward_cells;

  // Tasks: reads sorted longest first; FP32 packs consecutive pairs below 256 bases.
  struct Key {
    Kind kind;
    int rows;
    bool operator<(const Key& o) const { return kind != o.kind ? kind < o.kind : rows < o.rows; }
  };
  std::map<Key, std::vector<std::pair<uint64_t, Task>>> by_bin;
  std::vector<int> rescue_count(kRowBins, 0);
  for (int g = 0; g < N; ++g) {
    const int n_reads = in.region_reads[g];
    if (n_reads == 0 || in.region_haps[g] == 0) continue;
    std::vector<int> order(static_cast<size_t>(n_reads));
    for (int r = 0; r < n_reads; ++r) order[r] = r;
    auto len_of = [&](int r) { return static_cast<int>(in.read_off[first_read[g] + r + 1] - in.read_off[first_read[g] + r]); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return len_of(a) > len_of(b); });
    const uint64_t cost_cols = plans[g].shared.fwd.size() + plans[g].shared.bwd.size() + 31;
    for (int r = 0; r < n_reads; ++r) rescue_count[single_rows(len_of(r))]++;
    size_t i = 0;
    if (cfg.double_precision || plans[g].extra_codes) {
      for (; i < order.size(); ++i) {
        const int rows = single_rows(len_of(order[i]));
        by_bin[{Kind::kOneF64, rows}].push_back(
            {cost_cols * rows, Task{g, {static_cast<int32_t>(first_read[g] + order[i]), -1}, rows}});
      }
    } else {
      while (i < order.size() && packed_rows(len_of(order[i])) > 8) {
        const int rows = single_rows(len_of(order[i]));
        by_bin[{Kind::kOneF32, rows}].push_back(
            {cost_cols * rows, Task{g, {static_cast<int32_t>(first_read[g] + order[i]), -1}, rows}});
        ++i;
      }
      for (; i < order.size(); i += 2) {
        const int rows = packed_rows(len_of(order[i]));
        const int32_t a = static_cast<int32_t>(first_read[g] + order[i]);
        const int32_t b = i + 1 < order.size() ? static_cast<int32_t>(first_read[g] + order[i + 1]) : -1;
        by_bin[{Kind::kPackedF32, rows}].push_back({cost_cols * rows, Task{g, {a, b}, rows}});
      }
    }
  }
  std::vector<Task> tasks;
  std::vector<std::pair<uint64_t, Bin>> first;
  for (auto& [key, list] : by_bin) {
    std::stable_sort(list.begin(), list.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    Bin b{key.kind, key.rows, static_cast<int>(tasks.size()), static_cast<int>(list.size()), 0, 0, 0};
    uint64_t cost = 0;
    for (auto& e : list) {
      tasks.push_back(e.second);
      cost += e.first;
    }
    int per_sm = 0, threads = 0;
    occupancy(b.kind, b.rows, &per_sm, &threads);
    if (per_sm <= 0) return fail(FGKL_E_CUDA, "kernel instantiation unavailable on this device");
    b.blocks = std::max(1, std::min((b.n_tasks + kWarpsPerBlock - 1) / kWarpsPerBlock, per_sm * sms_));
    first.push_back({cost, b});
  }
  // The bin with the most work launches first; the others fill the SMs its tail frees.
  std::stable_sort(first.begin(), first.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  for (auto& f : first) bins_.push_back(f.second);
  std::vector<int> queue_off(kRowBins, 0);
  {
    int acc = 0;
    for (int r = 0; r < kRowBins; ++r) {
      queue_off[r] = acc;
      acc += rescue_count[r];
    }
  }
  if (cfg.double_fallback) {
    for (int r = 1; r < kRowBins; ++r) {
      if (rescue_count[r] == 0) continue;
      int per_sm = 0, threads = 0;
      occupancy(Kind::kOneF64, r, &per_sm, &threads);
      if (per_sm <= 0) return fail(FGKL_E_CUDA, "recomputation kernel unavailable on this device");
      Bin b{Kind::kOneF64, r, queue_off[r], rescue_count[r], 0, 0, 0};
      b.blocks = std::max(1, std::min((b.n_tasks + kWarpsPerBlock - 1) / kWarpsPerBlock, per_sm * sms_));
      rescue_bins_.push_back(b);
    }
  }
  // Bins of one pass run concurrently, so each owns a slice of the scratch.
  size_t scratch_total = 256;
  for (auto* list : {&bins_, &rescue_bins_}) {
    size_t off = 0;
    for (Bin& b : *list) {
      b.stride = align_up(scratch_bytes(b.kind, b.rows, max_slots, max_nodes, max_segs));
      b.scratch_off = off;
      off += static_cast<size_t>(b.blocks) * kWarpsPerBlock * b.stride;
    }
    scratch_total = std::max(scratch_total, off);
  }

  // Plan blob: regions | haps | stream | segs | sweeps | code tables.
  std::vector<uint8_t> blob;
  size_t o_regions, o_haps, o_stream, o_segs, o_sweeps, o_codes;
  append_section(blob, regions, o_regions);
  append_section(blob, haps, o_haps);
  append_section(blob, stream, o_stream);
  append_section(blob, segs, o_segs);
  append_section(blob, sweeps, o_sweeps);
  append_section(blob, codes, o_codes);

  // Device buffers.
  const int64_t read_bytes = total_reads > 0 ? in.read_off[total_reads] : 0;
  n_small_ = static_cast<int>(bins_.size() + rescue_bins_.size()) + 2 * kRowBins;
  if (!grow(d_reads_, cap_reads_, static_cast<size_t>(read_bytes) * 5 + 16) ||
      !grow(d_read_off_, cap_read_off_, static_cast<size_t>(total_reads) + 1) || !grow(d_plan_, cap_plan_, blob.size()) ||
      !grow(d_tasks_, cap_tasks_, tasks.size() + 1) || !grow(d_queue_, cap_queue_, static_cast<size_t>(total_reads) + 1) ||
      !grow(d_small_, cap_small_, static_cast<size_t>(n_small_)) || !grow(d_out_, cap_out_, static_cast<size_t>(out_len_) + 1) ||
      !grow(d_scratch_, cap_scratch_, scratch_total))
    return fail(FGKL_E_CUDA, "device allocation failed");

  // Stage and upload: reads (five arrays), read offsets, plan, tasks, queue offsets.
  const size_t stage_bytes = align_up(static_cast<size_t>(read_bytes) * 5) + align_up((total_reads + 1) * sizeof(int64_t)) +
                             align_up(blob.size()) + align_up(tasks.size() * sizeof(Task)) + align_up(kRowBins * sizeof(int)) +
                             align_up(static_cast<size_t>(out_len_) * sizeof(double)) + align_up(sizeof(Counters));
  if (stage_bytes > cap_stage_) {
    if (h_stage_) cudaFreeHost(h_stage_);
    h_stage_ = nullptr;
    if (cudaMallocHost(&h_stage_, stage_bytes) != cudaSuccess) {
      cap_stage_ = 0;
      return fail(FGKL_E_CUDA, "pinned host allocation failed");
    }
    cap_stage_ = stage_bytes;
  }
  cudaStreamSynchronize(stream_);  // the staging buffer may still feed an earlier copy
  uint8_t* p = h_stage_;
  const uint8_t* srcs[5] = {in.bases, in.quals, in.ins, in.del, in.gcp};
  for (int a = 0; a < 5; ++a)
    if (read_bytes) std::memcpy(p + static_cast<size_t>(a) * read_bytes, srcs[a], static_cast<size_t>(read_bytes));
  int rc;
  if ((rc = check(cudaMemcpyAsync(d_reads_, p, static_cast<size_t>(read_bytes) * 5, cudaMemcpyHostToDevice, stream_), "upload reads")))
    return rc;
  p += align_up(static_cast<size_t>(read_bytes) * 5);
  std::memcpy(p, in.read_off, (total_reads + 1) * sizeof(int64_t));
  if ((rc = check(cudaMemcpyAsync(d_read_off_, p, (total_reads + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, stream_), "upload offsets")))
    return rc;
  p += align_up((total_reads + 1) * sizeof(int64_t));
  std::memcpy(p, blob.data(), blob.size());
  if ((rc = check(cudaMemcpyAsync(d_plan_, p, blob.size(), cudaMemcpyHostToDevice, stream_), "upload plan"))) return rc;
  p += align_up(blob.size());
  if (!tasks.empty()) {
    std::memcpy(p, tasks.data(), tasks.size() * sizeof(Task));
    if ((rc = check(cudaMemcpyAsync(d_tasks_, p, tasks.size() * sizeof(Task), cudaMemcpyHostToDevice, stream_), "upload tasks")))
      return rc;
  }
  p += align_up(tasks.size() * sizeof(Task));
  std::memcpy(p, queue_off.data(), kRowBins * sizeof(int));
  if ((rc = check(cudaMemcpyAsync(d_small_ + (n_small_ - 2 * kRowBins), p, kRowBins * sizeof(int), cudaMemcpyHostToDevice, stream_),
                  "upload queue offsets")))
    return rc;

  view_.bases = d_reads_;
  view_.quals = d_reads_ + read_bytes;
  view_.ins = d_reads_ + 2 * read_bytes;
  view_.del = d_reads_ + 3 * read_bytes;
  view_.gcp = d_reads_ + 4 * read_bytes;
  view_.read_off = d_read_off_;
  view_.regions = reinterpret_cast<const Region*>(d_plan_ + o_regions);
  view_.haps = reinterpret_cast<const HapInfo*>(d_plan_ + o_haps);
  view_.stream = reinterpret_cast<const uint32_t*>(d_plan_ + o_stream);
  view_.segs = reinterpret_cast<const Segment*>(d_plan_ + o_segs);
  view_.sweeps = reinterpret_cast<const Sweep*>(d_plan_ + o_sweeps);
  view_.code_of_byte = d_plan_ + o_codes;
  view_.err_prob = d_err_;
  view_.m2m = d_m2m_;
  view_.out = d_out_;
  view_.counters = d_counters_;
  (void)total_haps;
  return FGKL_OK;
}

int Engine::run() {
  cudaSetDevice(device_);
  int rc;
  int* counters = d_small_;                                // one per launch
  int* queue_off = d_small_ + (n_small_ - 2 * kRowBins);  // uploaded by prepare
  int* queue_tail = d_small_ + (n_small_ - kRowBins);
  const size_t n_launch = bins_.size() + rescue_bins_.size();
  if ((rc = check(cudaMemsetAsync(counters, 0, n_launch * sizeof(int), stream_), "reset task counters"))) return rc;
  if ((rc = check(cudaMemsetAsync(queue_tail, 0, kRowBins * sizeof(int), stream_), "reset queues"))) return rc;
  if ((rc = check(cudaMemsetAsync(d_counters_, 0, sizeof(Counters), stream_), "reset counters"))) return rc;
  planned_.kernel_launches = 0;
  int i = 0;
  // Each pass forks its bins onto the auxiliary streams and joins them back.
  auto pass = [&](const std::vector<Bin>& list, bool rescue) -> int {
    if (list.empty()) return FGKL_OK;
    if ((rc = check(cudaEventRecord(fork_, stream_), "fork"))) return rc;
    for (size_t b = 0; b < list.size(); ++b) {
      const Bin& bin = list[b];
      cudaStream_t s = aux_[b % kAuxStreams];
      if ((rc = check(cudaStreamWaitEvent(s, fork_, 0), "fork wait"))) return rc;
      LaunchArgs a{};
      a.v = view_;
      a.tasks = (rescue ? d_queue_ : d_tasks_) + bin.task_off;
      a.n_tasks = bin.n_tasks;
      a.count = rescue ? queue_tail + bin.rows : nullptr;
      a.task_counter = counters + i++;
      a.scratch = d_scratch_ + bin.scratch_off;
      a.scratch_stride = bin.stride;
      a.use_prefix = rescue ? 1 : (cfg_.share_suffixes ? 0 : 1);
      a.rescue = rescue ? 1 : 0;
      a.queue = (!rescue && cfg_.double_fallback) ? d_queue_ : nullptr;
      a.queue_off = queue_off;
      a.queue_tail = queue_tail;
      a.min_accept_plain = (!rescue && !cfg_.double_precision) ? 1 : 0;
      if ((rc = check(launch(bin.kind, bin.rows, bin.blocks, a, s), rescue ? "recomputation launch" : "first-pass launch")))
        return rc;
      planned_.kernel_launches++;
      if ((rc = check(cudaEventRecord(join_[b % kAuxStreams], s), "join"))) return rc;
    }
    for (size_t b = 0; b < std::min<size_t>(list.size(), kAuxStreams); ++b)
      if ((rc = check(cudaStreamWaitEvent(stream_, join_[b], 0), "join wait"))) return rc;
    return FGKL_OK;
  };
  if ((rc = pass(bins_, false))) return rc;
  if ((rc = pass(rescue_bins_, true))) return rc;
  return FGKL_OK;
}

int Engine::fetch(double* out, int64_t out_len, BatchStats* stats) {
  cudaSetDevice(device_);
  if (out_len != out_len_)
    return fail(FGKL_E_OUTPUT_LENGTH, "output has " + std::to_string(out_len) + " elements but reads x haplotypes is " +
                                          std::to_string(out_len_));
  int rc;
  double* h_out = reinterpret_cast<double*>(h_stage_);
  Counters* h_cnt = reinterpret_cast<Counters*>(h_stage_ + align_up(static_cast<size_t>(out_len_) * sizeof(double)));
  if (out_len_ > 0 &&
      (rc = check(cudaMemcpyAsync(h_out, d_out_, static_cast<size_t>(out_len_) * sizeof(double), cudaMemcpyDeviceToHost, stream_),
                  "download results")))
    return rc;
  if ((rc = check(cudaMemcpyAsync(h_cnt, d_counters_, sizeof(Counters), cudaMemcpyDeviceToHost, stream_), "download counters")))
    return rc;
  if ((rc = check(cudaStreamSynchronize(stream_), "kernel execution"))) return rc;
  if (out_len_ > 0) std::memcpy(out, h_out, static_cast<size_t>(out_len_) * sizeof(double));
  if (stats) {
    *stats = planned_;
    stats->fallback_pairs = h_cnt->lost_pairs;
    stats->rescue_reads = h_cnt->rescue_reads;
  }
  return FGKL_OK;
}

int Engine::compute(const BatchInput& in, const EngineConfig& cfg, double* out, int64_t out_len, BatchStats* stats) {
  int rc = prepare(in, cfg);
  if (rc) return rc;
  if (out_len != out_len_)
    return fail(FGKL_E_OUTPUT_LENGTH, "output has " + std::to_string(out_len) + " elements but reads x haplotypes is " +
                                          std::to_string(out_len_));
  if (out_len_ == 0) {
    if (stats) *stats = planned_;
    return FGKL_OK;
  }
  if ((rc = run())) return rc;
  return fetch(out, out_len, stats);
}

}  // namespace fgkl
