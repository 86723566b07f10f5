#include "engine.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstddef>
#include <cstring>
#include <string>
#include <thread>

#include "../../include/fgkl_b200.h"
#include "planner.h"
#include "tables.h"

namespace fgkl {

namespace {
std::atomic<int64_t> g_allocation_limit{0};
}  // namespace

int64_t allocation_limit() { return g_allocation_limit.load(std::memory_order_relaxed); }
int64_t set_allocation_limit(int64_t bytes) { return g_allocation_limit.exchange(bytes); }

bool over_allocation_limit(size_t bytes) {
  const int64_t lim = allocation_limit();
  return lim > 0 && bytes > static_cast<size_t>(lim);
}

cudaError_t device_alloc(void** p, size_t bytes) {
  const int64_t lim = allocation_limit();
  if (lim > 0 && bytes > static_cast<size_t>(lim)) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

cudaError_t pinned_alloc(void** p, size_t bytes) {
  const int64_t lim = allocation_limit();
  if (lim > 0 && bytes > static_cast<size_t>(lim)) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(p, bytes);
}

namespace {

constexpr int kWarpsPerBlock = 4;

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
  ProgramBuild prog;
  std::vector<HapInfo> haps;
  std::vector<uint8_t> seq;        // prior codes of the distinct sorted haplotypes, concatenated
  std::vector<uint32_t> pd_seq;    // PD: their forward entries (code and deletion bits)
  std::vector<uint32_t> pd_sigs;   // PD: per match-set code, the read classes it accepts
  std::string error;               // a region the kernels cannot take
  uint8_t codes[256];
  SharedColumns cols;
  uint64_t read_bases = 0, hap_bases = 0;
  int n_distinct = 0;
  bool extra_codes = false;  // a haplotype byte outside ACGTN: the region runs on the FP64 kernel
  bool generic = false;      // PD: more read bytes than class bits, or more than 256 match sets
};

// PD regions: the reads' distinct bytes become classes 0..30 (first-seen order) and each match-set
// code the bit set of classes it accepts, so the kernel's prior is one bit test per row.
bool pd_read_classes(const BatchInput& in, int64_t first_read, int n_reads, const SortedHaps& s, RegionPlan& out) {
  std::memset(out.codes, kNoCode, 256);
  std::vector<uint8_t> bytes;
  for (int r = 0; r < n_reads; ++r)
    for (int64_t o = in.read_off[first_read + r]; o < in.read_off[first_read + r + 1]; ++o) {
      const uint8_t b = in.bases[o];
      if (out.codes[b] != kNoCode) continue;
      if (static_cast<int>(bytes.size()) >= kPdMaxReadClasses) return false;
      out.codes[b] = static_cast<uint8_t>(bytes.size());
      bytes.push_back(b);
    }
  out.pd_sigs.assign(s.match_sets.size(), 0u);
  for (size_t code = 0; code < s.match_sets.size(); ++code)
    for (size_t c = 0; c < bytes.size(); ++c)
      if (s.match_sets[code].accepts(bytes[c])) out.pd_sigs[code] |= 1u << c;
  return true;
}

void plan_region(const BatchInput& in, int g, int64_t first_read, int64_t first_hap, bool share, RegionPlan& out) {
  const int n_haps = in.region_haps[g], n_reads = in.region_reads[g];
  std::vector<HapView> views(static_cast<size_t>(n_haps));
  std::vector<const uint8_t*> flags(in.hap_flags ? static_cast<size_t>(n_haps) : 0);
  for (int h = 0; h < n_haps; ++h) {
    const int64_t lo = in.hap_off[first_hap + h], hi = in.hap_off[first_hap + h + 1];
    views[h] = HapView{in.hap_bases + lo, static_cast<int32_t>(hi - lo)};
    if (in.hap_flags) flags[h] = in.hap_flags + lo;
    out.hap_bases += static_cast<uint64_t>(hi - lo);
  }
  for (int r = 0; r < n_reads; ++r)
    out.read_bases += static_cast<uint64_t>(in.read_off[first_read + r + 1] - in.read_off[first_read + r]);
  if (n_haps == 0 || n_reads == 0) return;
  const bool pd = in.hap_flags != nullptr;
  SortedHaps s;
  try {
    s = pd ? SortedHaps::make_pd(views, flags) : SortedHaps::make(views, share);
    emit_program(s, share && !pd, out.prog);
  } catch (const std::exception& e) {
    out.error = e.what();
    return;
  }
  if (pd) {
    // Regions the class bits cannot describe compare bytes in the kernel instead (every pair then
    // runs unshared, as fgkl's answer for them does not depend on sharing).
    out.generic = s.too_many_sets || !pd_read_classes(in, first_read, n_reads, s, out);
    if (out.generic) out.pd_sigs.clear();
  } else {
    code_table(s, out.codes);
    out.extra_codes = s.num_codes() > 5;
  }
  out.cols = s.columns();
  out.haps.resize(static_cast<size_t>(n_haps));
  int seg = -1, src = 0;
  for (int k = 0; k < n_haps; ++k) {
    if (!s.dup[k]) {
      ++seg;
      src = k;
      if (pd) {
        out.haps[k].seq = static_cast<int32_t>(out.pd_seq.size());
        for (int32_t j = 0; j < s.bases[k].len; ++j) {
          if (out.generic) {
            // The column's own byte and ALT bits (shifted to bit 0) in place of a match-set code.
            const MatchSet set = MatchSet::of(s.bases[k].bases[j], s.flags[k][j]);
            out.pd_seq.push_back(set.base | (static_cast<uint32_t>(set.alts >> 3) << kPdPayloadShift) | s.pd_bits[k][j]);
          } else {
            out.pd_seq.push_back(s.codes[k][j] | s.pd_bits[k][j]);
          }
        }
      } else {
        out.haps[k].seq = static_cast<int32_t>(out.seq.size());
        out.seq.insert(out.seq.end(), s.codes[k].begin(), s.codes[k].end());
      }
      ++out.n_distinct;
    } else {
      out.haps[k].seq = out.haps[src].seq;
    }
    HapInfo& h = out.haps[k];
    h.order = s.order[k];
    h.seg = seg;
    h.src = src;
    h.len = s.bases[k].len;
    h.pad_[0] = h.pad_[1] = h.pad_[2] = 0;
  }
}

// Runs fn(i) for i in [0, n) on up to `threads` threads, the calling thread among them. Each thread
// takes the next item when it finishes one, so uneven items (regions of 8 to 256 reads) balance.
template <class F>
void parallel_for(int64_t n, int threads, F&& fn) {
  threads = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(threads, n)));
  if (threads == 1) {
    for (int64_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int64_t> next{0};
  auto work = [&] {
    for (int64_t i = next.fetch_add(1, std::memory_order_relaxed); i < n; i = next.fetch_add(1, std::memory_order_relaxed))
      fn(i);
  };
  std::vector<std::thread> pool;
  pool.reserve(static_cast<size_t>(threads) - 1);
  for (int t = 1; t < threads; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

int host_threads() { return std::max(1, static_cast<int>(std::thread::hardware_concurrency())); }

// Copies `bytes` bytes in `chunks` pieces on several threads.
void parallel_copy(uint8_t* dst, const uint8_t* src, size_t bytes) {
  constexpr size_t kChunk = size_t{4} << 20;
  const int64_t chunks = static_cast<int64_t>((bytes + kChunk - 1) / kChunk);
  parallel_for(chunks, std::min(host_threads(), 16), [&](int64_t c) {
    const size_t lo = static_cast<size_t>(c) * kChunk, n = std::min(kChunk, bytes - lo);
    std::memcpy(dst + lo, src + lo, n);
  });
}

}  // namespace

Engine::Engine(int device, cudaStream_t stream) : device_(device), stream_(stream) {
  DeviceGuard device_guard(device_);
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
  cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking);
  cudaEventCreateWithFlags(&uploaded_, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&computed_, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&fetched_, cudaEventDisableTiming);
}

Engine::~Engine() {
  DeviceGuard device_guard(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  if (copy_) cudaStreamSynchronize(copy_);
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
  if (h_reads_) cudaFreeHost(h_reads_);
  for (int i = 0; i < kAuxStreams; ++i) {
    cudaStreamDestroy(aux_[i]);
    cudaEventDestroy(join_[i]);
  }
  cudaEventDestroy(fork_);
  cudaEventDestroy(uploaded_);
  cudaEventDestroy(computed_);
  cudaEventDestroy(fetched_);
  if (copy_) cudaStreamDestroy(copy_);
  for (cudaEvent_t e : ev_) cudaEventDestroy(e);
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
  if (over_allocation_limit(bytes)) return nullptr;  // the buffer held so far is kept
  if (bytes > cap) {
    // Half as much again as the old size: a caller whose batches vary in size stops reallocating
    // after a few calls (cudaFree waits for the whole device, other callers' streams included).
    const size_t want = cap > 0 ? std::max(bytes, cap + cap / 2) : bytes;
    cudaFree(ptr);
    ptr = nullptr;
    if (device_alloc(reinterpret_cast<void**>(&ptr), want) == cudaSuccess) {
      cap = want;
    } else if (want > bytes && (cudaGetLastError(), device_alloc(reinterpret_cast<void**>(&ptr), bytes) == cudaSuccess)) {
      cap = bytes;
    } else {
      cudaGetLastError();
      cap = 0;
      ptr = nullptr;
      return nullptr;
    }
  }
  return ptr;
}

namespace {
double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

namespace {
// Whether [p, p + bytes) lies in one page-locked host allocation (cudaMallocHost, cudaHostAlloc or
// cudaHostRegister): both ends are host memory the device maps, at device addresses `bytes - 1`
// apart. Pageable memory answers false.
bool host_pinned(const void* p, size_t bytes) {
  if (!p || bytes == 0) return false;
  cudaPointerAttributes lo{}, hi{};
  if (cudaPointerGetAttributes(&lo, p) != cudaSuccess ||
      cudaPointerGetAttributes(&hi, static_cast<const uint8_t*>(p) + bytes - 1) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (lo.type != cudaMemoryTypeHost || hi.type != cudaMemoryTypeHost || !lo.devicePointer || !hi.devicePointer) return false;
  return static_cast<const uint8_t*>(hi.devicePointer) - static_cast<const uint8_t*>(lo.devicePointer) ==
         static_cast<std::ptrdiff_t>(bytes - 1);
}

// Grows a pinned host buffer to at least `bytes`, by half again at least (cudaFreeHost waits for the
// whole device); false when the allocation fails.
bool grow_pinned(uint8_t*& p, size_t& cap, size_t bytes) {
  if (over_allocation_limit(bytes)) return false;
  if (bytes <= cap) return true;
  const size_t want = cap > 0 ? std::max(bytes, cap + cap / 2) : bytes;
  if (p) cudaFreeHost(p);
  p = nullptr;
  if (pinned_alloc(reinterpret_cast<void**>(&p), want) == cudaSuccess) {
    cap = want;
    return true;
  }
  cudaGetLastError();
  if (want > bytes && pinned_alloc(reinterpret_cast<void**>(&p), bytes) == cudaSuccess) {
    cap = bytes;
    return true;
  }
  cudaGetLastError();
  p = nullptr;
  cap = 0;
  return false;
}

// Runs a callable on a helper thread and joins it when it goes out of scope, so an early return
// from prepare() never leaves the copy running.
class Helper {
 public:
  template <class F>
  explicit Helper(bool on, F&& f) {
    if (on) th_ = std::thread(std::forward<F>(f));
    else f();
  }
  ~Helper() { join(); }
  void join() {
    if (th_.joinable()) th_.join();
  }

 private:
  std::thread th_;
};
}  // namespace

int plan_region_cells(const BatchInput& in, const EngineConfig& cfg, uint64_t* cells, std::string* error) {
  const int N = in.num_regions;
  if (N < 0) return (*error = "negative region count", FGKL_E_INVALID_ARGUMENT);
  std::vector<int64_t> first_read(N + 1, 0), first_hap(N + 1, 0);
  for (int g = 0; g < N; ++g) {
    if (in.region_reads[g] < 0 || in.region_haps[g] < 0) return (*error = "negative region size", FGKL_E_INVALID_ARGUMENT);
    first_read[g + 1] = first_read[g] + in.region_reads[g];
    first_hap[g + 1] = first_hap[g] + in.region_haps[g];
  }
  for (int64_t h = 0; h < first_hap[N]; ++h)
    if (in.hap_off[h + 1] - in.hap_off[h] <= 0) return (*error = "haplotype " + std::to_string(h) + " has no bases", FGKL_E_EMPTY_HAPLOTYPE);
  for (int64_t r = 0; r < first_read[N]; ++r)
    if (in.read_off[r + 1] - in.read_off[r] <= 0) return (*error = "read " + std::to_string(r) + " has no bases", FGKL_E_EMPTY_READ);
  // The cells each region's tasks compute (the counts prepare() gives the launches): reads of one
  // block walk the region's program (forward and backward columns); strip-mined reads and the reads
  // of byte-compared PD regions run each distinct haplotype unshared.
  parallel_for(N, host_threads(), [&](int64_t gi) {
    const int g = static_cast<int>(gi);
    RegionPlan rp;
    plan_region(in, g, first_read[g], first_hap[g], cfg.share_suffixes, rp);
    uint64_t distinct_len = 0;
    for (int k = 0; k < static_cast<int>(rp.haps.size()); ++k)
      if (rp.haps[k].src == k) distinct_len += static_cast<uint64_t>(rp.haps[k].len);
    uint64_t c = 0;
    for (int64_t r = first_read[g]; r < first_read[g + 1]; ++r) {
      const uint64_t len = static_cast<uint64_t>(in.read_off[r + 1] - in.read_off[r]);
      if (rp.generic || len > static_cast<uint64_t>(kMaxBlockRead))
        c += len * distinct_len;
      else
        c += len * (rp.prog.fwd_columns + rp.prog.bwd_columns);
    }
    cells[g] = rp.error.empty() ? c : 0;
  });
  return FGKL_OK;
}

int Engine::prepare(const BatchInput& in, const EngineConfig& cfg) {
  DeviceGuard device_guard(device_);
  const auto t_start = std::chrono::steady_clock::now();
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
  n_regions_ = N;
  for (int g = 0; g < N; ++g) {
    for (int64_t r = first_read[g]; r < first_read[g + 1]; ++r) {
      const int64_t len = in.read_off[r + 1] - in.read_off[r];
      if (len <= 0) return fail(FGKL_E_EMPTY_READ, "read " + std::to_string(r - first_read[g]) + " has no bases");
      if (len > INT32_MAX) return fail(FGKL_E_INVALID_ARGUMENT, "read " + std::to_string(r - first_read[g]) + " is longer than 2^31 - 1 bases");
    }
    for (int64_t h = first_hap[g]; h < first_hap[g + 1]; ++h)
      if (in.hap_off[h + 1] - in.hap_off[h] <= 0)
        return fail(FGKL_E_EMPTY_HAPLOTYPE, "haplotype " + std::to_string(h - first_hap[g]) + " has no bases");
  }

  // This engine's previous batch: its kernels may still read the device inputs about to be
  // overwritten, and its copies may still read or fill the staging buffers. Events recorded before
  // anything was enqueued complete at once.
  int rc0;
  if ((rc0 = check(cudaEventSynchronize(computed_), "previous batch"))) return rc0;
  if ((rc0 = check(cudaEventSynchronize(uploaded_), "previous upload"))) return rc0;
  if ((rc0 = check(cudaEventSynchronize(fetched_), "previous download"))) return rc0;

  // The five read arrays: uploaded from where they lie when the caller holds them in page-locked
  // memory; otherwise copied to pinned staging first, on a helper thread while the regions are
  // planned (large batches only; a small call copies them in line).
  const int64_t read_bytes = total_reads > 0 ? in.read_off[total_reads] : 0;
  const uint8_t* const read_arrays[5] = {in.bases, in.quals, in.ins, in.del, in.gcp};
  bool direct_reads = read_bytes > 0;
  for (int a = 0; a < 5 && direct_reads; ++a) direct_reads = host_pinned(read_arrays[a], static_cast<size_t>(read_bytes));
  if (!direct_reads && !grow_pinned(h_reads_, cap_h_reads_, static_cast<size_t>(read_bytes) * 5 + 16))
    return fail(FGKL_E_OUT_OF_MEMORY, "pinned host allocation failed");
  Helper read_copy(!direct_reads && read_bytes >= (int64_t{8} << 20), [this, &read_arrays, read_bytes, direct_reads] {
    if (direct_reads) return;
    for (int a = 0; a < 5; ++a)
      if (read_bytes) parallel_copy(h_reads_ + static_cast<size_t>(a) * read_bytes, read_arrays[a], static_cast<size_t>(read_bytes));
  });
  // Page-locked reads start uploading now, under the planning. Any return from here on waits for
  // these copies first: they read the caller's memory.
  struct UploadGuard {
    cudaStream_t s = nullptr;
    ~UploadGuard() {
      if (s) cudaStreamSynchronize(s);
    }
  } upload_guard;
  if (direct_reads) {
    if (!grow(d_reads_, cap_reads_, static_cast<size_t>(read_bytes) * 5 + 16)) return fail(FGKL_E_OUT_OF_MEMORY, "device allocation failed");
    upload_guard.s = copy_;
    for (int a = 0; a < 5; ++a)
      if ((rc0 = check(cudaMemcpyAsync(d_reads_ + static_cast<size_t>(a) * read_bytes, read_arrays[a], static_cast<size_t>(read_bytes),
                                       cudaMemcpyHostToDevice, copy_),
                       "upload reads")))
        return rc0;
  }

  // Plan the regions in parallel, one region a thread for small batches (a region takes about
  // 75 us to plan; a combined batch of per-call requests holds a few).
  std::vector<RegionPlan> plans(static_cast<size_t>(N));
  const bool share = cfg.share_suffixes;
  parallel_for(N, host_threads(),
               [&](int64_t g) { plan_region(in, static_cast<int>(g), first_read[g], first_hap[g], share, plans[g]); });

  for (int g = 0; g < N; ++g)
    if (!plans[g].error.empty()) return fail(FGKL_E_UNSUPPORTED, "region " + std::to_string(g) + ": " + plans[g].error);
  const bool pd = in.hap_flags != nullptr;

  planned_.host_plan_ms = ms_since(t_start);
  const auto t_pack = std::chrono::steady_clock::now();
  // Section offsets. Each stream gets kStreamPad zero entries on both sides.
  std::vector<Region> regions(static_cast<size_t>(N));
  int64_t n_haps = 0, n_stream = kStreamPad, n_segs = 0, n_sweeps = 0, n_seq = 0, n_pd_seq = 0, n_sigs = 0;
  int max_slots = 1, max_nodes = 1, max_segs = 1;
  std::vector<int64_t> queue_cap(kQueueBins, 0);
  int max_hap_len = 1;  // scratch of the strip-mined kinds: one carry column per haplotype base
  for (int g = 0; g < N; ++g) {
    const RegionPlan& rp = plans[g];
    Region& R = regions[g];
    std::memset(&R, 0, sizeof R);
    Program& p = R.prog;
    auto put_stream = [&](const std::vector<uint32_t>& v, int32_t& off, int32_t& len) {
      off = static_cast<int32_t>(n_stream);
      len = v.empty() ? 0 : static_cast<int32_t>(v.size()) - 1;  // the last entry only carries post events
      n_stream += static_cast<int64_t>(v.size()) + kStreamPad;
    };
    put_stream(rp.prog.fwd, p.fwd_off, p.fwd_len);
    put_stream(rp.prog.bwd, p.bwd_off, p.bwd_len);
    p.seg_off = static_cast<int32_t>(n_segs);
    p.n_segs = static_cast<int32_t>(rp.prog.segs.size());
    n_segs += p.n_segs;
    p.sweep_off = static_cast<int32_t>(n_sweeps);
    p.n_sweeps = static_cast<int32_t>(rp.prog.sweeps.size());
    n_sweeps += p.n_sweeps;
    p.n_slots = rp.prog.n_slots;
    p.n_nodes = rp.prog.n_nodes;
    max_slots = std::max(max_slots, rp.prog.n_slots);
    max_nodes = std::max(max_nodes, rp.prog.n_nodes);
    max_segs = std::max(max_segs, p.n_segs);
    R.hap_off = static_cast<int32_t>(n_haps);
    R.n_haps = in.region_haps[g];
    n_haps += static_cast<int64_t>(rp.haps.size());
    R.read_off = static_cast<int32_t>(first_read[g]);
    R.n_reads = in.region_reads[g];
    R.out_off = out_off[g];
    R.code_off = g * 256;
    R.seq_off = static_cast<int32_t>(pd ? n_pd_seq : n_seq);
    n_seq += static_cast<int64_t>(rp.seq.size());
    n_pd_seq += static_cast<int64_t>(rp.pd_seq.size());
    R.sig_off = static_cast<int32_t>(n_sigs);
    R.flags = rp.generic ? kRegionGeneric : 0;
    n_sigs += static_cast<int64_t>(rp.pd_sigs.size());
    planned_.nominal_cells += rp.read_bases * rp.hap_bases;
    planned_.prefix_only_cells += rp.read_bases * rp.cols.prefix_only;
    for (const HapInfo& h : rp.haps) max_hap_len = std::max(max_hap_len, static_cast<int>(h.len));
    if (rp.n_distinct > 0)
      for (int64_t r = first_read[g]; r < first_read[g + 1]; ++r)
        queue_cap[queue_bin(static_cast<int>(in.read_off[r + 1] - in.read_off[r]), rp.generic)] += rp.n_distinct;
  }
  if (n_stream > INT32_MAX || n_seq > INT32_MAX || n_pd_seq > INT32_MAX || n_haps > INT32_MAX)
    return fail(FGKL_E_INVALID_ARGUMENT, "batch too large for 32-bit plan offsets; split it");

  // Tasks: reads sorted longest first; FP32 packs consecutive pairs below 256 bases. A task costs
  // its region's stream length times its rows, so within a bin (one rows value) the costliest
  // regions' tasks come first: regions are visited in that order (ties by index), which lists each
  // bin's tasks longest first without sorting them.
  constexpr int kKinds = kNumKinds;
  struct BinList {
    std::vector<std::pair<uint64_t, Task>> list;
    uint64_t fwd_cells = 0, bwd_cells = 0;  // forward, backward DP cells
  };
  std::vector<BinList> by_bin(static_cast<size_t>(kKinds) * kRowBins);
  auto bin_at = [&](Kind kind, int rows) -> BinList& { return by_bin[static_cast<size_t>(kind) * kRowBins + rows]; };
  std::vector<int> region_order(static_cast<size_t>(N));
  for (int g = 0; g < N; ++g) region_order[g] = g;
  auto cost_of = [&](int g) { return plans[g].prog.fwd.size() + plans[g].prog.bwd.size() + 31; };
  std::stable_sort(region_order.begin(), region_order.end(), [&](int a, int b) { return cost_of(a) > cost_of(b); });
  // Each region's tasks, built in parallel (its reads sorted longest first, then packed), then
  // appended to the bins serially in region order.
  struct RegionTask {
    Kind kind;
    int rows;
    int len;  // read bases of the task, for the bin's cell counts
    Task task;
    uint64_t cost;  // strip-mined pairs: steps x rows; 0 for the region's program tasks
  };
  std::vector<std::vector<RegionTask>> region_tasks(static_cast<size_t>(N));
  parallel_for(N, std::min(host_threads(), (N + 63) / 64), [&](int64_t gi) {
    const int g = static_cast<int>(gi);
    const int n_reads = in.region_reads[g];
    if (n_reads == 0 || in.region_haps[g] == 0) return;
    std::vector<int> order(static_cast<size_t>(n_reads));
    for (int r = 0; r < n_reads; ++r) order[r] = r;
    auto len_of = [&](int r) { return static_cast<int>(in.read_off[first_read[g] + r + 1] - in.read_off[first_read[g] + r]); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return len_of(a) > len_of(b); });
    std::vector<RegionTask>& out = region_tasks[g];
    out.reserve(static_cast<size_t>(n_reads));
    auto one = [&](Kind kind, int rows, size_t i) {
      out.push_back({kind, rows, len_of(order[i]), Task{g, {static_cast<int32_t>(first_read[g] + order[i]), -1}, rows, -1}, 0});
    };
    auto two = [&](Kind kind, int rows, size_t i) {
      const int32_t a = static_cast<int32_t>(first_read[g] + order[i]);
      const int32_t b = i + 1 < order.size() ? static_cast<int32_t>(first_read[g] + order[i + 1]) : -1;
      out.push_back({kind, rows, len_of(order[i]) + (i + 1 < order.size() ? len_of(order[i + 1]) : 0), Task{g, {a, b}, rows, -1}, 0});
    };
    // One task per distinct sorted haplotype of read order[i], strip-mined over row blocks.
    const RegionPlan& rp = plans[g];
    auto pairs = [&](Kind kind, size_t i) {
      const int len = len_of(order[i]);
      const int rows = long_rows(len, kind == Kind::kLongF32);
      const uint64_t blocks = static_cast<uint64_t>(long_blocks(len, rows));
      for (int k = 0; k < static_cast<int>(rp.haps.size()); ++k)
        if (rp.haps[k].src == k)
          out.push_back({kind, rows, len, Task{g, {static_cast<int32_t>(first_read[g] + order[i]), -1}, rows, k},
                         (static_cast<uint64_t>(rp.haps[k].len) + 32) * blocks * static_cast<uint64_t>(rows)});
    };
    size_t i = 0;
    const bool dbl = cfg.double_precision;
    if (rp.generic) {
      for (; i < order.size(); ++i) pairs(dbl ? Kind::kGenericF64Pd : Kind::kGenericF32Pd, i);
      return;
    }
    const Kind long_kind = pd ? (dbl ? Kind::kLongF64Pd : Kind::kLongF32Pd) : ((dbl || rp.extra_codes) ? Kind::kLongF64 : Kind::kLongF32);
    for (; i < order.size() && len_of(order[i]) > kMaxBlockRead; ++i) pairs(long_kind, i);
    if (pd && cfg.double_precision) {
      // PD in FP64: one read per warp.
      for (; i < order.size(); ++i) one(Kind::kOneF64Pd, single_rows(len_of(order[i])), i);
    } else if (pd) {
      // PD in FP32: reads above 248 bases one per warp, the others in pairs (FP32x2) unless the
      // launch configuration asks for one read per warp.
      for (; i < order.size() && (packed_rows(len_of(order[i])) > 8 || tuning_.reads_per_warp == 1); ++i)
        one(Kind::kOneF32Pd, single_rows(len_of(order[i])), i);
      for (; i < order.size(); i += 2) two(Kind::kPackedF32Pd, packed_rows(len_of(order[i])), i);
    } else if (cfg.double_precision || plans[g].extra_codes) {
      for (; i < order.size(); ++i) one(Kind::kOneF64, single_rows(len_of(order[i])), i);
    } else {
      // The tile-shape axis: rows_extra moves each read to the next instantiated rows-per-lane
      // (more padding rows, other registers and occupancy; the same bits).
      const bool up = tuning_.rows_extra != 0;
      auto single_up = [&](int rows) { return up && rows + 2 <= max_rows(Kind::kOneF32) ? rows + 2 : rows; };  // even, 10..20
      auto packed_up = [&](int rows) { return up && rows < 8 ? rows + 1 : rows; };
      for (; i < order.size() && packed_rows(len_of(order[i])) > 8; ++i) one(Kind::kOneF32, single_up(single_rows(len_of(order[i]))), i);
      for (; i < order.size(); i += 2) two(Kind::kPackedF32, packed_up(packed_rows(len_of(order[i]))), i);
    }
  });
  {
    std::vector<size_t> bin_size(by_bin.size(), 0);
    for (const auto& v : region_tasks)
      for (const RegionTask& t : v) ++bin_size[static_cast<size_t>(t.kind) * kRowBins + t.rows];
    for (size_t k = 0; k < by_bin.size(); ++k) by_bin[k].list.reserve(bin_size[k]);
  }
  for (const int g : region_order) {
    const uint64_t cost_cols = cost_of(g);
    const uint64_t fcols = plans[g].prog.fwd_columns, bcols = plans[g].prog.bwd_columns;
    for (const RegionTask& t : region_tasks[g]) {
      BinList& bl = bin_at(t.kind, t.rows);
      if (t.task.hap >= 0) {
        // An unshared strip-mined pair: read length x haplotype length forward cells.
        bl.list.push_back({t.cost, t.task});
        bl.fwd_cells += static_cast<uint64_t>(plans[g].haps[t.task.hap].len) * static_cast<uint64_t>(t.len);
        continue;
      }
      bl.list.push_back({cost_cols * static_cast<uint64_t>(t.rows), t.task});
      bl.fwd_cells += fcols * static_cast<uint64_t>(t.len);
      bl.bwd_cells += bcols * static_cast<uint64_t>(t.len);
    }
  }
  for (const BinList& bl : by_bin) {
    planned_.forward_cells += bl.fwd_cells;
    planned_.backward_cells += bl.bwd_cells;
  }
  planned_.computed_cells = planned_.forward_cells + planned_.backward_cells;
  std::vector<Task> tasks;
  std::vector<std::pair<uint64_t, Bin>> first;
  size_t n_tasks_all = 0;
  for (const BinList& bl : by_bin) n_tasks_all += bl.list.size();
  tasks.reserve(n_tasks_all);
  for (int kind = 0; kind < kKinds; ++kind)
    for (int rows = 0; rows < kRowBins; ++rows) {
      const BinList& bl = by_bin[static_cast<size_t>(kind) * kRowBins + rows];
      const auto& list = bl.list;
      if (list.empty()) continue;
      Bin b{static_cast<Kind>(kind), rows, static_cast<int>(tasks.size()), static_cast<int>(list.size()), 0, 0, 0};
      b.fwd_cells = bl.fwd_cells;
      b.bwd_cells = bl.bwd_cells;
      uint64_t cost = 0;
      for (auto& e : list) {
        tasks.push_back(e.second);
        cost += e.first;
      }
      const bool fp32 = b.kind == Kind::kPackedF32 || b.kind == Kind::kOneF32 || b.kind == Kind::kPackedF32Pd || b.kind == Kind::kOneF32Pd;
      b.warps = fp32 ? tuning_.warps_per_block : kWarpsPerBlock;
      int per_sm = 0, threads = 0;
      occupancy(b.kind, b.rows, &per_sm, &threads, b.warps);
      if (per_sm <= 0) return fail(FGKL_E_CUDA, "kernel instantiation unavailable on this device");
      const int grid = std::max(sms_, per_sm * sms_ * tuning_.grid_percent / 100);
      b.blocks = std::max(1, std::min((b.n_tasks + b.warps - 1) / b.warps, grid));
      first.push_back({cost, b});
    }
  // The bin with the most work launches first; the others fill the SMs its tail frees.
  std::stable_sort(first.begin(), first.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  for (auto& f : first) bins_.push_back(f.second);
  // Recomputation queues: room for every (read, distinct haplotype) pair of each rows-per-lane bin.
  // Pairs either pass loses (an FP32 underflow, or a joined FP64 result below the backward range)
  // are recomputed in FP64 (lib.rs:461-520): after an FP32 pass, a read lost against a third of its
  // haplotypes or more once with its region's shared program, any pair that sweep loses again and
  // every other lost pair without sharing, which cannot lose a pair.
  const bool queue_on = cfg.double_fallback;
  std::vector<int> queue_off(kQueueBins + 1, 0);
  {
    int64_t acc = 0;
    for (int r = 0; r < kQueueBins; ++r) {
      queue_off[r] = static_cast<int>(acc);
      if (queue_on) acc += queue_cap[r];
    }
    if (acc > INT32_MAX) return fail(FGKL_E_INVALID_ARGUMENT, "batch too large for the recomputation queue; split it");
    queue_off[kQueueBins] = static_cast<int>(acc);
  }
  if (queue_on) {
    for (int q = 1; q < kQueueBins; ++q) {
      const int cap = queue_off[q + 1] - queue_off[q];
      if (cap == 0) continue;
      // Queue bin -> the FP64 form of the pairs it holds (queue_bin).
      const int r = queue_bin_rows(q);
      const Kind kind = q >= 2 * kRowBins ? Kind::kGenericF64Pd
                                          : (q >= kRowBins ? (pd ? Kind::kLongF64Pd : Kind::kLongF64) : (pd ? Kind::kOneF64Pd : Kind::kOneF64));
      int per_sm = 0, threads = 0;
      occupancy(kind, r, &per_sm, &threads);
      if (per_sm <= 0) return fail(FGKL_E_CUDA, "recomputation kernel unavailable on this device");
      Bin b{kind, r, queue_off[q], cap, 0, 0, 0};
      b.queue_bin = q;
      b.blocks = std::max(1, std::min((cap + kWarpsPerBlock - 1) / kWarpsPerBlock, per_sm * sms_));
      rescue_bins_.push_back(b);
    }
  }
  // Bins of one pass run concurrently, so each owns a slice of the scratch.
  size_t scratch_total = 256;
  for (auto* list : {&bins_, &rescue_bins_}) {
    const bool rescue = list == &rescue_bins_;
    size_t off = 0;
    for (Bin& b : *list) {
      // Short-read recomputation bins also run dense reads' whole programs after an FP32 pass.
      const bool whole = !rescue || !cfg.double_precision;
      b.stride = align_up(is_long(b.kind) ? long_scratch_bytes(b.kind, b.rows, max_hap_len)
                          : whole         ? scratch_bytes(b.kind, b.rows, max_slots, max_nodes, max_segs)
                                          : scratch_bytes(b.kind, b.rows, 0, 0, 1));
      b.scratch_off = off;
      off += static_cast<size_t>(b.blocks) * b.warps * b.stride;
    }
    scratch_total = std::max(scratch_total, off);
  }

  // Plan blob: regions | haps | stream | segs | sweeps | code tables | haplotype codes | PD entries | PD signatures.
  size_t o_regions, o_haps, o_stream, o_segs, o_sweeps, o_codes, o_seq, o_pd_seq, o_sigs, blob_bytes = 0;
  auto section = [&](size_t bytes, size_t& off) {
    off = align_up(blob_bytes, 16);
    blob_bytes = off + bytes;
  };
  section(regions.size() * sizeof(Region), o_regions);
  section(static_cast<size_t>(n_haps) * sizeof(HapInfo), o_haps);
  section(static_cast<size_t>(n_stream) * sizeof(uint32_t), o_stream);
  section(static_cast<size_t>(n_segs) * sizeof(Segment), o_segs);
  section(static_cast<size_t>(n_sweeps) * sizeof(Sweep), o_sweeps);
  section(static_cast<size_t>(N) * 256, o_codes);
  section(static_cast<size_t>(n_seq) + 16, o_seq);
  section(static_cast<size_t>(n_pd_seq) * sizeof(uint32_t) + 16, o_pd_seq);
  section(static_cast<size_t>(n_sigs) * sizeof(uint32_t) + 16, o_sigs);

  // Device buffers.
  n_small_ = static_cast<int>(bins_.size() + rescue_bins_.size()) + 2 * kQueueBins + 1;
  if (!grow(d_reads_, cap_reads_, static_cast<size_t>(read_bytes) * 5 + 16) ||
      !grow(d_read_off_, cap_read_off_, static_cast<size_t>(total_reads) + 1) || !grow(d_plan_, cap_plan_, blob_bytes) ||
      !grow(d_tasks_, cap_tasks_, tasks.size() + 1) || !grow(d_queue_, cap_queue_, static_cast<size_t>(queue_off[kQueueBins]) + 1) ||
      !grow(d_small_, cap_small_, static_cast<size_t>(n_small_)) || !grow(d_out_, cap_out_, static_cast<size_t>(out_len_) + 1) ||
      !grow(d_scratch_, cap_scratch_, scratch_total))
    return fail(FGKL_E_OUT_OF_MEMORY, "device allocation failed");

  // Pinned staging (the reads have their own buffer): read offsets | plan | tasks | queue offsets |
  // results | counters.
  const size_t s_read_off = 0;
  const size_t s_blob = s_read_off + align_up((total_reads + 1) * sizeof(int64_t));
  const size_t s_tasks = s_blob + align_up(blob_bytes);
  const size_t s_qoff = s_tasks + align_up(tasks.size() * sizeof(Task));
  const size_t s_out = s_qoff + align_up((kQueueBins + 1) * sizeof(int));
  const size_t stage_bytes = s_out + align_up(static_cast<size_t>(out_len_) * sizeof(double)) + align_up(sizeof(Counters));
  if (over_allocation_limit(stage_bytes)) return fail(FGKL_E_OUT_OF_MEMORY, "pinned host allocation failed");
  if (stage_bytes > cap_stage_) {
    // Grown by half again at least, as the device buffers are (cudaFreeHost waits for the device).
    const size_t want = cap_stage_ > 0 ? std::max(stage_bytes, cap_stage_ + cap_stage_ / 2) : stage_bytes;
    if (h_stage_) cudaFreeHost(h_stage_);
    h_stage_ = nullptr;
    if (pinned_alloc(reinterpret_cast<void**>(&h_stage_), want) == cudaSuccess) {
      cap_stage_ = want;
    } else if (want > stage_bytes && (cudaGetLastError(), pinned_alloc(reinterpret_cast<void**>(&h_stage_), stage_bytes) == cudaSuccess)) {
      cap_stage_ = stage_bytes;
    } else {
      cudaGetLastError();
      cap_stage_ = 0;
      h_stage_ = nullptr;
      return fail(FGKL_E_OUT_OF_MEMORY, "pinned host allocation failed");
    }
  }
  out_stage_ = s_out;
  uint8_t* const st = h_stage_;
  std::memcpy(st + s_read_off, in.read_off, (total_reads + 1) * sizeof(int64_t));
  {
    uint8_t* blob = st + s_blob;
    std::memcpy(blob + o_regions, regions.data(), regions.size() * sizeof(Region));
    uint32_t* stream = reinterpret_cast<uint32_t*>(blob + o_stream);
    std::memset(stream, 0, kStreamPad * sizeof(uint32_t));
    std::memset(blob + o_seq + n_seq, 0, 16);
    std::memset(blob + o_pd_seq + n_pd_seq * sizeof(uint32_t), 0, 16);
    std::memset(blob + o_sigs + n_sigs * sizeof(uint32_t), 0, 16);
    parallel_for(N, std::min(host_threads(), (N + 31) / 32), [&](int64_t g) {
      const RegionPlan& rp = plans[g];
      const Region& R = regions[g];
      if (!rp.haps.empty()) std::memcpy(blob + o_haps + static_cast<size_t>(R.hap_off) * sizeof(HapInfo), rp.haps.data(), rp.haps.size() * sizeof(HapInfo));
      auto put = [&](const std::vector<uint32_t>& v, int32_t off) {
        if (!v.empty()) std::memcpy(stream + off, v.data(), v.size() * sizeof(uint32_t));
        std::memset(stream + off + v.size(), 0, kStreamPad * sizeof(uint32_t));
      };
      put(rp.prog.fwd, R.prog.fwd_off);
      put(rp.prog.bwd, R.prog.bwd_off);
      if (!rp.prog.segs.empty())
        std::memcpy(blob + o_segs + static_cast<size_t>(R.prog.seg_off) * sizeof(Segment), rp.prog.segs.data(), rp.prog.segs.size() * sizeof(Segment));
      if (!rp.prog.sweeps.empty())
        std::memcpy(blob + o_sweeps + static_cast<size_t>(R.prog.sweep_off) * sizeof(Sweep), rp.prog.sweeps.data(), rp.prog.sweeps.size() * sizeof(Sweep));
      if (!rp.haps.empty()) std::memcpy(blob + o_codes + static_cast<size_t>(g) * 256, rp.codes, 256);
      else std::memset(blob + o_codes + static_cast<size_t>(g) * 256, 0, 256);
      if (!rp.seq.empty()) std::memcpy(blob + o_seq + R.seq_off, rp.seq.data(), rp.seq.size());
      if (!rp.pd_seq.empty())
        std::memcpy(blob + o_pd_seq + static_cast<size_t>(R.seq_off) * sizeof(uint32_t), rp.pd_seq.data(), rp.pd_seq.size() * sizeof(uint32_t));
      if (!rp.pd_sigs.empty())
        std::memcpy(blob + o_sigs + static_cast<size_t>(R.sig_off) * sizeof(uint32_t), rp.pd_sigs.data(), rp.pd_sigs.size() * sizeof(uint32_t));
    });
  }
  if (!tasks.empty()) std::memcpy(st + s_tasks, tasks.data(), tasks.size() * sizeof(Task));
  std::memcpy(st + s_qoff, queue_off.data(), (kQueueBins + 1) * sizeof(int));

  read_copy.join();
  planned_.host_pack_ms = ms_since(t_pack);
  const auto t_up = std::chrono::steady_clock::now();
  int rc;
  if (!direct_reads && (rc = check(cudaMemcpyAsync(d_reads_, h_reads_, static_cast<size_t>(read_bytes) * 5, cudaMemcpyHostToDevice, copy_),
                                   "upload reads")))
    return rc;
  if ((rc = check(cudaMemcpyAsync(d_read_off_, st + s_read_off, (total_reads + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, copy_),
                  "upload offsets")))
    return rc;
  if ((rc = check(cudaMemcpyAsync(d_plan_, st + s_blob, blob_bytes, cudaMemcpyHostToDevice, copy_), "upload plan"))) return rc;
  if (!tasks.empty() &&
      (rc = check(cudaMemcpyAsync(d_tasks_, st + s_tasks, tasks.size() * sizeof(Task), cudaMemcpyHostToDevice, copy_), "upload tasks")))
    return rc;
  if ((rc = check(cudaMemcpyAsync(d_small_ + (n_small_ - 2 * kQueueBins - 1), st + s_qoff, (kQueueBins + 1) * sizeof(int),
                                  cudaMemcpyHostToDevice, copy_),
                  "upload queue offsets")))
    return rc;
  if ((rc = check(cudaEventRecord(uploaded_, copy_), "upload event"))) return rc;
  // Uploaded from the caller's own memory: done before returning, so the caller may reuse it.
  if (direct_reads) {
    upload_guard.s = nullptr;
    if ((rc = check(cudaEventSynchronize(uploaded_), "upload reads"))) return rc;
  }

  planned_.host_upload_ms = ms_since(t_up);
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
  view_.hap_codes = d_plan_ + o_seq;
  view_.pd_entries = reinterpret_cast<const uint32_t*>(d_plan_ + o_pd_seq);
  view_.pd_sigs = reinterpret_cast<const uint32_t*>(d_plan_ + o_sigs);
  view_.err_prob = d_err_;
  view_.m2m = d_m2m_;
  view_.out = d_out_;
  view_.counters = d_counters_;
  (void)total_haps;
  return FGKL_OK;
}

int Engine::begin_run() {
  DeviceGuard device_guard(device_);
  return check(cudaStreamWaitEvent(stream_, uploaded_, 0), "wait for the uploads");
}

int Engine::end_run() {
  DeviceGuard device_guard(device_);
  return check(cudaEventRecord(computed_, stream_), "kernels event");
}

int Engine::run() {
  DeviceGuard device_guard(device_);
  int rc;
  int* counters = d_small_;                                // one per launch
  int* queue_off = d_small_ + (n_small_ - 2 * kQueueBins - 1);  // kQueueBins + 1 entries, uploaded by prepare
  int* queue_tail = d_small_ + (n_small_ - kQueueBins);
  const size_t n_launch = bins_.size() + rescue_bins_.size();
  if ((rc = check(cudaMemsetAsync(counters, 0, n_launch * sizeof(int), stream_), "reset task counters"))) return rc;
  if ((rc = check(cudaMemsetAsync(queue_tail, 0, kQueueBins * sizeof(int), stream_), "reset queues"))) return rc;
  if ((rc = check(cudaMemsetAsync(d_counters_, 0, sizeof(Counters), stream_), "reset counters"))) return rc;
  planned_.kernel_launches = 0;
  int i = 0;
  if (profile_) {
    const size_t need = 2 * (bins_.size() + rescue_bins_.size() + 1);
    while (ev_.size() < need) {
      cudaEvent_t e;
      if ((rc = check(cudaEventCreate(&e), "profiling event"))) return rc;
      ev_.push_back(e);
    }
  }
  // Each pass forks its bins onto the auxiliary streams and joins them back.
  auto pass = [&](const std::vector<Bin>& list, bool rescue) -> int {
    if (list.empty()) return FGKL_OK;
    if ((rc = check(cudaEventRecord(fork_, stream_), "fork"))) return rc;
    for (size_t b = 0; b < list.size(); ++b) {
      const Bin& bin = list[b];
      // Profiled runs serialise the launches on the main stream so each one's events time it alone.
      const int lanes = std::max(1, std::min(tuning_.streams, kAuxStreams));
      cudaStream_t s = profile_ ? stream_ : aux_[b % lanes];
      if ((rc = check(cudaStreamWaitEvent(s, fork_, 0), "fork wait"))) return rc;
      LaunchArgs a{};
      a.v = view_;
      a.tasks = (rescue ? d_queue_ : d_tasks_) + bin.task_off;
      a.n_tasks = bin.n_tasks;
      a.count = rescue ? queue_tail + bin.queue_bin : nullptr;
      a.task_counter = counters + i++;
      a.scratch = d_scratch_ + bin.scratch_off;
      a.scratch_stride = bin.stride;
      a.min_accept_plain = (!rescue && !cfg_.double_precision) ? 1 : 0;
      a.only_lost = rescue ? 1 : 0;
      const int li = i - 1;  // this launch's index, for profiling events
      if (profile_ && (rc = check(cudaEventRecord(ev_[2 * li], s), "profiling event"))) return rc;
      if ((rc = check(launch(bin.kind, bin.rows, bin.blocks, a, s, bin.warps), rescue ? "recomputation launch" : "first-pass launch")))
        return rc;
      if (profile_ && (rc = check(cudaEventRecord(ev_[2 * li + 1], s), "profiling event"))) return rc;
      planned_.kernel_launches++;
      if ((rc = check(cudaEventRecord(join_[b % lanes], s), "join"))) return rc;
    }
    const size_t used = std::min<size_t>(list.size(), static_cast<size_t>(std::max(1, std::min(tuning_.streams, kAuxStreams))));
    for (size_t b = 0; b < used; ++b)
      if ((rc = check(cudaStreamWaitEvent(stream_, join_[b], 0), "join wait"))) return rc;
    return FGKL_OK;
  };
  if ((rc = pass(bins_, false))) return rc;
  if (!rescue_bins_.empty()) {
    CollectArgs c{view_, d_queue_, queue_off, queue_tail, cfg_.double_precision ? 0 : 1};
    if ((rc = check(launch_collect(c, n_regions_, stream_), "lost-pair collection"))) return rc;
    planned_.kernel_launches++;
  }
  if ((rc = pass(rescue_bins_, true))) return rc;
  return FGKL_OK;
}

void Engine::set_tuning(const Tuning& t) {
  tuning_.streams = std::max(1, std::min(t.streams, kAuxStreams));
  tuning_.grid_percent = std::max(10, std::min(t.grid_percent, 100));
  tuning_.reads_per_warp = t.reads_per_warp == 1 ? 1 : 2;
  tuning_.rows_extra = t.rows_extra ? 1 : 0;
  tuning_.warps_per_block = (t.warps_per_block == 1 || t.warps_per_block == 2) ? t.warps_per_block : kWarpsPerBlock;
}

int Engine::time_run(int repeats, double* ms) {
  DeviceGuard device_guard(device_);
  if (repeats < 1) repeats = 1;
  int rc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if ((rc = check(cudaEventCreate(&e0), "timing event")) || (rc = check(cudaEventCreate(&e1), "timing event"))) return rc;
  std::vector<double> t;
  for (int i = 0; i <= repeats && rc == FGKL_OK; ++i) {
    if ((rc = begin_run())) break;
    if ((rc = check(cudaEventRecord(e0, stream_), "timing event"))) break;
    if ((rc = run())) break;
    if ((rc = check(cudaEventRecord(e1, stream_), "timing event"))) break;
    if ((rc = end_run())) break;
    if ((rc = check(cudaEventSynchronize(e1), "timed run"))) break;
    float f = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    if (i > 0) t.push_back(f);  // the first run is a warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return FGKL_OK;
}

int Engine::bin_profile(std::vector<BinProfile>* out) {
  DeviceGuard device_guard(device_);
  out->clear();
  if (!profile_) return fail(FGKL_E_INVALID_ARGUMENT, "profiling is off");
  int rc;
  if ((rc = check(cudaStreamSynchronize(stream_), "profiled run"))) return rc;
  int i = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (const Bin& b : pass == 0 ? bins_ : rescue_bins_) {
      float ms = 0.f;
      if (2 * i + 1 < static_cast<int>(ev_.size())) cudaEventElapsedTime(&ms, ev_[2 * i], ev_[2 * i + 1]);
      out->push_back(BinProfile{static_cast<int>(b.kind), b.rows, b.n_tasks, b.blocks, pass, b.fwd_cells, b.bwd_cells, ms});
      ++i;
    }
  return FGKL_OK;
}

int Engine::fetch(double* out, int64_t out_len, BatchStats* stats) {
  DeviceGuard device_guard(device_);
  const auto t_fetch = std::chrono::steady_clock::now();
  if (out_len != out_len_)
    return fail(FGKL_E_OUTPUT_LENGTH, "output has " + std::to_string(out_len) + " elements but reads x haplotypes is " +
                                          std::to_string(out_len_));
  int rc;
  double* h_out = reinterpret_cast<double*>(h_stage_ + out_stage_);
  Counters* h_cnt = reinterpret_cast<Counters*>(h_stage_ + out_stage_ + align_up(static_cast<size_t>(out_len_) * sizeof(double)));
  if ((rc = check(cudaStreamWaitEvent(copy_, computed_, 0), "wait for the kernels"))) return rc;
  // Results go straight into a page-locked output array, else through pinned staging.
  const size_t out_bytes = static_cast<size_t>(out_len_) * sizeof(double);
  const bool direct_out = out_len_ > 0 && host_pinned(out, out_bytes);
  if (out_len_ > 0 &&
      (rc = check(cudaMemcpyAsync(direct_out ? out : h_out, d_out_, out_bytes, cudaMemcpyDeviceToHost, copy_), "download results")))
    return rc;
  if ((rc = check(cudaMemcpyAsync(h_cnt, d_counters_, sizeof(Counters), cudaMemcpyDeviceToHost, copy_), "download counters")))
    return rc;
  if ((rc = check(cudaEventRecord(fetched_, copy_), "download event"))) return rc;
  if ((rc = check(cudaEventSynchronize(fetched_), "kernel execution"))) return rc;
  if (out_len_ > 0 && !direct_out) parallel_copy(reinterpret_cast<uint8_t*>(out), reinterpret_cast<const uint8_t*>(h_out), out_bytes);
  planned_.host_fetch_ms = ms_since(t_fetch);
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
  if ((rc = begin_run()) || (rc = run()) || (rc = end_run())) return rc;
  return fetch(out, out_len, stats);
}

}  // namespace fgkl
